"""ysg_traces_noalloc: the time-series stage for callers that cannot let the
library allocate device memory (their host owns the GPU's memory, or an
allocation would synchronise the device).  It must give the traces of
ysg_event_traces, call after call, using only the buffers the caller passes
and the array compiled into the library.

Collected last on purpose (file name), and self-contained so it also passes
alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import yo
from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, native as N, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _bind():
    L = N.lib()
    f = L.ysg_traces_noalloc
    f.argtypes = [C.POINTER(N.YsgTime), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int), C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("cfg", [dict(), dict(ats=1, out=2, cor=1, dt=10.0, tout=60.0)])
def test_noalloc_traces_equal_allocating_path(workdir, cfg):
    import torch

    base = dict(lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)
    base.update(cfg)
    p = W.config("c1", seed=5, **base)[0]
    p.receivers = p.receivers[:5]
    pf = p.write(workdir / "na.in")
    model = Model(p.model_file)
    eng = Engine(0)
    eng.upload(model)
    ev = Event(model, Params(pf))
    ur, ut, up = eng.spectra(ev)                       # (nr, nw) complex, on the host
    want = eng.traces(ev)                              # allocating path: (nr, 4, nout)

    dev = torch.device("cuda", 0)
    def to_dev(a):
        return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).to(dev)
    d_ur, d_ut, d_up = to_dev(ur), to_dev(ut), to_dev(up)
    azep = np.ctypeslib.as_array(ev.raw.azep, shape=(ev.nr,)).copy()
    d_az = torch.from_numpy(azep).to(dev)
    nout = ev.nout()
    f = _bind()
    for call in range(2):                              # two calls in a row share the array
        d_out = torch.full((ev.nr, 4, nout), float("nan"), dtype=torch.float64, device=dev)
        n = C.c_int()
        torch.cuda.synchronize()
        rc = f(C.byref(ev.raw.tm), d_ur.data_ptr(), d_ut.data_ptr(), d_up.data_ptr(),
               d_az.data_ptr(), d_out.data_ptr(), C.byref(n), None)
        assert rc == 0, N.lib().ysh_status_string(rc)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert n.value == nout
        np.testing.assert_array_equal(got[:, 0], want[:, 0])
        for k in range(ev.nr):
            for c in range(1, 4):
                err = rel_l2(got[k, c], want[k, c])
                assert err <= TOL, f"call {call}: receiver {k} comp {c}: {err:.3e}"
    ref = yo.Problem(pf).run(nthreads=4)               # and directly against the oracle
    for k in range(ev.nr):
        for c in range(1, 4):
            assert rel_l2(got[k, c], ref[k, c]) <= TOL, (k, c)


def test_noalloc_rejects_oversize():
    t = N.YsgTime(nt=1 << 19, i1=2, i2=10, nr=1, df=1.0, dt=1.0, ep=1.0, tout=1.0)
    f = _bind()
    rc = f(C.byref(t), 1, 1, 1, 1, 1, None, None)      # pointers are never touched
    assert rc == 7                                      # YSG_ERR_LIMIT


def test_noalloc_rejects_short_transforms():
    t = N.YsgTime(nt=4, i1=2, i2=3, nr=1, df=1.0, dt=1.0, ep=1.0, tout=1.0)
    rc = _bind()(C.byref(t), 1, 1, 1, 1, 1, None, None)
    assert rc == 1                                      # YSG_ERR_ARG, as ysg_event_traces


def test_noalloc_many_receivers_short_transform():
    """nt = 8 fits 43,690 receivers of rows in the array but only 21,845 in
    one launch's grid (three rows per receiver): 22,000 receivers run in
    grid-sized chunks, and receivers either side of a chunk boundary equal a
    run of those receivers alone."""
    import torch

    dev = torch.device("cuda", 0)
    nr, nt, i1, i2 = 22000, 8, 2, 4
    nw = i2 - i1 + 1
    rng = np.random.default_rng(3)
    spec = [torch.from_numpy(rng.standard_normal((nr, nw, 2))).to(dev) for _ in range(3)]
    az = torch.from_numpy(rng.uniform(0, 2 * np.pi, nr)).to(dev)
    t = N.YsgTime(nt=nt, i1=i1, i2=i2, nr=nr, df=0.01, dt=5.0, ep=0.002, tout=30.0,
                  f11=0.0, f12=0.0, f21=0.0, f22=0.0, t_norm=1.0, amp_norm=1.0)
    f = _bind()
    n = C.c_int()
    rows = N.lib().ysg_trace_rows(C.byref(t))
    out = torch.zeros((nr, 4, rows), dtype=torch.float64, device=dev)
    rc = f(C.byref(t), *[x.data_ptr() for x in spec], az.data_ptr(), out.data_ptr(), C.byref(n), None)
    assert rc == 0
    torch.cuda.synchronize()
    pick = [0, 21844, 21845, 21999]
    t.nr = len(pick)
    sub = [x[pick].contiguous() for x in spec]
    out1 = torch.zeros((len(pick), 4, rows), dtype=torch.float64, device=dev)
    rc = f(C.byref(t), *[x.data_ptr() for x in sub], az[pick].contiguous().data_ptr(),
           out1.data_ptr(), C.byref(n), None)
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out[pick].cpu().numpy(), out1.cpu().numpy())
