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


def test_noalloc_rejects_oversize():
    t = N.YsgTime(nt=1 << 19, i1=2, i2=10, nr=1, df=1.0, dt=1.0, ep=1.0, tout=1.0)
    f = _bind()
    rc = f(C.byref(t), 1, 1, 1, 1, 1, None, None)      # pointers are never touched
    assert rc == 7                                      # YSG_ERR_LIMIT
