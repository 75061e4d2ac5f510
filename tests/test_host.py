"""Host side of the yspec program (C++ mirror of the Fortran host) on CPU.

The host code that stays on the CPU (parameter file, model deck with its
normalisation, splines and gravity, event set-up, writer) must agree bit for
bit with the oracle, and the library must export every C-ABI symbol the
headers declare.  No GPU is needed; device entry points report NO_DEVICE.
"""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import yo
from conftest import ROOT, has_gpu
from yspec_b200 import Event, Model, Params, native as N, workloads as W

DECKS = ["model200.deck", "model400.deck", "model200_ocean.deck", "model200_fic.deck"]
ARRAYS = ["r", "rho", "rho_cs", "acon", "acon_cs", "ccon", "ccon_cs", "fcon", "fcon_cs", "lcon",
          "lcon_cs", "ncon", "ncon_cs", "kappa", "kappa_cs", "mu", "mu_cs", "qkappa", "qkappa_cs",
          "qmu", "qmu_cs", "grav", "grav_cs", "xlam", "xlam_cs", "xa2", "xa2_cs", "alpha", "beta"]


def test_library_exports_every_declared_symbol():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(ys[gh]_[a-z0-9_]+)\s*\(", txt))
    assert len(names) > 30
    L = N.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_output_array_lengths_match_header():
    """The buffers the Python API hands to the engine's fill-in entry points
    are as long as the arrays include/yspec_gpu.h declares: a shorter one
    would be written past its end."""
    from yspec_b200 import api
    txt = (ROOT / "include" / "yspec_gpu.h").read_text()
    want = {"ysg_last_timings": api.N_STAGE_TIMES, "ysg_last_schedule": api.N_SCHEDULES}
    for fn, n in want.items():
        m = re.search(fn + r"\([^)]*\bfloat\s+\w+\[(\d+)\]\)", txt)
        assert m, fn
        assert int(m.group(1)) == n, fn


@pytest.mark.parametrize("deck", DECKS)
def test_model_bit_identical_to_oracle(workdir, deck):
    p = W.config("c1", seed=2, model_file=str(W.GOLDEN / deck), depth_r=3.0)[0]
    P = yo.Problem(p.write(workdir / "m.in"))
    m = Model(p.model_file)
    for name in ARRAYS:
        np.testing.assert_array_equal(m.array(name), P.array(name), err_msg=name)
    v = m.view()
    assert (v.nknot, v.nic, v.noc, v.nsl, v.ocean, v.fic) == (
        P.model.nknot, P.model.nic, P.model.noc, P.model.nsl, P.model.ocean, P.model.fic)
    assert v.tref == P.model.tref


@pytest.mark.parametrize("cfg", ["c1", "c2", "c4"])
def test_event_setup_bit_identical_to_oracle(workdir, cfg):
    p = W.config(cfg, seed=9)[0]
    pf = p.write(workdir / "e.in")
    P = yo.Problem(pf)
    ev = Event(Model(p.model_file), Params(pf))
    g = P.grid
    e, t = ev.ev, ev.tm
    assert (e.nw, e.is_, e.ir, t.nt, t.i1, t.i2) == (g.nw, g.is_, g.ir, g.nt, g.i1, g.i2)
    assert (e.wmin, e.dw, e.ep, e.rs, e.rr) == (g.wmin, g.dw, g.ep, g.rs, g.rr)
    assert (t.df, t.dt, t.tout, t.f11, t.f12, t.f21, t.f22) == (g.df, g.dt, g.tout, g.f11, g.f12, g.f21, g.f22)
    assert list(e.mm) == list(g.mm)
    d, azep, azst = P.geometry()
    nr = ev.nr
    np.testing.assert_array_equal(np.ctypeslib.as_array(ev.raw.delta, (nr,)), d)
    np.testing.assert_array_equal(np.ctypeslib.as_array(ev.raw.azep, (nr,)), azep)
    np.testing.assert_array_equal(np.ctypeslib.as_array(ev.raw.azst, (nr,)), azst)


def _param_text_variants(model):
    """Parameter files exercising list-directed reads: comment lines are
    skipped positionally, a value may sit after blank records, quoted
    strings may hold '/', an unquoted '/' ends the read."""
    p = W.Params(model_file=str(model), receivers=[(0.0, 10.0), (-20.5, 33.0), (45.0, -170.0)])
    base = p.text()
    blank_before_receivers = base.replace("# receiver latitudes and longitudes\n",
                                          "# receiver latitudes and longitudes\n \n")
    return {"plain": base, "blank_records": blank_before_receivers,
            "slash_prefix": base.replace("  yspec.out", "  run/out.x")}


@pytest.mark.parametrize("variant", ["plain", "blank_records", "slash_prefix"])
def test_params_match_oracle(workdir, variant):
    txt = _param_text_variants(W.MODEL200)[variant]
    pf = workdir / "p.in"
    pf.write_text(txt)
    P = yo.Problem(pf)
    got = Params(pf)
    o = P.params
    for f in ("ats", "grav", "out", "cor", "lmin", "lmax", "f1", "f2", "tout", "dt", "f11", "f12",
              "f21", "f22", "depth_s", "lat_s", "lon_s", "depth_r", "nr"):
        assert getattr(got, f) == getattr(o, f), f
    assert got.pref_out == o.pref_out.decode() and got.model_file == o.model_file.decode()
    assert list(got.raw.mm) == list(o.mm)
    nr = o.nr
    assert np.ctypeslib.as_array(got.raw.lat_r, (nr,)).tolist() == np.ctypeslib.as_array(o.lat_r, (nr,)).tolist()
    if variant == "slash_prefix":
        assert got.pref_out == "run"            # '/' ends a list-directed read


def _status(model_file, **over):
    p = W.Params(model_file=str(model_file), **over)
    return p


@pytest.mark.parametrize("case,status", [
    (dict(model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_r=0.0), 110),   # receiver in ocean
    (dict(model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_s=1.0), 108),   # source in ocean
    (dict(depth_s=7000.0), 107),                                                  # source not in model
    (dict(fmax=60.0, dt=10.0), 105),                                              # Nyquist below fmax
])
def test_stop_conditions(workdir, case, status):
    p = W.Params(**case)
    pf = p.write(workdir / "s.in")
    m = Model(p.model_file)
    with pytest.raises(N.YspecError) as ei:
        Event(m, Params(pf))
    assert ei.value.status == status


def test_missing_files(workdir):
    with pytest.raises(N.YspecError) as ei:
        Params(workdir / "nope.in")
    assert ei.value.status == 101
    with pytest.raises(N.YspecError) as ei:
        Model(workdir / "nope.deck")
    assert ei.value.status == 103


@pytest.mark.parametrize("nout,nr", [(7, 12), (3, 1037)])
def test_writer_byte_identical_to_oracle(workdir, nout, nr):
    """The threaded writer (receivers' files on several threads) against the
    oracle's serial writer, byte for byte, including 4-digit file suffixes."""
    rng = np.random.default_rng(0)
    out = rng.normal(size=(nr, 4, nout)) * 10.0 ** rng.integers(-120, 120, size=(nr, 4, nout))
    out[0, 1, 0] = -0.0
    out[0, 2, 1] = 0.0
    out[1, 3, 2] = 9.9999995e-8          # rounds up across a decade
    out = np.ascontiguousarray(out)
    (workdir / "a").mkdir()
    (workdir / "b").mkdir()
    assert N.lib().ysh_write_traces(str(workdir / "a" / "syn").encode(), N.dptr(out), nout, nr) == 0
    assert yo.lib().yo_write_traces(str(workdir / "b" / "syn").encode(), yo._p(out), nout, nr) == 0
    names = sorted(x.name for x in (workdir / "a").iterdir())
    assert names == sorted(x.name for x in (workdir / "b").iterdir())
    assert "syn.1" in names and "syn.10" in names and "syn.12" in names
    for n in names:
        assert (workdir / "a" / n).read_bytes() == (workdir / "b" / n).read_bytes(), n
    line = (workdir / "a" / "syn.1").read_text().splitlines()[0]
    assert len(line) == 60 and line[15:30].strip().startswith("-0.000000E+00")


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    from yspec_b200 import Engine

    with pytest.raises(N.YspecError) as ei:
        Engine(0)
    assert ei.value.status == 6               # YSG_ERR_NO_DEVICE: no CPU fallback


def test_run_batch_reports_failing_file(workdir):
    """Several parameter files: every file is read before any device work,
    and a missing one is reported with its index (no GPU needed)."""
    from yspec_b200 import workloads as W

    p = W.config("c1", seed=1)[0]
    p.write(workdir / "a.in")
    files = (C.c_char_p * 3)(b"a.in", b"missing.in", b"a.in")
    failed = C.c_int(-2)
    rc = N.lib().ysh_run_batch(3, files, 0, 0, C.byref(failed))
    assert rc == 101 and failed.value == 1
    rc = N.lib().ysh_run_batch(0, files, 0, 0, C.byref(failed))
    assert rc != 0


def test_fortran_module_matches_the_c_abi():
    """include/yspec_gpu.f90 (no Fortran compiler here): every bind(C) name is
    exported by the library, and each derived type lists the C struct's
    fields in the C order (ctypes mirrors of include/yspec_gpu.h)."""
    import re

    from yspec_b200 import native as N

    src = (ROOT / "include" / "yspec_gpu.f90").read_text()
    names = re.findall(r'bind\(C, name="(\w+)"\)', src)
    assert len(names) >= 12
    lib = N.lib()
    for n in names:
        if n != "strlen":
            assert hasattr(lib, n), n
    for ftype, ctype in (("ysg_model", N.YsgModel), ("ysg_event", N.YsgEvent), ("ysg_time", N.YsgTime)):
        body = re.search(rf"type, bind\(C\) :: {ftype}\n(.*?)end type", src, re.S).group(1)
        fields = []
        for line in body.splitlines():
            line = line.split("!")[0]
            if "::" in line:
                fields += [re.sub(r"\(.*\)", "", f).strip() for f in line.split("::")[1].split(",")]
        want = [f.rstrip("_") for f, _ in ctype._fields_]
        assert fields == want, (ftype, fields, want)


def _e15_6_reference(x: float) -> str:
    """gfortran's E15.6 as the reference writes it: [-]0.dddddd E+ee, digits
    from the correctly rounded %.5e of |x|."""
    import math

    ax = abs(x)
    if ax == 0.0:
        dig, e10 = "000000", 0
    else:
        t = f"{ax:.5e}"
        dig = t[0] + t[2:7]
        e10 = int(t.split("e")[1]) + 1
    sg = "-" if math.copysign(1.0, x) < 0 else ""
    ae = abs(e10)
    body = (f"{sg}0.{dig}E{'-' if e10 < 0 else '+'}{ae:02d}" if ae <= 99
            else f"{sg}0.{dig}{'-' if e10 < 0 else '+'}{ae:03d}")
    return f"{body:>15.15}"


def test_e15_6_formatter_exact():
    """The writer's formatter (digits without snprintf where the rounding is
    certain) against correctly rounded %.5e on values of every magnitude,
    exact ties, values next to rounding boundaries and powers of ten."""
    import struct

    from yspec_b200 import native as N

    rng = np.random.default_rng(5)
    vals = list(rng.standard_normal(20000) * 10.0 ** rng.uniform(-40, 40, 20000))
    vals += list(rng.standard_normal(20000) * 10.0 ** rng.integers(-12, 4, 20000))
    vals += [0.0, -0.0, 1.0, -1.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
             1234565.0, 1234575.0, 12345650.0, 0.5, 2.5e-5, 999999.5, 9999995.0, 99999.95]
    for e in range(-30, 31):
        for m in (1.0, 9.999995, 9.9999949999, 9.99999500001, 1.0000005, 1.00000049999, 1.2345650):
            v = m * 10.0 ** e
            vals += [v, -v, np.nextafter(v, 0.0), np.nextafter(v, np.inf)]
    buf = C.create_string_buffer(16)
    for x in vals:
        x = float(x)
        N.lib().ysh_format_e15_6(x, buf)
        assert buf.value.decode() == _e15_6_reference(x), (x, struct.pack("<d", x).hex())
