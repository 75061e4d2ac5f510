"""The `yspec` command on the GPU: same parameter file in, same
per-receiver ASCII files out.

The files are compared with the oracle's own command (`oracle/yo_cli`, the
CPU restatement of the reference program) after parsing: the E15.6 text
carries six significant digits, so the bar is the text's precision (a
field may differ by one unit in its last digit where the 1e-9 agreement
straddles a rounding boundary); file names, line counts and the time
column must be identical.  Several parameter files on one command line run
as one batch and must give the files each single run gives.
"""
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from yspec_b200 import workloads as W

pytestmark = pytest.mark.gpu

YSPEC = ROOT / "yspec_b200" / "bin" / "yspec"
YO_CLI = ROOT / "oracle" / "yo_cli"


def _params(seed, **over):
    base = dict(lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0, ats=1)
    base.update(over)
    p = W.config("c1", seed=seed, **base)[0]
    p.receivers = p.receivers[:3]
    return p


def _read(prefix, nr):
    out = []
    for k in range(1, nr + 1):
        rows = [[float(line[15 * c:15 * (c + 1)]) for c in range(4)]
                for line in open(f"{prefix}.{k}").read().splitlines()]
        out.append(np.array(rows))
    return out


def _same_text(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        np.testing.assert_array_equal(x[:, 0], y[:, 0])
        for c in range(1, 4):
            scale = np.max(np.abs(y[:, c])) or 1.0
            # one unit in the 6th significant digit of the largest sample
            assert np.max(np.abs(x[:, c] - y[:, c])) <= 1.0e-5 * scale


def _run(args, cwd):
    res = subprocess.run([str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr


def test_cli_matches_oracle_cli(workdir):
    p = _params(5, out=2, cor=1)
    (workdir / "g").mkdir()
    (workdir / "o").mkdir()
    p.pref_out = "g/syn"
    p.write(workdir / "g.in")
    p.pref_out = "o/syn"
    p.write(workdir / "o.in")
    _run([YSPEC, "g.in"], workdir)
    _run([YO_CLI, "o.in"], workdir)
    assert sorted(x.name for x in (workdir / "g").iterdir()) == \
        sorted(x.name for x in (workdir / "o").iterdir())
    _same_text(_read(workdir / "g" / "syn", 3), _read(workdir / "o" / "syn", 3))


def test_cli_batch_matches_single_runs(workdir):
    specs = [dict(seed=1), dict(seed=2, depth_s=400.0, out=1),
             dict(seed=3, grav=1, lmax=30, fmax=5.0, f21=3.5, f22=4.5),
             dict(seed=4, model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_r=3.0)]
    files = []
    for i, sp in enumerate(specs):
        sp = dict(sp)
        p = _params(sp.pop("seed"), **sp)
        for mode in ("batch", "single"):
            (workdir / f"{mode}{i}").mkdir()
            p.pref_out = f"{mode}{i}/syn"
            p.write(workdir / f"{mode}{i}.in")
        files.append(f"batch{i}.in")
        _run([YSPEC, f"single{i}.in"], workdir)
    _run([YSPEC] + files, workdir)          # two model decks: two batches
    for i in range(len(specs)):
        _same_text(_read(workdir / f"batch{i}" / "syn", 3), _read(workdir / f"single{i}" / "syn", 3))


def test_cli_reports_bad_file(workdir):
    p = _params(1)
    p.pref_out = "syn"
    p.write(workdir / "ok.in")
    res = subprocess.run([str(YSPEC), "ok.in", "missing.in"], cwd=workdir, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 1
    assert "missing.in" in res.stderr and "parameter file" in res.stderr


def test_cli_potential_files(workdir):
    """`yspec --potential input.in` writes prefix.pot.1 .. prefix.pot.nr, two
    E15.6 fields per line (time, potential), equal to the oracle's potential
    traces to the text's precision."""
    import yo

    p = _params(5, out=1)
    pf = p.write(workdir / "pot.in")
    res = subprocess.run([str(YSPEC), "--potential", str(pf)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    want = yo.Problem(pf).potential_traces(nthreads=8)
    for k in range(1, len(p.receivers) + 1):
        lines = open(f"{p.pref_out}.pot.{k}").read().splitlines()
        assert all(len(line) == 30 for line in lines)
        got = np.array([[float(line[15 * c:15 * (c + 1)]) for c in range(2)] for line in lines])
        assert got.shape == (want.shape[2], 2)
        np.testing.assert_allclose(got[:, 0], want[k - 1, 0], rtol=1e-6, atol=0)
        # one unit in the 6th significant digit of the largest sample, as above
        scale = np.abs(want[k - 1, 1]).max()
        assert np.abs(got[:, 1] - want[k - 1, 1]).max() <= 1e-5 * scale
