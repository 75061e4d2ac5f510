"""The reverse sweep of single (omega, l) pairs (ysg_pair_adjoint.cuh, the
code of k_solve_adjoint.cu) against the tangent-linear pair solve, on the
CPU: tests/device_on_host/pair_adjoint_check.cpp compiles the device solver
headers as host C++ (the looped-step form the sweep kernel uses) and
compares <dL/d(knot arrays), d> from the reverse sweep with the directional
derivative of the same pair solve in dual numbers, for radial, toroidal and
spheroidal pairs from l = 0 to lmax, with self-gravitation, in the Cowling
approximation and without gravity, with a solid or a fluid inner core and
with or without an ocean, receivers above and below the source, to 1e-9
relative.  The GPU form of the
same comparison, through the whole gradient pipeline, is
tests/test_gpu_reverse.py."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = Path(__file__).resolve().parent / "device_on_host"
LIBDIR = ROOT / "yspec_b200" / "lib"
CUDA_INC = Path("/usr/local/cuda/include")

CASES = [
    ("c1", {}),
    ("c4", {}),
    ("c4", {"out": 2, "cor": 1}),
    ("c4", {"out": 1, "depth_r": 50.0}),
    ("c1", {"model_file": "model200_ocean.deck", "depth_r": 3.0, "ats": 1}),
    ("c1", {"model_file": "model200_fic.deck", "depth_r": 3.0, "ats": 1, "out": 2, "cor": 1}),
    ("c1", {"grav": 1, "ats": 1}),
    ("c1", {"grav": 0, "ats": 1, "out": 2, "cor": 1}),
    ("c1", {"grav": 1, "model_file": "model200_ocean.deck", "depth_r": 3.0}),
    ("c1", {"grav": 0, "model_file": "model200_fic.deck", "depth_r": 3.0, "ats": 1}),
    # receivers below the source
    ("c4", {"depth_s": 20.0, "depth_r": 250.0}),
    ("c1", {"grav": 1, "depth_s": 20.0, "depth_r": 250.0, "ats": 1}),
    ("c1", {"grav": 0, "depth_s": 20.0, "depth_r": 250.0, "ats": 1, "out": 2, "cor": 1}),
    ("c1", {"model_file": "model200_ocean.deck", "depth_s": 3.0, "depth_r": 250.0, "ats": 1}),
    ("c1", {"model_file": "model200_fic.deck", "depth_s": 3.0, "depth_r": 250.0, "ats": 1, "out": 2, "cor": 1}),
    ("c1", {"grav": 1, "model_file": "model200_ocean.deck", "depth_s": 3.0, "depth_r": 250.0}),
    ("c1", {"grav": 0, "model_file": "model200_fic.deck", "depth_s": 3.0, "depth_r": 250.0, "ats": 1}),
]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not (CUDA_INC / "cuda_runtime.h").exists():
        pytest.skip("g++ or the CUDA headers missing")
    if not (LIBDIR / "libyspec_b200.so").exists():
        pytest.fail("native library not built (python -m yspec_b200.build)")
    out = tmp_path_factory.mktemp("adjoint_host") / "pair_adjoint_check"
    cmd = [gxx, "-std=c++17", "-O1", "-ffp-contract=off", "-DYSG_LOOPED_STEP=1",
           "-include", str(SRC / "host_shim.h"), f"-I{CUDA_INC}", f"-I{ROOT / 'yspec_b200' / 'csrc'}",
           f"-I{ROOT / 'include'}", str(SRC / "pair_adjoint_check.cpp"), "-o", str(out),
           f"-L{LIBDIR}", "-lyspec_b200", f"-Wl,-rpath,{LIBDIR}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    return out


@pytest.mark.parametrize("cfg,over", CASES)
def test_pair_adjoint_matches_tangent(checker, tmp_path, cfg, over):
    from yspec_b200 import workloads as W

    over = dict(over)
    if "model_file" in over:
        over["model_file"] = str(W.GOLDEN / over["model_file"])
    pf = W.config(cfg, seed=0, **over)[0].write(tmp_path / f"{cfg}.in")
    res = subprocess.run([str(checker), str(pf)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-2000:]
    worst = float(res.stdout.strip().splitlines()[-1].split()[-1])
    assert worst < 1e-9
