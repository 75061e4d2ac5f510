"""The batched solve's b-vector responses from the transposed propagator,
on the CPU.  The batched form obtains each response row a pair uses from
one backward integration of the transposed b-vector system (sph_solver_g,
yint_T, rkck_step_loop_T in yspec_b200/csrc) instead of four forward
integrations, one per source jump (module_solver.f90:640-823,
1203-1382).  tests/device_on_host/bvec_transpose_check.cpp compiles the
shared-memory form and the plain form of the solver headers as host C++
and compares the ten spheroidal coefficients of every pair (l >= 1) at a
frequency stride, and one transposed Cash-Karp step against the forward
step's matrix.  Cases: the receiver above and below the source, the
acceleration with potential and tilt correction (three rows), a fluid inner
core, an ocean, no gravity and the Cowling approximation (the four-component
b-vector system of sph_solver_nc), and strided samples of the single event at scale and of a
deep-source batch event."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = Path(__file__).resolve().parent / "device_on_host"
LIBDIR = ROOT / "yspec_b200" / "lib"
CUDA_INC = Path("/usr/local/cuda/include")

BAND = {"lmax": 80, "fmax": 8.0, "f21": 6.0, "f22": 7.0}
CASES = [
    ("c1", dict(BAND, depth_s=20.0, depth_r=250.0, ats=1), 7),
    ("c1", dict(BAND, out=2, cor=1, ats=1), 7),
    ("c1", dict(BAND, model_file="model200_fic.deck", depth_s=20.0, depth_r=250.0, out=2, cor=1), 7),
    ("c1", dict(BAND, model_file="model200_ocean.deck", depth_r=3.0, ats=1), 7),
    ("c1", dict(BAND, model_file="model200_ocean.deck", depth_s=3.0, depth_r=250.0, ats=1, out=1), 7),
    ("c1", dict(BAND, grav=0, depth_s=20.0, depth_r=250.0, ats=1), 7),
    ("c1", dict(BAND, grav=1, model_file="model200_ocean.deck", depth_r=3.0, ats=1), 7),
    ("c1", dict(BAND, grav=1, model_file="model200_fic.deck", depth_s=20.0, depth_r=250.0), 7),
    ("c1", dict(BAND, grav=0, model_file="model200_fic.deck", depth_r=3.0, ats=1), 7),
    ("c2", {}, 205),
    ("c3", {}, 97),
]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not (CUDA_INC / "cuda_runtime.h").exists():
        pytest.skip("g++ or the CUDA headers missing")
    if not (LIBDIR / "libyspec_b200.so").exists():
        pytest.fail("native library not built (python -m yspec_b200.build)")
    d = tmp_path_factory.mktemp("bvec_transpose")
    flags = ["-std=c++17", "-O2", "-ffp-contract=off", "-include", str(SRC / "host_shim.h"),
             f"-I{CUDA_INC}", f"-I{ROOT / 'yspec_b200' / 'csrc'}", f"-I{ROOT / 'include'}"]
    src = str(SRC / "bvec_transpose_check.cpp")
    objs = []
    for part in (0, 1, 2):
        o = d / f"part{part}.o"
        res = subprocess.run([gxx] + flags + [f"-DBVT_PART={part}", "-c", src, "-o", str(o)],
                             capture_output=True, text=True)
        assert res.returncode == 0, res.stderr[-4000:]
        objs.append(str(o))
    out = d / "bvec_transpose_check"
    res = subprocess.run([gxx] + objs + ["-o", str(out), f"-L{LIBDIR}", "-lyspec_b200",
                                         f"-Wl,-rpath,{LIBDIR}"], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    return out


@pytest.mark.parametrize("cfg,over,stride", CASES)
def test_transposed_bvec_matches_forward(checker, tmp_path, cfg, over, stride):
    from yspec_b200 import workloads as W

    over = dict(over)
    if "model_file" in over:
        over["model_file"] = str(W.GOLDEN / over["model_file"])
    pf = W.config(cfg, seed=0, **over)[0].write(tmp_path / f"{cfg}.in")
    res = subprocess.run([str(checker), str(pf), str(stride)], capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-2000:]
    lines = res.stdout.strip().splitlines()
    assert float(lines[0].split()[-1]) < 1e-12      # one transposed step
    assert float(lines[-1].split()[-1]) < 1e-10     # worst pair
