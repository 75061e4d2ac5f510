"""The pair scheduler's cost model on the CPU: the count-only solve reads
the steps of whole knot intervals from a per-frequency prefix table
(k_step_prefix, k_schedule.cu) and computes only the two end intervals of
each integration.  tests/device_on_host/count_prefix_check.cpp compiles the
count-only solver headers as host C++ and compares, for every (omega, l)
pair and both parts of an event, each system class's step count with the
interval-by-interval loop: they must be equal (the schedule is built from
exact counts).  It also compares every start-level search the drivers make
(now reading 1/v^2 and r^2 from the knot records) with the search in its
direct form, which must pick the same level.  Events: c2 at size (1.23 M solve parts) and the branches
the drivers take (receiver below the source, fluid inner core, ocean,
Cowling and no gravity)."""
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
    ("c2", {}),
    ("c1", {"depth_s": 20.0, "depth_r": 250.0, "ats": 1}),
    ("c1", {"model_file": "model200_fic.deck", "depth_r": 3.0, "ats": 1}),
    ("c1", {"model_file": "model200_ocean.deck", "depth_r": 3.0, "grav": 1}),
    ("c1", {"model_file": "model200_fic.deck", "depth_s": 20.0, "depth_r": 250.0, "grav": 0}),
]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not (CUDA_INC / "cuda_runtime.h").exists():
        pytest.skip("g++ or the CUDA headers missing")
    if not (LIBDIR / "libyspec_b200.so").exists():
        pytest.fail("native library not built (python -m yspec_b200.build)")
    out = tmp_path_factory.mktemp("count_host") / "count_prefix_check"
    cmd = [gxx, "-std=c++17", "-O1", "-ffp-contract=off", "-DYSG_COUNT_ONLY=1",
           "-include", str(SRC / "host_shim.h"), f"-I{CUDA_INC}", f"-I{ROOT / 'yspec_b200' / 'csrc'}",
           f"-I{ROOT / 'include'}", str(SRC / "count_prefix_check.cpp"), "-o", str(out),
           f"-L{LIBDIR}", "-lyspec_b200", f"-Wl,-rpath,{LIBDIR}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    return out


@pytest.mark.parametrize("cfg,over", CASES)
def test_prefix_counts_equal_interval_loop(checker, tmp_path, cfg, over):
    from yspec_b200 import workloads as W

    over = dict(over)
    if "model_file" in over:
        over["model_file"] = str(W.GOLDEN / over["model_file"])
    pf = W.config(cfg, seed=0, **over)[0].write(tmp_path / f"{cfg}.in")
    res = subprocess.run([str(checker), str(pf)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-2000:]
    assert res.stdout.strip().splitlines()[-1].endswith("mismatches 0")
