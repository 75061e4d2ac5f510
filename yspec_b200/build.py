"""Build the native library, the `yspec` command and the CPU oracle in-tree.

    python -m yspec_b200.build            # incremental
    python -m yspec_b200.build --clean

Outputs (git-ignored, shipped with the source tree):
    yspec_b200/lib/libyspec_b200.so   C-ABI of include/yspec_gpu.h and include/yspec_host.h
    yspec_b200/bin/yspec              the `yspec input.in` command
    oracle/liboracle.so, oracle/yo_cli  CPU oracle (test infrastructure)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libyspec_b200.so"
BIN = PKG / "bin" / "yspec"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    f"-I{ROOT / 'include'}", f"-I{CSRC}", "--expt-relaxed-constexpr",
]
# files whose rounding must not be fused (see the file headers)
NO_FMA = {"k_legendre.cu"}

SOURCES = [
    CSRC / "capi.cu",
    CSRC / "k_solve_plain.cu",
    CSRC / "k_solve_batched.cu",
    CSRC / "k_solve_tangent.cu",
    CSRC / "k_solve_adjoint.cu",
    CSRC / "k_schedule.cu",
    CSRC / "k_legendre.cu",
    CSRC / "k_lsum.cu",
    CSRC / "k_ifft.cu",
    CSRC / "k_peak.cu",
    CSRC / "k_ifft_noalloc.cu",
    CSRC / "host" / "ysh_host.cpp",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: Path) -> list[Path]:
    hdrs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return [src] + hdrs


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _compile(src: Path) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not _stale(obj, _deps(src)):
        return obj
    flags = list(NVCC_FLAGS)
    if src.name in NO_FMA:
        flags.append("-fmad=false")
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu"] + flags + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [nvcc()] + flags + ["-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build_native(verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    BIN.parent.mkdir(parents=True, exist_ok=True)
    srcs = [s for s in SOURCES if s.exists()]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, srcs))
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + [
            "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    main_src = CSRC / "host" / "yspec_main.cpp"
    if main_src.exists() and _stale(BIN, [main_src, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(main_src), "-o", str(BIN),
               f"-L{LIB.parent}", "-lyspec_b200", "-Wl,-rpath,$ORIGIN/../lib"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"yspec link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_oracle() -> None:
    """Compile the CPU oracle (test infrastructure) with its Makefile."""
    res = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    a = ap.parse_args(argv)
    if a.clean and BUILD.exists():
        shutil.rmtree(BUILD)
    build_native(verbose=True)
    if not a.no_oracle:
        build_oracle()
    return 0


if __name__ == "__main__":
    sys.exit(main())
