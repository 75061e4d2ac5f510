"""yspec_b200 -- B200-native direct radial integration for YSpec-style synthetics.

The `yspec input.in` program with its parameter file, deck-format model and
per-receiver ASCII outputs, running the (omega,l) radial solves, the
receiver l-sum and the filter + inverse FFT on an sm_100a GPU through the
C-ABI declared in include/yspec_gpu.h.
"""
from .api import Engine, Event, Model, Params, fp64_peak_tflops, norms, run_file  # noqa: F401
from .native import LIB_PATH, YspecError, lib  # noqa: F401

__all__ = ["Engine", "Event", "Model", "Params", "fp64_peak_tflops", "norms", "run_file", "lib",
           "LIB_PATH", "YspecError"]
