"""ctypes bindings of the native library (include/yspec_gpu.h, include/yspec_host.h).

The library is built in-tree by ``python -m yspec_b200.build``.  There is no
CPU fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libyspec_b200.so"

_dp = C.POINTER(C.c_double)


class YsgModel(C.Structure):
    _fields_ = [
        ("nknot", C.c_int), ("nic", C.c_int), ("noc", C.c_int), ("nsl", C.c_int),
        ("ocean", C.c_int), ("fic", C.c_int),
        ("tref", C.c_double), ("pibigg", C.c_double), ("fre_norm", C.c_double),
        ("r", _dp), ("val", _dp * 13), ("cs", _dp * 13), ("alpha", _dp), ("beta", _dp),
    ]


class YsgEvent(C.Structure):
    _fields_ = [
        ("lmin", C.c_int), ("lmax", C.c_int), ("nw", C.c_int), ("is_", C.c_int), ("ir", C.c_int),
        ("ats", C.c_int), ("grav", C.c_int), ("out", C.c_int), ("cor", C.c_int), ("nr", C.c_int),
        ("jofs", C.c_int), ("jstride", C.c_int),
        ("wmin", C.c_double), ("dw", C.c_double), ("ep", C.c_double),
        ("rs", C.c_double), ("rr", C.c_double), ("mm", C.c_double * 6),
        ("delta", _dp), ("azst", _dp),
    ]


class YsgTime(C.Structure):
    _fields_ = [
        ("nt", C.c_int), ("i1", C.c_int), ("i2", C.c_int), ("nr", C.c_int),
        ("df", C.c_double), ("dt", C.c_double), ("ep", C.c_double), ("tout", C.c_double),
        ("f11", C.c_double), ("f12", C.c_double), ("f21", C.c_double), ("f22", C.c_double),
        ("t_norm", C.c_double), ("amp_norm", C.c_double), ("azep", _dp),
    ]


class YshParams(C.Structure):
    _fields_ = [
        ("pref_out", C.c_char * 256), ("model_file", C.c_char * 256),
        ("ats", C.c_int), ("grav", C.c_int), ("out", C.c_int), ("cor", C.c_int),
        ("lmin", C.c_int), ("lmax", C.c_int),
        ("f1", C.c_double), ("f2", C.c_double), ("tout", C.c_double), ("dt", C.c_double),
        ("f11", C.c_double), ("f12", C.c_double), ("f21", C.c_double), ("f22", C.c_double),
        ("depth_s", C.c_double), ("lat_s", C.c_double), ("lon_s", C.c_double),
        ("mm", C.c_double * 6), ("depth_r", C.c_double), ("nr", C.c_int),
        ("lat_r", _dp), ("lon_r", _dp),
    ]


class YshEvent(C.Structure):
    _fields_ = [
        ("ev", YsgEvent), ("tm", YsgTime), ("nt", C.c_int), ("i1", C.c_int), ("i2", C.c_int),
        ("delta", _dp), ("azst", _dp), ("azep", _dp),
    ]


class YshNorms(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "r_norm", "rho_norm", "vel_norm", "acl_norm", "fre_norm", "t_norm",
        "con_norm", "grav_norm", "moment_norm", "pot_norm", "pibigg")]


# Status of ysg_event_gradient for a path the reverse solver does not cover
# (include/yspec_gpu.h).
YSG_ERR_UNSUPPORTED = 8

# Symbols declared in include/*.h, checked by the CPU test suite.
EXPORTS = [
    "ysg_create", "ysg_model_upload", "ysg_model_tangent_upload", "ysg_model_tangents_upload", "ysg_event_spectra", "ysg_event_spectra_device",
    "ysg_event_traces", "ysg_trace_rows",
    "ysg_event_run", "ysg_event_prepare", "ysg_event_execute", "ysg_event_fetch", "ysg_get_stream",
    "ysg_batch_run", "ysg_event_coef", "ysg_event_gradient", "ysg_event_potential", "ysg_legendre_table", "ysg_set_solver", "ysg_set_schedule", "ysg_last_schedule",
    "ysg_last_timings", "ysg_last_work", "ysg_last_bytes", "ysg_last_launches", "ysg_fp64_peak", "ysg_status_string",
    "ysg_last_cuda_error", "ysg_destroy", "ysg_traces_noalloc",
    "ysh_norms_get", "ysh_read_params", "ysh_free_params", "ysh_read_model", "ysh_model_view",
    "ysh_model_nknot", "ysh_model_array", "ysh_free_model", "ysh_event_setup", "ysh_free_event",
    "ysh_write_traces", "ysh_format_e15_6", "ysh_run", "ysh_run_batch", "ysh_run_potential",
    "ysh_write_potential", "ysh_free", "ysh_status_string",
]

_lib = None


class YspecError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().ysh_status_string(status).decode()
        if status == 2:
            msg += ": " + lib().ysg_last_cuda_error().decode()
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Load the native library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"native library missing: {LIB_PATH} (run python -m yspec_b200.build)")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    L.ysg_create.argtypes = [C.POINTER(vp), C.c_int]
    L.ysg_model_upload.argtypes = [vp, C.POINTER(YsgModel)]
    L.ysg_model_tangent_upload.argtypes = [vp, C.POINTER(YsgModel)]
    L.ysg_model_tangents_upload.argtypes = [vp, C.c_int, C.POINTER(YsgModel)]
    L.ysg_event_spectra.argtypes = [vp, C.POINTER(YsgEvent), _dp, _dp, _dp]
    L.ysg_event_spectra_device.argtypes = [vp, C.POINTER(YsgEvent), vp, vp, vp]
    L.ysg_event_traces.argtypes = [vp, C.POINTER(YsgTime), _dp, C.POINTER(C.c_int)]
    L.ysg_traces_noalloc.argtypes = [C.POINTER(YsgTime)] + [vp] * 5 + [C.POINTER(C.c_int), vp]
    L.ysg_trace_rows.argtypes = [C.POINTER(YsgTime)]
    L.ysg_event_run.argtypes = [vp, C.POINTER(YsgEvent), C.POINTER(YsgTime), _dp, C.POINTER(C.c_int)]
    L.ysg_event_prepare.argtypes = [vp, C.POINTER(YsgEvent), C.POINTER(YsgTime)]
    L.ysg_event_execute.argtypes = [vp]
    L.ysg_event_fetch.argtypes = [vp, _dp, C.POINTER(C.c_int)]
    L.ysg_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.ysg_batch_run.argtypes = [vp, C.c_int, C.POINTER(YsgEvent), C.POINTER(YsgTime),
                                C.POINTER(_dp), C.POINTER(C.c_int)]
    L.ysg_event_coef.argtypes = [vp, C.POINTER(YsgEvent), _dp]
    L.ysg_event_gradient.argtypes = [vp, C.POINTER(YsgEvent), C.POINTER(YsgTime), _dp, _dp, _dp]
    L.ysg_event_potential.argtypes = [vp, C.POINTER(YsgEvent), C.POINTER(YsgTime), _dp, C.POINTER(C.c_int)]
    L.ysg_legendre_table.argtypes = [vp, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
    L.ysg_set_solver.argtypes = [vp, C.c_int]
    L.ysg_set_schedule.argtypes = [vp, C.c_int]
    L.ysg_last_schedule.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_float)]
    L.ysg_last_timings.argtypes = [vp, C.POINTER(C.c_float)]
    L.ysg_last_work.argtypes = [vp, _dp, _dp]
    L.ysg_last_bytes.argtypes = [vp, _dp, _dp]
    L.ysg_last_launches.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.ysg_fp64_peak.argtypes = [C.c_int, _dp]
    L.ysg_status_string.argtypes = [C.c_int]
    L.ysg_status_string.restype = C.c_char_p
    L.ysg_last_cuda_error.argtypes = []
    L.ysg_last_cuda_error.restype = C.c_char_p
    L.ysg_destroy.argtypes = [vp]
    L.ysg_destroy.restype = None
    L.ysh_norms_get.argtypes = [C.POINTER(YshNorms)]
    L.ysh_norms_get.restype = None
    L.ysh_read_params.argtypes = [C.c_char_p, C.POINTER(YshParams)]
    L.ysh_free_params.argtypes = [C.POINTER(YshParams)]
    L.ysh_free_params.restype = None
    L.ysh_read_model.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.ysh_model_view.argtypes = [vp, C.POINTER(YsgModel)]
    L.ysh_model_view.restype = None
    L.ysh_model_nknot.argtypes = [vp]
    L.ysh_model_array.argtypes = [vp, C.c_char_p]
    L.ysh_model_array.restype = _dp
    L.ysh_free_model.argtypes = [vp]
    L.ysh_free_model.restype = None
    L.ysh_event_setup.argtypes = [vp, C.POINTER(YshParams), C.POINTER(YshEvent)]
    L.ysh_free_event.argtypes = [C.POINTER(YshEvent)]
    L.ysh_free_event.restype = None
    L.ysh_write_traces.argtypes = [C.c_char_p, _dp, C.c_int, C.c_int]
    L.ysh_format_e15_6.argtypes = [C.c_double, C.c_char_p]
    L.ysh_format_e15_6.restype = None
    L.ysh_run.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(_dp), C.POINTER(C.c_int),
                          C.POINTER(C.c_int)]
    L.ysh_run_potential.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(_dp), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int)]
    L.ysh_run_batch.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.ysh_free.argtypes = [vp]
    L.ysh_free.restype = None
    L.ysh_status_string.argtypes = [C.c_int]
    L.ysh_status_string.restype = C.c_char_p
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != 0:
        raise YspecError(status, where)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)
