"""Python mirror of the yspec program and of its (omega,l) solver boundary.

The names follow the reference (da380/YSpec): a parameter file
(yspec.f90:79-139), a deck-format model (module_model.f90:175-383), an event
set up as yspec.f90:144-215 does, then spectra (the (omega,l) loop and
l-sum, yspec.f90:250-426) and traces (ifft and post-processing,
yspec.f90:432-486).  Everything numerical runs on the GPU through the
ysg_* C-ABI; this module only moves arrays.

Array shapes (row-major views of the reference's column-major arrays):
    spectra ur, ut, up     complex (nr, nw)          == ur(nw, nr)
    traces                 float64 (nr, 4, nout)     == out(nout, 4, nr); columns t, Z, N, E
    coefficients           complex (L, 15, nw)       uu(1:5), vv(1:5), ww(1:5) per (l, omega)
    Legendre table         float64 (lmax+1, nr, 8)   X_l0..2, dX_l0..2, X_l1/sin, X_l2/sin
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import native as N

# lengths of the arrays the engine fills (include/yspec_gpu.h)
N_STAGE_TIMES = 4   # ysg_last_timings: legendre, solve, l-sum, time series
N_SCHEDULES = 3     # ysg_last_schedule: tuning time of each batched-solver schedule


def norms() -> dict:
    n = N.YshNorms()
    N.lib().ysh_norms_get(C.byref(n))
    return {f: getattr(n, f) for f, _ in N.YshNorms._fields_}


class Params:
    """Parameter file contents (yspec.f90:88-137)."""

    def __init__(self, path: str | os.PathLike):
        self.raw = N.YshParams()
        N.check(N.lib().ysh_read_params(os.fsencode(path), C.byref(self.raw)), "read_params")
        self.path = os.fspath(path)

    def __del__(self):
        try:
            N.lib().ysh_free_params(C.byref(self.raw))
        except Exception:
            pass

    def __getattr__(self, name):
        raw = self.__dict__.get("raw")
        if raw is None:
            raise AttributeError(name)
        v = getattr(raw, name)
        return v.decode() if isinstance(v, bytes) else v


class Model:
    """Normalised, splined earth model (module_model.f90:175-383)."""

    def __init__(self, path: str | os.PathLike):
        self.ptr = C.c_void_p()
        N.check(N.lib().ysh_read_model(os.fsencode(path), C.byref(self.ptr)), "read_model")
        self.nknot = N.lib().ysh_model_nknot(self.ptr)

    def __del__(self):
        if getattr(self, "ptr", None):
            try:
                N.lib().ysh_free_model(self.ptr)
            except Exception:       # interpreter shutdown: the module may be gone
                pass
            self.ptr = None

    def view(self) -> N.YsgModel:
        v = N.YsgModel()
        N.lib().ysh_model_view(self.ptr, C.byref(v))
        return v

    def array(self, name: str) -> np.ndarray:
        p = N.lib().ysh_model_array(self.ptr, name.encode())
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(self.nknot,)).copy()


class Event:
    """One event after yspec.f90:144-215 (normalisation, fcal, indices, delaz)."""

    def __init__(self, model: Model, params: Params):
        self.raw = N.YshEvent()
        self.model, self.params = model, params
        N.check(N.lib().ysh_event_setup(model.ptr, C.byref(params.raw), C.byref(self.raw)), "event_setup")

    def __del__(self):
        try:
            N.lib().ysh_free_event(C.byref(self.raw))
        except Exception:
            pass

    @property
    def ev(self) -> N.YsgEvent:
        return self.raw.ev

    @property
    def tm(self) -> N.YsgTime:
        return self.raw.tm

    @property
    def nw(self) -> int:
        return self.raw.ev.nw

    @property
    def nr(self) -> int:
        return self.raw.ev.nr

    @property
    def L(self) -> int:
        return self.raw.ev.lmax - self.raw.ev.lmin + 1

    def nout(self) -> int:
        return N.lib().ysg_trace_rows(C.byref(self.raw.tm))

    def delta(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.raw.delta, shape=(self.nr,)).copy()


class Engine:
    """A ysg handle on one GPU: upload a model, then run events."""

    def __init__(self, device: int = 0, solver: str = "batched"):
        self.h = C.c_void_p()
        self._nknot = 0
        N.check(N.lib().ysg_create(C.byref(self.h), device), "ysg_create")
        self.solver = solver
        self.set_solver(solver)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                N.lib().ysg_destroy(self.h)
            except Exception:       # interpreter shutdown: the module may be gone
                pass
            self.h = None

    def set_solver(self, which: str) -> None:
        """"plain", "batched" or "tangent" (derivative of every output along the
        model direction given to upload_tangent)."""
        N.check(N.lib().ysg_set_solver(self.h, {"plain": 0, "batched": 1, "tangent": 2}[which]),
                "set_solver")
        self.solver = which

    def set_schedule(self, sched: int) -> None:
        """Batched-solver schedule: 0 tiles, 1 cost-sorted pair lists, 2 the same lists
        as a spheroidal and a toroidal launch, -1 autotuned."""
        N.check(N.lib().ysg_set_schedule(self.h, sched), "set_schedule")

    def last_schedule(self) -> tuple[int, list[float]]:
        """Schedule of the last batched solve and the last autotuning times (ms)."""
        s = C.c_int()
        ms = (C.c_float * N_SCHEDULES)()
        N.check(N.lib().ysg_last_schedule(self.h, C.byref(s), ms), "last_schedule")
        return s.value, list(ms)

    def upload(self, model: Model) -> None:
        """Upload a model: a Model read from a deck, or any object whose view()
        returns a filled N.YsgModel (yspec_b200.model_chain.ArrayModel)."""
        v = model.view()
        N.check(N.lib().ysg_model_upload(self.h, C.byref(v)), "model_upload")
        self._nknot = v.nknot

    def upload_tangent(self, dmodel) -> None:
        """Derivative of the uploaded model along one direction (an object with
        view(), e.g. model_chain.ArrayModel holding derivative arrays)."""
        v = dmodel.view()
        N.check(N.lib().ysg_model_tangent_upload(self.h, C.byref(v)), "model_tangent_upload")

    def upload_tangents(self, dmodels) -> None:
        """Several directions: with solver "tangent", slot s of batch_run takes
        direction s."""
        views = (N.YsgModel * len(dmodels))(*[d.view() for d in dmodels])
        N.check(N.lib().ysg_model_tangents_upload(self.h, len(dmodels), views), "model_tangents_upload")

    def spectra(self, event: Event, copy: bool = True):
        nw, nr = event.nw, event.nr
        if not copy:
            N.check(N.lib().ysg_event_spectra(self.h, C.byref(event.raw.ev), None, None, None), "spectra")
            return None
        bufs = [np.zeros((nr, nw, 2)) for _ in range(3)]
        N.check(N.lib().ysg_event_spectra(self.h, C.byref(event.raw.ev),
                                          *[N.dptr(b) for b in bufs]), "spectra")
        return tuple(b[..., 0] + 1j * b[..., 1] for b in bufs)

    def traces(self, event: Event) -> np.ndarray:
        nout = event.nout()
        out = np.zeros((event.nr, 4, nout))
        n = C.c_int()
        N.check(N.lib().ysg_event_traces(self.h, C.byref(event.raw.tm), N.dptr(out), C.byref(n)), "traces")
        return out

    def run(self, event: Event) -> np.ndarray:
        nout = event.nout()
        out = np.zeros((event.nr, 4, nout))
        n = C.c_int()
        N.check(N.lib().ysg_event_run(self.h, C.byref(event.raw.ev), C.byref(event.raw.tm),
                                      N.dptr(out), C.byref(n)), "run")
        return out

    def prepare(self, event: Event) -> None:
        N.check(N.lib().ysg_event_prepare(self.h, C.byref(event.raw.ev), C.byref(event.raw.tm)), "prepare")

    def execute(self) -> None:
        N.check(N.lib().ysg_event_execute(self.h), "execute")

    def fetch(self, out: np.ndarray | None = None, out_ptr: int | None = None) -> int:
        n = C.c_int()
        ptr = N.dptr(out) if out is not None else (C.cast(out_ptr, N._dp) if out_ptr else None)
        N.check(N.lib().ysg_event_fetch(self.h, ptr, C.byref(n)), "fetch")
        return n.value

    def stream(self) -> int:
        s = C.c_void_p()
        N.check(N.lib().ysg_get_stream(self.h, C.byref(s)), "stream")
        return s.value or 0

    def batch_run(self, events: list[Event], outs: list[np.ndarray] | None = None) -> list[np.ndarray]:
        """Run several events as one batch.  `outs` are caller-owned (nr, 4, nout)
        float64 arrays, one per event; the same array may serve several events
        (each overwrites it in turn), for batches whose traces exceed host memory."""
        nev = len(events)
        evs = (N.YsgEvent * nev)(*[e.raw.ev for e in events])
        tms = (N.YsgTime * nev)(*[e.raw.tm for e in events])
        if outs is None:
            outs = [np.zeros((e.nr, 4, e.nout())) for e in events]
        if len(outs) != nev:
            raise ValueError("one output array per event")
        for e, o in zip(events, outs):
            if o.shape != (e.nr, 4, e.nout()) or o.dtype != np.float64 or not o.flags.c_contiguous:
                raise ValueError("output array must be C-contiguous float64 (nr, 4, nout)")
        ptrs = (N._dp * nev)(*[N.dptr(o) for o in outs])
        nouts = (C.c_int * nev)()
        N.check(N.lib().ysg_batch_run(self.h, nev, evs, tms, ptrs, nouts), "batch_run")
        return outs

    def potential(self, event: Event) -> np.ndarray:
        """Potential traces (nr, 2, nout): time in seconds and the perturbation
        of the gravitational potential at each receiver in SI units, in the
        event's output type (potential, or its first or second time
        derivative)."""
        nrm = norms()
        out_type = event.raw.ev.out
        tm = N.YsgTime.from_buffer_copy(event.raw.tm)
        tm.amp_norm = nrm["pot_norm"] / nrm["t_norm"] ** out_type
        out = np.zeros((event.nr, 2, event.nout()))
        n = C.c_int()
        N.check(N.lib().ysg_event_potential(self.h, C.byref(event.raw.ev), C.byref(tm), N.dptr(out), C.byref(n)),
                "event_potential")
        return out

    def gradient(self, event: Event, gout: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Reverse mode: the gradient of L = sum(gout * traces) with respect to
        the uploaded model's knot arrays.  gout is (nr, 4, nout) like run()'s
        output (column 0, time, ignored).  Returns (gval, gcs), each (13, nknot):
        dL/d(knot value) and dL/d(spline second derivative) per parameter, in
        the order of model_chain.PARAMS.  Raises for paths the reverse solver
        does not cover (status 8)."""
        g = np.ascontiguousarray(gout, dtype=np.float64)
        if g.shape != (event.nr, 4, event.nout()):
            raise ValueError("gout must be (nr, 4, nout)")
        n = self._nknot
        gval = np.zeros((13, n))
        gcs = np.zeros((13, n))
        N.check(N.lib().ysg_event_gradient(self.h, C.byref(event.raw.ev), C.byref(event.raw.tm), N.dptr(g),
                                           N.dptr(gval), N.dptr(gcs)), "event_gradient")
        return gval, gcs

    def coef(self, event: Event) -> np.ndarray:
        buf = np.zeros((event.L, 15, event.nw, 2))
        N.check(N.lib().ysg_event_coef(self.h, C.byref(event.raw.ev), N.dptr(buf)), "coef")
        return buf[..., 0] + 1j * buf[..., 1]

    def legendre(self, delta: np.ndarray, lmax: int) -> np.ndarray:
        delta = np.ascontiguousarray(delta, dtype=np.float64)
        nr = delta.size
        ct, st = np.cos(delta), np.sin(delta)
        tab = np.zeros((lmax + 1, nr, 8))
        N.check(N.lib().ysg_legendre_table(self.h, nr, lmax, N.dptr(delta), N.dptr(ct), N.dptr(st),
                                           N.dptr(tab)), "legendre")
        return tab

    def timings(self) -> list[float]:
        ms = (C.c_float * N_STAGE_TIMES)()
        N.check(N.lib().ysg_last_timings(self.h, ms), "timings")
        return list(ms)

    def bytes_moved(self) -> tuple[float, float]:
        a, b = C.c_double(), C.c_double()
        N.check(N.lib().ysg_last_bytes(self.h, C.byref(a), C.byref(b)), "bytes")
        return a.value, b.value

    def launches(self) -> int:
        """Kernels of this library enqueued since the last prepare / run."""
        n = C.c_longlong()
        N.check(N.lib().ysg_last_launches(self.h, C.byref(n)), "launches")
        return n.value

    def work(self) -> tuple[float, float]:
        p, f = C.c_double(), C.c_double()
        N.check(N.lib().ysg_last_work(self.h, C.byref(p), C.byref(f)), "work")
        return p.value, f.value


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput of the device (TFLOP/s)."""
    t = C.c_double()
    N.check(N.lib().ysg_fp64_peak(device, C.byref(t)), "fp64_peak")
    return t.value


def run_file(param_file: str | os.PathLike, device: int = 0, write_files: bool = False,
             potential: bool = False) -> np.ndarray:
    """The whole `yspec input.in` program; returns traces (nr, 4, nout).
    With potential=True, `yspec --potential input.in`: the potential traces
    (nr, 2, nout), files prefix.pot.k when write_files."""
    out = N._dp()
    nout, nr = C.c_int(), C.c_int()
    fn = N.lib().ysh_run_potential if potential else N.lib().ysh_run
    N.check(fn(os.fsencode(param_file), device, int(write_files), C.byref(out), C.byref(nout), C.byref(nr)),
            "ysh_run_potential" if potential else "ysh_run")
    try:
        arr = np.ctypeslib.as_array(out, shape=(nr.value, 2 if potential else 4, nout.value)).copy()
    finally:
        N.lib().ysh_free(out)
    return arr
