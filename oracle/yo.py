"""ctypes loader of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
check the device traces, and by bench.py for the CPU baseline leg.  The product
(yspec_b200) never imports it.  Parity status: unpinned (see yo.h).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_dp = C.POINTER(C.c_double)


class Norms(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "r_norm", "rho_norm", "vel_norm", "acl_norm", "fre_norm", "t_norm",
        "con_norm", "grav_norm", "moment_norm", "pot_norm", "pibigg")]


class Params(C.Structure):
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


class Model(C.Structure):
    _fields_ = ([("ifanis", C.c_int), ("ocean", C.c_int), ("fic", C.c_int),
                 ("nlayer", C.c_int), ("nknot", C.c_int), ("nic", C.c_int), ("noc", C.c_int),
                 ("nsl", C.c_int), ("layer_lo", C.POINTER(C.c_int)), ("layer_hi", C.POINTER(C.c_int)),
                 ("tref", C.c_double)] +
                [(n, _dp) for n in (
                    "r", "rho", "rho_cs", "acon", "acon_cs", "ccon", "ccon_cs", "fcon", "fcon_cs",
                    "lcon", "lcon_cs", "ncon", "ncon_cs", "kappa", "kappa_cs", "mu", "mu_cs",
                    "lambda_", "qkappa", "qkappa_cs", "qmu", "qmu_cs", "grav", "grav_cs",
                    "beta", "alpha", "rat", "rat_cs", "xlam", "xlam_cs", "xa2", "xa2_cs")])


class Grid(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("nt", "i1", "i2", "nw", "is_", "ir")] +
                [(n, C.c_double) for n in ("df", "ep", "dw", "wmin", "dt", "tout", "rs", "rr",
                                            "f1", "f2", "f11", "f12", "f21", "f22")] +
                [("mm", C.c_double * 6)])


class CD(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class Counts(C.Structure):
    _fields_ = [("nrhs", C.c_longlong * 16), ("nstep", C.c_longlong * 16),
                ("nsolve_tor", C.c_longlong), ("nsolve_sph", C.c_longlong),
                ("nsolve_rad", C.c_longlong)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"oracle not built: {LIB} (make -C oracle)")
        L = C.CDLL(str(LIB))
        L.yo_set_parameters.argtypes = [C.POINTER(Norms)]
        L.yo_read_params.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.yo_read_model.argtypes = [C.c_char_p, C.POINTER(Norms), C.POINTER(Model)]
        L.yo_event_setup.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.POINTER(Params), C.POINTER(Grid)]
        L.yo_solve_pair.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.POINTER(Params), C.POINTER(Grid),
                                    C.c_int, C.c_int, _dp, C.POINTER(Counts)]
        L.yo_spectra.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.POINTER(Params), C.POINTER(Grid),
                                 _dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(Counts)]
        L.yo_spectra_shard.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.POINTER(Params),
                                       C.POINTER(Grid), C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                       C.c_int]
        _ip = C.POINTER(C.c_int)
        L.yo_coef_list.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.POINTER(Params),
                                   C.POINTER(Grid), C.c_int, _ip, _ip, _dp, C.c_int]
        L.yo_green.argtypes = [C.POINTER(Model), C.POINTER(Norms), C.c_int, C.c_int, C.c_double,
                               C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _dp]
        L.yo_find_radius_index.argtypes = [C.POINTER(Model), C.c_double]
        L.yo_set_step_refine.argtypes = [C.c_int]
        L.yo_set_potential.argtypes = [C.c_int]
        L.yo_geometry.argtypes = [C.POINTER(Params), _dp, _dp, _dp]
        L.yo_legendre_table.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp, _dp]
        L.yo_traces.argtypes = [C.POINTER(Norms), C.POINTER(Params), C.POINTER(Grid), _dp, _dp, _dp,
                                _dp, _dp, C.POINTER(C.c_int)]
        L.yo_legendre.argtypes = [C.c_double, C.c_int, C.c_int, _dp, _dp, _dp]
        L.yo_fcal.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp,
                              C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.yo_spline.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double, _dp]
        L.yo_splint_dis.argtypes = [_dp, _dp, _dp, C.c_double, C.c_int]
        L.yo_splint_dis.restype = C.c_double
        L.yo_bfs.argtypes = [C.c_int, CD, C.c_double, _dp]
        L.yo_delaz.argtypes = [C.c_double] * 4 + [_dp] * 3
        L.yo_write_traces.argtypes = [C.c_char_p, _dp, C.c_int, C.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Problem:
    """A parameter file read and set up by the oracle (yspec.f90:74-215)."""

    def __init__(self, param_file: str | os.PathLike):
        L = lib()
        self.norms = Norms()
        L.yo_set_parameters(C.byref(self.norms))
        self.params = Params()
        rc = L.yo_read_params(os.fsencode(param_file), C.byref(self.params))
        if rc:
            raise RuntimeError(f"oracle: read_params stop {rc}")
        self.model = Model()
        mf = self.params.model_file
        if not os.path.isabs(mf.decode()):
            mf = os.fsencode(os.path.join(os.path.dirname(os.path.abspath(param_file)), mf.decode()))
        rc = L.yo_read_model(mf, C.byref(self.norms), C.byref(self.model))
        if rc:
            raise RuntimeError(f"oracle: read_model stop {rc}")
        self.grid = Grid()
        self.setup_rc = L.yo_event_setup(C.byref(self.model), C.byref(self.norms),
                                         C.byref(self.params), C.byref(self.grid))

    @property
    def nw(self):
        return self.grid.nw

    @property
    def nr(self):
        return self.params.nr

    def array(self, name: str) -> np.ndarray:
        n = self.model.nknot
        p = getattr(self.model, "lambda_" if name == "lambda" else name)
        return np.ctypeslib.as_array(p, shape=(n + 1,))[1:].copy()

    def coef(self, l: int, j: int, counts: Counts | None = None) -> np.ndarray:
        buf = np.zeros(30)
        lib().yo_solve_pair(C.byref(self.model), C.byref(self.norms), C.byref(self.params),
                            C.byref(self.grid), l, j, _p(buf), C.byref(counts) if counts else None)
        return buf[0::2] + 1j * buf[1::2]

    def spectra(self, nthreads: int = 0, lsub=None, jsub: int = 0, counts: Counts | None = None):
        nw, nr = self.nw, self.nr
        bufs = [np.zeros((max(nr, 1), nw, 2)) for _ in range(3)]
        lo, hi = (lsub if lsub is not None else (0, -1))
        lib().yo_spectra(C.byref(self.model), C.byref(self.norms), C.byref(self.params),
                         C.byref(self.grid), *[_p(b) for b in bufs], nthreads, lo, hi, jsub,
                         C.byref(counts) if counts else None)
        return tuple((b[..., 0] + 1j * b[..., 1])[:nr] for b in bufs)

    def spectra_shard(self, jofs: int, jstride: int, count: int, nthreads: int = 0):
        """Spectra (nr, count) of the frequencies j = 1 + jofs + c jstride."""
        nr = self.nr
        bufs = [np.zeros((max(nr, 1), count, 2)) for _ in range(3)]
        rc = lib().yo_spectra_shard(C.byref(self.model), C.byref(self.norms), C.byref(self.params),
                                    C.byref(self.grid), jofs, jstride, count,
                                    *[_p(b) for b in bufs], nthreads)
        if rc:
            raise ValueError(f"oracle: spectra_shard rc {rc}")
        return tuple((b[..., 0] + 1j * b[..., 1])[:nr] for b in bufs)

    def coef_list(self, ls, js, nthreads: int = 0) -> np.ndarray:
        """Coefficients (npair, 15) of the (l, j) pairs (j 1-based), on threads."""
        ls = np.ascontiguousarray(ls, dtype=np.int32)
        js = np.ascontiguousarray(js, dtype=np.int32)
        if ls.shape != js.shape or ls.ndim != 1:
            raise ValueError("ls and js: equal 1-d lengths")
        buf = np.zeros((ls.size, 15, 2))
        ip = C.POINTER(C.c_int)
        rc = lib().yo_coef_list(C.byref(self.model), C.byref(self.norms), C.byref(self.params),
                                C.byref(self.grid), ls.size, ls.ctypes.data_as(ip),
                                js.ctypes.data_as(ip), _p(buf), nthreads)
        if rc:
            raise ValueError(f"oracle: coef_list rc {rc}")
        return buf[..., 0] + 1j * buf[..., 1]

    GREEN_SHAPE = {0: (2, 2), 1: (2, 2), 2: (2, 2), 3: (6, 4), 4: (4, 4), 5: (4, 4)}

    def radius_index(self, r: float) -> int:
        """find_radius_index (module_model.f90:537) of a normalised radius."""
        return lib().yo_find_radius_index(C.byref(self.model), r)

    def green(self, kind: int, l: int, w: complex, rr: float, rs: float, ats: int = 0) -> np.ndarray:
        """Solution at normalised radius rr for unit jumps at rs (see yo_green)."""
        shape = self.GREEN_SHAPE[kind]
        buf = np.zeros(shape + (2,))
        rc = lib().yo_green(C.byref(self.model), C.byref(self.norms), kind, l, w.real, w.imag, ats,
                            rr, rs, self.radius_index(rr), self.radius_index(rs), _p(buf))
        if rc:
            raise ValueError(f"oracle: green rc {rc}")
        return buf[..., 0] + 1j * buf[..., 1]

    def geometry(self):
        nr = self.nr
        d, ae, ast = np.zeros(nr), np.zeros(nr), np.zeros(nr)
        lib().yo_geometry(C.byref(self.params), _p(d), _p(ae), _p(ast))
        return d, ae, ast

    def legendre_table(self, lmax: int | None = None) -> np.ndarray:
        """(lmax+1, 3, nr) column-major tables xa, xpa, xca as (3, nr, 3, lmax+1) row-major."""
        lmax = self.params.lmax if lmax is None else lmax
        d, _, _ = self.geometry()
        nr = self.nr
        xa, xpa, xca = (np.zeros((nr, 3, lmax + 1)) for _ in range(3))
        lib().yo_legendre_table(_p(d), nr, lmax, _p(xa), _p(xpa), _p(xca))
        return xa, xpa, xca

    def traces(self, ur, ut, up) -> np.ndarray:
        nw, nr = self.nw, self.nr
        def pack(a):
            b = np.zeros((nr, nw, 2))
            b[..., 0], b[..., 1] = a.real, a.imag
            return b
        bu, bt, bp = pack(ur), pack(ut), pack(up)
        _, azep, _ = self.geometry()
        nt = self.grid.nt
        nout = nt
        for i in range(1, nt + 1):
            if (i - 1) * self.grid.dt > self.grid.tout:
                nout = i
                break
        out = np.zeros((nr, 4, nout))
        n = C.c_int()
        lib().yo_traces(C.byref(self.norms), C.byref(self.params), C.byref(self.grid),
                        _p(bu), _p(bt), _p(bp), _p(azep), _p(out), C.byref(n))
        return out

    def run(self, nthreads: int = 0) -> np.ndarray:
        return self.traces(*self.spectra(nthreads=nthreads))

    def potential_traces(self, nthreads: int = 0) -> np.ndarray:
        """Potential traces (nr, 2, nout): time and the perturbation of the
        gravitational potential at each receiver in SI units, in the
        output type (see yo_set_potential)."""
        with potential():
            ur, ut, up = self.spectra(nthreads=nthreads)
        out = self.traces(ur, ut, up)
        n = self.norms
        o = self.params.out
        amp = n.r_norm if o == 0 else (n.vel_norm if o == 1 else n.acl_norm)
        res = np.empty((out.shape[0], 2, out.shape[2]))
        res[:, 0] = out[:, 0]
        res[:, 1] = out[:, 1] / amp * (n.pot_norm / n.t_norm ** o)
        return res


class potential:
    """Context manager: the oracle's solves return potential coefficients
    (yo_set_potential)."""

    def __enter__(self):
        lib().yo_set_potential(1)
        return self

    def __exit__(self, *exc):
        lib().yo_set_potential(0)
        return False


class step_refine:
    """Context manager: the oracle's integrations take `k` times the
    reference's step count per knot interval (convergence checks only)."""

    def __init__(self, k: int):
        self.k = k

    def __enter__(self):
        lib().yo_set_step_refine(self.k)
        return self

    def __exit__(self, *exc):
        lib().yo_set_step_refine(1)
        return False


def legendre(theta: float, l: int, m: int):
    x, xp, xc = np.zeros(m + 1), np.zeros(m + 1), np.zeros(m + 1)
    lib().yo_legendre(theta, l, m, _p(x), _p(xp), _p(xc))
    return x, xp, xc


def fcal(f1, f2, dt, tout, mex=5, qex=1):
    a, b = C.c_double(f1), C.c_double(f2)
    df, ep = C.c_double(), C.c_double()
    nt, i1, i2 = C.c_int(), C.c_int(), C.c_int()
    rc = lib().yo_fcal(C.byref(a), C.byref(b), dt, tout, mex, qex, C.byref(df), C.byref(ep),
                       C.byref(nt), C.byref(i1), C.byref(i2))
    return rc, nt.value, i1.value, i2.value, df.value, ep.value


def bfs(l: int, xsq: complex, eps: float = 1e-9) -> complex:
    fp = np.zeros(2)
    arg = CD(xsq.real, xsq.imag)
    lib().yo_bfs(l, arg, eps, _p(fp))
    return complex(fp[0], fp[1])


def spline(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, float)
    y = np.ascontiguousarray(y, float)
    y2 = np.zeros_like(x)
    lib().yo_spline(_p(x), _p(y), x.size, 1e40, 1e40, _p(y2))
    return y2


def splint(x: np.ndarray, y: np.ndarray, y2: np.ndarray, xv: float, klo: int) -> float:
    """klo 1-based as in the reference."""
    xa = np.concatenate([[0.0], x]); ya = np.concatenate([[0.0], y]); y2a = np.concatenate([[0.0], y2])
    return lib().yo_splint_dis(_p(xa), _p(ya), _p(y2a), xv, klo)
