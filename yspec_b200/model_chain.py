"""The earth-model chain of read_model as a differentiable function of the
per-knot density, P velocity and S velocity.

read_model (module_model.f90:175-383) turns a deck into the arrays the
solvers read: it normalises radii, densities and velocities (:253-263),
forms the moduli A, C, F, L, N, kappa, mu and the attenuation combinations
xlam, xa2 (:263-290), fits a natural cubic spline per layer to each array
(spline_r / tridag_ser_r, module_spline.f90:40-73, 426-449; layers split at
repeated radii, :294-352) and integrates gravity with a 5-point
Gauss-Legendre rule on a spline of r^2 rho (gauslv, :356-378).

`KnotModel.arrays` restates that chain in torch (float64) on the knot
parameters rho, Vp, Vs.  A P- (S-) velocity change moves the vertical and
the horizontal velocity of a knot together (Vpv and Vph, Vsv and Vsh).  The
chain reproduces the host's arrays (ysh_read_model) to rounding.  Every
operation in it is analytic in the parameters, so its derivative comes by
the complex step (Im f(p + i h d) / h, exact to rounding for tiny h): the
derivative arrays that the tangent-linear solver takes
(Engine.upload_tangent), one direction at a time or the whole Jacobian in
one evaluation.

alpha and beta (module_model.f90:276-277) only steer integer decisions of
the solver (start levels, step counts).  `ArrayModel` can hold them fixed
at the base model, which is the setting the tangent solver differentiates.
"""
from __future__ import annotations

import os

import numpy as np

from . import native as N
from .api import Model, norms

# order of the device's 13 spline parameters (ysg_model.cuh, Param)
PARAMS = ["rho", "acon", "ccon", "fcon", "lcon", "ncon", "kappa", "mu",
          "qkappa", "qmu", "grav", "xlam", "xa2"]

# Gauss-Legendre nodes and weights of gauslv (module_model.f90:507-535)
_GL_X = (0.538469310105683, 0.906179845938664)
_GL_W = (0.478628670499366, 0.236926885056189)
_GL_W0 = 0.568888888888889


def _real(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def read_deck(path: str | os.PathLike) -> dict:
    """Raw deck values (module_model.f90:185-222): radius, rho, Vpv, Vsv, Q_kappa,
    Q_mu and, for an anisotropic deck, Vph, Vsh, eta (else Vph = Vpv,
    Vsh = Vsv, eta = 1)."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    ians = int(lines[1].split()[0])
    n = int(lines[2].split()[0])
    rows = [lines[3 + i].split() for i in range(n)]
    cols = np.array([[_real(t) for t in row[: (9 if ians == 1 else 6)]] for row in rows])
    d = {"r": cols[:, 0], "rho": cols[:, 1], "vpv": cols[:, 2], "vsv": cols[:, 3],
         "qk": cols[:, 4], "qm": cols[:, 5]}
    if ians == 1:
        d.update(vph=cols[:, 6], vsh=cols[:, 7], eta=cols[:, 8])
    else:
        d.update(vph=cols[:, 2].copy(), vsh=cols[:, 3].copy(), eta=np.ones(n))
    return d


def _layers(r: np.ndarray) -> list[tuple[int, int]]:
    """0-based inclusive knot ranges of the layers (split at repeated radii)."""
    out, lo = [], 0
    for i in range(1, r.size):
        if r[i] == r[i - 1]:
            out.append((lo, i - 1))
            lo = i
    out.append((lo, r.size - 1))
    return out


class _LayerSpline:
    """Natural cubic spline second derivatives on one layer's knots x, by the
    recurrences of spline_r / tridag_ser_r (module_spline.f90:40-73,
    426-449): the coefficients that depend only on x are formed once, in the
    same order of operations, and the sweeps run on the values."""

    def __init__(self, x: np.ndarray):
        n = self.n = x.size
        c = np.zeros(n)
        a = np.zeros(n)
        b = np.zeros(n)
        for i in range(1, n):
            c[i - 1] = x[i] - x[i - 1]
        self.h = c[: max(n - 1, 0)].copy()
        for i in range(2, n):
            a[i - 1] = c[i - 2]
            b[i - 1] = 2.0 * (c[i - 1] + a[i - 1])
        b[0] = 1.0
        b[n - 1] = 1.0
        c[0] = 0.0          # natural end conditions (both flags > 0.99e30)
        a[n - 1] = 0.0
        # tridag: row j has sub-diagonal a[j] and super-diagonal c[j]
        self.a = a
        self.gam = np.zeros(n)
        self.bet = np.zeros(n)
        bet = b[0]
        self.bet[0] = bet
        for j in range(1, n):
            self.gam[j] = c[j - 1] / bet
            bet = b[j] - a[j] * self.gam[j]
            self.bet[j] = bet

    def __call__(self, y):
        """y: (n, m) tensor of m arrays on the layer; returns their y2."""
        import torch

        n = self.n
        if n < 2:
            return torch.zeros_like(y)
        z = torch.zeros_like(y[0])
        # right-hand side 6 (slope_i - slope_{i-1}) inside, zero at both ends
        s = [6.0 * ((y[i] - y[i - 1]) / float(self.h[i - 1])) for i in range(1, n)]
        r = [z] + [s[i - 1] - s[i - 2] for i in range(2, n)] + [z]
        u = [r[0] / float(self.bet[0])]
        for j in range(1, n):
            u.append((r[j] - float(self.a[j]) * u[j - 1]) / float(self.bet[j]))
        for j in range(n - 2, -1, -1):
            u[j] = u[j] - float(self.gam[j + 1]) * u[j + 1]
        return torch.stack(u)


def _spline_fn():
    """The spline map as an autograd function: the forward runs the
    recurrences (the values the upload uses), the backward applies the
    transpose of the same linear map, S^T g."""
    import torch

    global _SPLINE_FN
    if _SPLINE_FN is None:
        class _SplineFn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, Y, km):
                ctx.km = km
                return km._spline_rec(Y)

            @staticmethod
            def backward(ctx, g):
                return ctx.km.spline_matrix().T @ g, None

        _SPLINE_FN = _SplineFn
    return _SPLINE_FN


_SPLINE_FN = None


class KnotModel:
    """A deck as a differentiable function of its knot parameters.

        km = KnotModel("model.deck")
        rho, vp, vs = km.params()            # float64 tensors (nknot,), SI units
        arrs = km.arrays(rho, vp, vs)        # normalised arrays and spline derivatives
        base = km.array_model(rho, vp, vs)   # for Engine.upload
        dm = km.tangent((drho, dvp, dvs))    # derivative arrays, for Engine.upload_tangent
    """

    def __init__(self, path: str | os.PathLike):
        import torch

        self.path = os.fspath(path)
        self.deck = read_deck(path)
        self.host = Model(path)
        self.view0 = self.host.view()
        self.nknot = self.host.nknot
        if self.deck["r"].size != self.nknot:
            raise ValueError("deck and host model disagree on the knot count")
        self.nrm = norms()
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        self.t = {k: t(v) for k, v in self.deck.items()}
        self.r = self.t["r"] / self.nrm["r_norm"]
        rn = self.r.numpy()
        self.layers = _layers(rn)
        self.spl = [_LayerSpline(rn[lo:hi + 1]) for lo, hi in self.layers]
        # Gauss-Legendre evaluation points of gauslv on every knot interval
        self._gl = self._gauss_setup(rn)

    # -- parameters --------------------------------------------------------
    def params(self):
        """Base (rho, Vp, Vs) per knot, SI units: Vp = Vpv, Vs = Vsv."""
        return self.t["rho"].clone(), self.t["vpv"].clone(), self.t["vsv"].clone()

    # -- the chain ----------------------------------------------------------
    def _spline(self, y):
        """Per-layer spline second derivatives of y: (nknot,) or (nknot, m).
        The map is linear in y; under autograd its transpose is applied as
        one product with the operator's matrix (_SplineFn) instead of
        reversing the per-knot recurrences op by op."""
        import torch

        col = y.dim() == 1
        Y = y[:, None] if col else y
        if torch.is_grad_enabled() and Y.requires_grad and not Y.is_complex():
            out = _spline_fn().apply(Y, self)
        else:
            out = self._spline_rec(Y)
        return out[:, 0] if col else out

    def _spline_rec(self, Y):
        """The recurrences of spline_r / tridag_ser_r, layer by layer."""
        import torch

        return torch.cat([sp(Y[lo:hi + 1]) for sp, (lo, hi) in zip(self.spl, self.layers)])

    def spline_matrix(self):
        """S with _spline(y) = S y (block diagonal, one block per layer),
        formed once by the recurrences on the identity."""
        import torch

        if getattr(self, "_S", None) is None:
            with torch.no_grad():
                self._S = self._spline_rec(torch.eye(self.nknot, dtype=torch.float64))
        return self._S

    def _gauss_setup(self, r: np.ndarray):
        """Interval index of the five gauslv nodes on every knot interval, and
        the splint_dis_r weights (module_spline.f90:262-283) of each node
        times its Gauss weight times the half-width."""
        import torch

        klo, w = [], []
        for i in range(r.size - 1):
            r1, r2 = r[i], r[i + 1]
            y1, y2 = 0.5 * (r2 + r1), 0.5 * (r2 - r1)
            xs = [y1] + [y1 + x * y2 for x in _GL_X] + [y1 - x * y2 for x in _GL_X]
            ws = [_GL_W0] + list(_GL_W) + list(_GL_W)
            h = r2 - r1
            for x, wq in zip(xs, ws):
                if h == 0.0:
                    coef = (1.0, 0.0, 0.0, 0.0)
                else:
                    a = (r2 - x) / h
                    b = (x - r1) / h
                    coef = (a, b, (a * a * a - a) * (h * h) / 6.0, (b * b * b - b) * (h * h) / 6.0)
                klo.append(i)
                w.append([wq * y2 * cq for cq in coef])
        return torch.tensor(klo), torch.tensor(w, dtype=torch.float64)

    def arrays(self, rho, vp, vs) -> dict:
        """The 13 normalised parameter arrays and their spline second derivatives
        (name and name + "_cs") for knot parameters rho, Vp, Vs (SI units).
        The parameters may be (nknot,) or (nknot, m) for m parameter sets at
        once, real or complex (complex-step derivatives: every operation of
        the chain is analytic in the parameters)."""
        import torch

        nm = self.nrm
        col = (lambda t: t[:, None]) if rho.dim() == 2 else (lambda t: t)
        d = {k: col(v) for k, v in self.t.items()}
        dvp, dvs = vp - d["vpv"], vs - d["vsv"]
        rho_n = rho / nm["rho_norm"]
        vn = nm["vel_norm"]
        a = (d["vph"] + dvp) / vn
        c = vp / vn
        l = vs / vn
        nn = (d["vsh"] + dvs) / vn
        acon = rho_n * (a * a)
        ccon = rho_n * (c * c)
        lcon = rho_n * (l * l)
        ncon = rho_n * (nn * nn)
        fcon = (acon - 2.0 * lcon) * d["eta"]
        kappa = (ccon + 4.0 * acon - 4.0 * ncon + 4.0 * fcon) / 9.0
        mu = (ccon + acon + 6.0 * lcon + 5.0 * ncon - 2.0 * fcon) / 15.0
        lam = kappa - 2.0 * mu / 3.0
        qk, qm = d["qk"], d["qm"]
        qkappa = torch.where(qk > 0.0, 1.0 / torch.where(qk > 0.0, qk, 1.0), qk)
        qmu = torch.where(qm > 0.0, 1.0 / torch.where(qm > 0.0, qm, 1.0), qm)
        rat = 4.0 * mu / (3.0 * (lam + 2.0 * mu))
        xlam = ((1.0 - rat) * qkappa - 0.5 * rat * qmu) / (1.0 - 1.5 * rat)
        xa2 = (1.0 - rat) * qkappa + rat * qmu
        like = lambda t: t.to(rho_n.dtype).expand_as(rho_n)
        out = {"rho": rho_n, "acon": acon, "ccon": ccon, "fcon": fcon, "lcon": lcon,
               "ncon": ncon, "kappa": kappa, "mu": mu, "qkappa": like(qkappa), "qmu": like(qmu),
               "xlam": xlam, "xa2": xa2}
        # gravity: Gauss-Legendre on the spline of r^2 rho, accumulated outward
        r = col(self.r)
        intg = r * r * rho_n
        qint = self._spline(intg)
        klo, W = self._gl
        w = [col(W[:, i]) for i in range(4)]
        vals = w[0] * intg[klo] + w[1] * intg[klo + 1] + w[2] * qint[klo] + w[3] * qint[klo + 1]
        tail = tuple(intg.shape[1:])
        per = torch.zeros((self.nknot - 1,) + tail, dtype=intg.dtype).index_add(0, klo, vals)
        fint = torch.cat([torch.zeros((1,) + tail, dtype=intg.dtype), torch.cumsum(per, 0)])
        pos = col(self.r > 0.0)
        out["grav"] = torch.where(pos, 4.0 * fint / torch.where(pos, r * r, 1.0), fint)
        names = list(out)
        stack = torch.stack([out[k] for k in names], dim=1)
        cs = self._spline(stack.reshape(self.nknot, -1)).reshape(stack.shape)
        for i, k in enumerate(names):
            out[k + "_cs"] = cs[:, i]
        return out

    def speeds(self, rho, vp, vs):
        """alpha, beta of module_model.f90:276-277 (normalised), no derivative."""
        import torch

        with torch.no_grad():
            a = self.arrays(rho.detach(), vp.detach(), vs.detach())
            beta = torch.sqrt(a["mu"] / a["rho"])
            alpha = torch.sqrt((a["kappa"] + 1.3333333333 * a["mu"]) / a["rho"])
        return alpha, beta

    # -- device views ---------------------------------------------------------
    def array_model(self, rho=None, vp=None, vs=None, freeze: bool = True) -> "ArrayModel":
        """A model for Engine.upload at knot parameters rho, Vp, Vs (default: the
        deck's).  With `freeze`, alpha and beta -- which only steer the
        solver's integer decisions -- stay the deck's, so start levels and step
        counts do not move with the parameters: the setting in which the
        tangent solver differentiates and finite differences agree with it."""
        import torch

        p0 = self.params()
        p = tuple(x if x is not None else y for x, y in zip((rho, vp, vs), p0))
        with torch.no_grad():
            arrs = self.arrays(*p)
        if freeze:
            alpha, beta = self.host.array("alpha"), self.host.array("beta")
        else:
            alpha, beta = self.speeds(*p)
        return ArrayModel(self.view0, self.r.numpy(), arrs, alpha, beta)

    # complex step: f(p + i h d) = f(p) + i h f'(p) d + O(h^2), with no
    # cancellation, so Im f / h is the derivative to rounding
    _H = 1e-30

    def _complex_step(self, p, dirs):
        import torch

        h = self._H
        pc = tuple(x.to(torch.complex128) + (1j * h) * dx.to(torch.complex128)
                   for x, dx in zip(p, dirs))
        return {k: (v.imag / h).contiguous() for k, v in self.arrays(*pc).items()}

    def tangent(self, direction, at=None) -> "ArrayModel":
        """Derivative arrays along direction (drho, dvp, dvs) at knot parameters
        `at` (default: the deck's), for Engine.upload_tangent."""
        p = at if at is not None else self.params()
        d = self._complex_step(tuple(x.detach() for x in p), tuple(direction))
        z = np.zeros(self.nknot)
        return ArrayModel(self.view0, self.r.numpy(), d, z, z)

    def jacobian(self, at=None) -> dict:
        """d(array)/d(parameter) for every array name: tensors (nknot, 3 nknot),
        columns ordered rho, Vp, Vs (knot fastest)."""
        import torch

        p = at if at is not None else self.params()
        n = self.nknot
        eye = torch.eye(3 * n, dtype=torch.float64)
        pm = tuple(x.detach()[:, None].expand(n, 3 * n) for x in p)
        return self._complex_step(pm, (eye[:n], eye[n:2 * n], eye[2 * n:]))


class ArrayModel:
    """Model arrays held in numpy for Engine.upload / upload_tangent: the
    scalar fields of a host model view plus the 13 arrays, their spline second
    derivatives, alpha and beta."""

    def __init__(self, view0: N.YsgModel, r: np.ndarray, arrs: dict, alpha, beta):
        f = lambda a: np.ascontiguousarray(a.detach().numpy() if hasattr(a, "detach") else a,
                                           dtype=np.float64)
        self.r = f(r)
        self.val = [f(arrs[p]) for p in PARAMS]
        self.cs = [f(arrs[p + "_cs"]) for p in PARAMS]
        self.alpha, self.beta = f(alpha), f(beta)
        self.view0 = view0

    def view(self) -> N.YsgModel:
        v = N.YsgModel()
        for k in ("nknot", "nic", "noc", "nsl", "ocean", "fic", "tref", "pibigg", "fre_norm"):
            setattr(v, k, getattr(self.view0, k))
        v.r = N.dptr(self.r)
        for p in range(13):
            v.val[p] = N.dptr(self.val[p])
            v.cs[p] = N.dptr(self.cs[p])
        v.alpha = N.dptr(self.alpha)
        v.beta = N.dptr(self.beta)
        return v

    def array(self, name: str) -> np.ndarray:
        if name in PARAMS:
            return self.val[PARAMS.index(name)]
        if name.endswith("_cs") and name[:-3] in PARAMS:
            return self.cs[PARAMS.index(name[:-3])]
        return {"r": self.r, "alpha": self.alpha, "beta": self.beta}[name]
