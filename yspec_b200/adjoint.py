"""Differentiable synthetics: traces and misfit gradients with respect to the
moment tensor.

Every trace of yspec is linear in the six moment-tensor components: they
enter only through the source vectors (module_solver.f90:145-215, 566-627,
1747-1847), which are linear in mm, and everything after the (omega,l)
solves (the l-sum, the inverse FFT, e^{eps t}, scaling, rotation) is
linear.  So

    traces(mm) = sum_i (mm_i / moment_norm) G_i,

where G_i are the traces of the same event with the unit normalised moment
tensor e_i.  `greens` computes the six G_i as one six-event batch (one
batched solve launch, one CUDA graph).  `MomentTensorSynthetics` is a
torch.autograd.Function over them.  Its backward is the exact adjoint of
the linear map, dL/dmm_i = <dL/dtraces, G_i> / moment_norm.

Gradients with respect to the earth model (per-knot rho, Vp, Vs) come in
reverse mode by default: Engine.gradient (ysg_event_gradient) carries the
trace adjoint back through the time stage and the l-sum (their transposes)
and through every (omega, l) solve (its discrete adjoint, k_solve_adjoint.cu)
to dL/d(knot arrays), and torch autograd takes it through the model chain
(model_chain.KnotModel.arrays) to rho, Vp and Vs: one reverse sweep per
pair, whatever the number of parameters.  The forward-mode alternative is
the tangent-linear solver (k_solve_tangent.cu): the per-pair solve compiled
with dual numbers returns the derivative of every coefficient along one
direction of the model, so a run with solver "tangent" returns the
derivative of the traces along that direction; `ModelSynthetics(...,
method="tangent")` sweeps the 3 nknot knot parameters that way, and events
the reverse solver does not cover fall back to it.  Start levels and step
counts stay those of the deck's model in both (they are piecewise constant
in the parameters).
"""
from __future__ import annotations

import numpy as np

from . import native as N
from .api import Engine, Event, norms


class _UnitSource:
    """A copy of an event with moment tensor e_i (normalised units); it shares
    the original's receiver arrays, which must outlive it."""

    def __init__(self, event: Event, i: int):
        self._owner = event
        self.raw = N.YshEvent.from_buffer_copy(event.raw)
        for q in range(6):
            self.raw.ev.mm[q] = 1.0 if q == i else 0.0
        self.nr = event.nr
        self._nout = event.nout()

    def nout(self) -> int:
        return self._nout


def greens(engine: Engine, event: Event) -> tuple[np.ndarray, np.ndarray]:
    """(time (nout,), G (6, nr, 3, nout)): the Z, N, E traces of the event for
    each unit normalised moment-tensor component, in the reference's order
    M_rr, M_rt, M_rp, M_tt, M_tp, M_pp."""
    units = [_UnitSource(event, i) for i in range(6)]
    outs = engine.batch_run(units)
    G = np.stack([o[:, 1:4, :] for o in outs])
    return outs[0][0, 0, :].copy() if event.nr else np.zeros(0), G


def _function():
    import torch

    class MomentTensorSynthetics(torch.autograd.Function):
        """traces = sum_i mm_i G_i / moment_norm (mm in N m); backward is
        the exact adjoint of this linear map."""

        @staticmethod
        def forward(ctx, mm, G, moment_norm):
            ctx.save_for_backward(G)
            ctx.moment_norm = moment_norm
            return torch.einsum("i,iktn->ktn", mm, G) / moment_norm

        @staticmethod
        def backward(ctx, grad):
            (G,) = ctx.saved_tensors
            return torch.einsum("ktn,iktn->i", grad, G) / ctx.moment_norm, None, None

    return MomentTensorSynthetics


class Synthetics:
    """Differentiable traces of one event with respect to its moment tensor.

        syn = Synthetics(engine, event, device="cuda")
        traces = syn(mm)           # mm: float64 tensor (6,), N m; (nr, 3, nout)
        loss = 0.5 * ((traces - observed) ** 2).sum()
        loss.backward()            # mm.grad
    """

    def __init__(self, engine: Engine, event: Event, device=None):
        import torch

        self.time, G = greens(engine, event)
        self.G = torch.from_numpy(G)
        if device is not None:
            self.G = self.G.to(device)
        self.moment_norm = norms()["moment_norm"]
        self._fn = _function()

    def __call__(self, mm):
        return self._fn.apply(mm, self.G, self.moment_norm)


class _MomentCopy(_UnitSource):
    def __init__(self, event: Event, mm_norm):
        super().__init__(event, 0)
        for q in range(6):
            self.raw.ev.mm[q] = float(mm_norm[q])


def with_moment(event: Event, mm) -> _MomentCopy:
    """The event with moment tensor mm (N m, reference order), for Engine.run
    or Engine.batch_run; it shares the event's receiver arrays."""
    mn = norms()["moment_norm"]
    return _MomentCopy(event, [m / mn for m in mm])


def tangent_traces(engine: Engine, event, knot_model, direction, at=None) -> np.ndarray:
    """Derivative of the event's Z, N, E traces (nr, 3, nout) along
    direction = (drho, dvp, dvs) of the knot parameters at `at` (default: the
    deck's), with the deck's start levels and step counts."""
    km = knot_model
    p = at if at is not None else km.params()
    prev = engine.solver
    engine.set_solver("tangent")
    try:
        engine.upload(km.array_model(*p))
        engine.upload_tangent(km.tangent(direction, at=p))
        return engine.run(event)[:, 1:4, :]
    finally:
        engine.set_solver(prev)


def tangent_traces_many(engine: Engine, event, knot_model, directions, at=None) -> np.ndarray:
    """Derivatives of the event's Z, N, E traces along several directions,
    (len(directions), nr, 3, nout): one batch of copies of the event, slot s
    on direction s, one tangent solve launch for all of them."""
    km = knot_model
    p = at if at is not None else km.params()
    prev = engine.solver
    engine.set_solver("tangent")
    try:
        engine.upload(km.array_model(*p))
        engine.upload_tangents([km.tangent(d, at=p) for d in directions])
        outs = engine.batch_run([event] * len(directions))
        return np.stack([o[:, 1:4, :] for o in outs])
    finally:
        engine.set_solver(prev)


def _model_function():
    import torch

    class _ModelFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, rho, vp, vs, mm, syn):
            # the solves run on the engine's GPU; results follow the inputs' device
            G = syn._greens(rho, vp, vs).to(device=mm.device, dtype=mm.dtype)
            ctx.save_for_backward(rho, vp, vs, mm, G)
            ctx.syn = syn
            return torch.einsum("i,iktn->ktn", mm, G) / syn.moment_norm

        @staticmethod
        def backward(ctx, grad):
            rho, vp, vs, mm, G = ctx.saved_tensors
            syn = ctx.syn
            g_mm = torch.einsum("ktn,iktn->i", grad, G) / syn.moment_norm
            g = syn._knot_gradient(rho, vp, vs, mm, grad).to(device=rho.device, dtype=rho.dtype)
            n = syn.km.nknot
            return g[:n], g[n:2 * n], g[2 * n:], g_mm, None

    return _ModelFn


class ModelSynthetics:
    """Differentiable traces of one event with respect to the per-knot rho, Vp,
    Vs of its earth model (SI units) and its moment tensor (N m).

        km = model_chain.KnotModel(deck)
        syn = ModelSynthetics(engine, event, km)
        rho, vp, vs = (t.requires_grad_() for t in km.params())
        traces = syn(rho, vp, vs, mm)        # (nr, 3, nout): Z, N, E
        loss = 0.5 * ((traces - observed) ** 2).sum()
        loss.backward()                      # rho.grad, vp.grad, vs.grad, mm.grad

    Forward: the six unit-moment responses of the model at (rho, vp, vs), one
    batched launch, combined with mm.  Backward: mm exactly as
    MomentTensorSynthetics; the knot parameters by the reverse sweep
    (method "adjoint": one Engine.gradient call and autograd through the
    model chain), or by a tangent-linear solve per knot parameter (method
    "tangent", `chunk` directions per batched launch; also the fallback for
    events the reverse sweep does not cover).  With `knots`, only those
    knots' parameters get a gradient, the others zero.
    """

    def __init__(self, engine: Engine, event: Event, knot_model, knots=None, chunk: int = 64,
                 method: str = "adjoint"):
        if method not in ("adjoint", "tangent"):
            raise ValueError("method must be 'adjoint' or 'tangent'")
        self.engine, self.event, self.km = engine, event, knot_model
        self.chunk = chunk
        self.method = method
        self.last_method = None
        self.moment_norm = norms()["moment_norm"]
        n = knot_model.nknot
        self.columns = (list(range(3 * n)) if knots is None else
                        [q * n + k for q in range(3) for k in knots])
        self._fn = _model_function()

    def __call__(self, rho, vp, vs, mm):
        return self._fn.apply(rho, vp, vs, mm, self)

    def _greens(self, rho, vp, vs):
        import torch

        eng = self.engine
        prev = eng.solver
        eng.set_solver("batched")
        try:
            eng.upload(self.km.array_model(rho.detach(), vp.detach(), vs.detach()))
            _, G = greens(eng, self.event)
        finally:
            eng.set_solver(prev)
        return torch.from_numpy(G)

    def _knot_gradient(self, rho, vp, vs, mm, grad):
        """sum over traces of grad * d(traces)/d(parameter), per knot parameter."""
        if self.method == "adjoint":
            try:
                out = self._knot_gradient_reverse(rho, vp, vs, mm, grad)
                self.last_method = "adjoint"
                return out
            except N.YspecError as e:
                if e.status != N.YSG_ERR_UNSUPPORTED:
                    raise
        self.last_method = "tangent"
        return self._knot_gradient_tangent(rho, vp, vs, mm, grad)

    def _knot_gradient_reverse(self, rho, vp, vs, mm, grad):
        """Reverse mode: dL/d(knot arrays) from Engine.gradient, then the
        transpose of the model chain by autograd."""
        import torch

        from .model_chain import PARAMS, ArrayModel

        km, eng = self.km, self.engine
        p = (rho.detach().cpu(), vp.detach().cpu(), vs.detach().cpu())
        ev = with_moment(self.event, [float(x) for x in mm.detach()])
        g = np.asarray(grad.detach().cpu().numpy(), dtype=np.float64)
        gout = np.zeros((g.shape[0], 4, g.shape[2]))
        gout[:, 1:4, :] = g
        # the chain at p once, with its graph (autograd runs backward passes
        # with gradients off): its values are the model the reverse sweep runs
        # on, as km.array_model(*p) would form them, and its graph carries
        # dL/d(arrays) back to the knot parameters
        with torch.enable_grad():
            pp = tuple(x.clone().requires_grad_() for x in p)
            arrs = km.arrays(*pp)
        eng.upload(ArrayModel(km.view0, km.r.numpy(), arrs, km.host.array("alpha"), km.host.array("beta")))
        gval, gcs = eng.gradient(ev, gout)
        with torch.enable_grad():
            s = sum((torch.from_numpy(gval[i]) * arrs[name]).sum() +
                    (torch.from_numpy(gcs[i]) * arrs[name + "_cs"]).sum() for i, name in enumerate(PARAMS))
            gr = torch.autograd.grad(s, pp, allow_unused=True)
        n = km.nknot
        out = torch.cat([x if x is not None else torch.zeros(n, dtype=torch.float64) for x in gr])
        if len(self.columns) != 3 * n:
            keep = torch.zeros(3 * n, dtype=torch.bool)
            keep[self.columns] = True
            out = torch.where(keep, out, torch.zeros_like(out))
        return out.detach()

    def _knot_gradient_tangent(self, rho, vp, vs, mm, grad):
        """Forward mode: one tangent-linear solve per knot parameter."""
        import torch

        km, eng = self.km, self.engine
        p = (rho.detach(), vp.detach(), vs.detach())
        jac = km.jacobian(at=p)
        n = km.nknot
        z = np.zeros(n)
        ev = with_moment(self.event, [float(x) for x in mm.detach()])
        g = np.asarray(grad.detach().cpu().numpy(), dtype=np.float64)
        out = np.zeros(3 * n)
        prev = eng.solver
        eng.set_solver("tangent")
        try:
            eng.upload(km.array_model(*p))
            from .model_chain import ArrayModel

            # `chunk` directions per batch: slot s of the batch on direction s
            for c0 in range(0, len(self.columns), self.chunk):
                cols = self.columns[c0:c0 + self.chunk]
                dms = [ArrayModel(km.view0, km.r.numpy(), {k: v[:, col] for k, v in jac.items()}, z, z)
                       for col in cols]
                eng.upload_tangents(dms)
                for col, o in zip(cols, eng.batch_run([ev] * len(cols))):
                    out[col] = float(np.sum(g * o[:, 1:4, :]))
        finally:
            eng.set_solver(prev)
        return torch.from_numpy(out)
