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

Gradients with respect to the model (per-knot rho, Vp, Vs) would need the
adjoint of the radial integration itself.  They are not provided here.
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
