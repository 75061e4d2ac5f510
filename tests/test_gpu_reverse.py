"""Reverse mode (ysg_event_gradient, k_solve_adjoint.cu) against the
tangent-linear solver, which differentiates the same discrete solve in
forward mode: for a random trace adjoint gout and random model directions d,
<gradient(gout), d> must equal <gout, d traces / dd> to 1e-10 relative.
Covered: the c1 and c4 configurations, displacement / velocity /
acceleration with the potential and tilt corrections, receivers at the
surface, at depth and below the source, an ocean and a fluid inner core, Cowling and no
gravity, and the whole ModelSynthetics backward pass against
its forward-mode counterpart and, at the c4 size, against central
differences of the misfit along 20 directions."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ("c1", {}),
    ("c4", {}),
    ("c4", {"out": 2, "cor": 1}),
    ("c4", {"out": 1, "depth_r": 50.0}),
    ("c4", {"model_file": "model200_ocean.deck", "depth_r": 3.0}),
    ("c1", {"model_file": "model200_fic.deck", "depth_r": 3.0, "ats": 1, "out": 2, "cor": 1}),
    ("c4", {"grav": 1}),
    ("c1", {"grav": 0, "ats": 1, "out": 2, "cor": 1}),
    # receivers below the source
    ("c4", {"depth_s": 20.0, "depth_r": 250.0}),
    ("c1", {"grav": 1, "depth_s": 20.0, "depth_r": 250.0, "ats": 1, "out": 1}),
    ("c1", {"grav": 0, "depth_s": 20.0, "depth_r": 250.0, "ats": 1, "out": 2, "cor": 1}),
    ("c1", {"model_file": "model200_ocean.deck", "depth_s": 3.0, "depth_r": 250.0, "ats": 1}),
    ("c1", {"model_file": "model200_fic.deck", "depth_s": 3.0, "depth_r": 250.0, "ats": 1, "out": 2, "cor": 1}),
]


def _setup(tmp_path, cfg, over):
    from yspec_b200 import Engine, Event, Params, workloads as W
    from yspec_b200.model_chain import KnotModel

    over = dict(over)
    if "model_file" in over:
        over["model_file"] = str(W.GOLDEN / over["model_file"])
    p = W.config(cfg, seed=0, **over)[0]
    pf = p.write(tmp_path / f"{cfg}.in")
    km = KnotModel(p.model_file)
    return Engine(0), Event(km.host, Params(pf)), km


@pytest.mark.parametrize("cfg,over", CASES)
def test_gradient_matches_tangent(tmp_path, cfg, over):
    import torch

    from yspec_b200.adjoint import tangent_traces

    eng, ev, km = _setup(tmp_path, cfg, over)
    eng.upload(km.array_model())
    rng = np.random.default_rng(7)
    gout = rng.standard_normal((ev.nr, 4, ev.nout()))
    gout[:, 0, :] = 0.0
    gval, gcs = eng.gradient(ev, gout)
    assert np.all(np.isfinite(gval)) and np.all(np.isfinite(gcs))
    for k in range(3):
        d = tuple(torch.from_numpy(rng.standard_normal(km.nknot)) * x * 1e-2 for x in km.params())
        dm = km.tangent(d)
        lhs = sum(float(np.dot(gval[i], dm.val[i]) + np.dot(gcs[i], dm.cs[i])) for i in range(13))
        rhs = float(np.sum(gout[:, 1:4, :] * tangent_traces(eng, ev, km, d)))
        assert abs(lhs - rhs) <= 1e-10 * abs(rhs), (cfg, over, k, lhs, rhs)


def test_model_synthetics_reverse_equals_forward_mode(tmp_path):
    """The knot-parameter gradient of a misfit through ModelSynthetics: the
    reverse sweep with autograd through the model chain against one
    tangent-linear solve per knot parameter (c1: 600 directions)."""
    import torch

    from yspec_b200 import adjoint

    eng, ev, km = _setup(tmp_path, "c1", {})
    P0 = km.params()
    mm0 = torch.tensor([1e20, 3e19, -2e19, 5e19, 1e19, -4e19], dtype=torch.float64)
    obs = adjoint.ModelSynthetics(eng, ev, km)(*(x * 1.01 for x in P0), mm0).detach()
    grads = {}
    for method in ("adjoint", "tangent"):
        syn = adjoint.ModelSynthetics(eng, ev, km, method=method)
        rho, vp, vs = (x.clone().requires_grad_() for x in P0)
        mm = mm0.clone().requires_grad_()
        loss = 0.5 * ((syn(rho, vp, vs, mm) - obs) ** 2).sum()
        loss.backward()
        assert syn.last_method == method
        grads[method] = torch.cat([rho.grad, vp.grad, vs.grad]).numpy()
    a, t = grads["adjoint"], grads["tangent"]
    assert np.max(np.abs(a - t)) <= 1e-9 * np.max(np.abs(t))


def test_unsupported_path_falls_back(tmp_path, monkeypatch):
    """An event the reverse sweep does not cover (a source in the outer core)
    returns status 8 from Engine.gradient before any device work, and
    ModelSynthetics falls back to the tangent-linear sweep when the gradient
    reports status 8."""
    import torch

    from yspec_b200 import adjoint
    from yspec_b200.native import YSG_ERR_UNSUPPORTED, YspecError

    eng, ev, km = _setup(tmp_path, "c1", {"depth_s": 3000.0})
    assert ev.raw.ev.is_ <= km.view0.noc
    eng.upload(km.array_model())
    with pytest.raises(YspecError) as ei:
        eng.gradient(ev, np.zeros((ev.nr, 4, ev.nout())))
    assert ei.value.status == YSG_ERR_UNSUPPORTED

    eng, ev, km = _setup(tmp_path, "c1", {})

    def unsupported(*args, **kwargs):
        raise YspecError(YSG_ERR_UNSUPPORTED, "event_gradient")

    monkeypatch.setattr(eng, "gradient", unsupported)
    syn = adjoint.ModelSynthetics(eng, ev, km, knots=[10, 100])
    rho, vp, vs = (x.clone().requires_grad_() for x in km.params())
    mm = torch.tensor([1e20, 0, 0, 0, 0, 0], dtype=torch.float64)
    (syn(rho, vp, vs, mm) ** 2).sum().backward()
    assert syn.last_method == "tangent"
    assert torch.count_nonzero(rho.grad) <= 2


def test_c4_misfit_gradient_against_differences(tmp_path):
    """The c4 workload at size (lmax 300, 20 mHz, 50 receivers, 200 knots):
    the reverse-mode gradient of an L2 waveform misfit with respect to the
    600 knot parameters and the moment tensor, along 20 random directions,
    against central differences of the misfit (step 1e-3, start levels and
    step counts of the deck's model), to 1e-6 relative."""
    import torch

    from yspec_b200 import adjoint

    from yspec_b200 import workloads as W

    eng, ev, km = _setup(tmp_path, "c4", {})
    p = W.config("c4", seed=0)[0]
    syn = adjoint.ModelSynthetics(eng, ev, km)
    P0 = km.params()
    mm0 = torch.tensor(p.mm, dtype=torch.float64)
    rng = np.random.default_rng(11)
    kern = np.exp(-0.5 * (np.arange(-9, 10) / 3.0) ** 2)
    kern /= kern.sum()
    Pobs = tuple(x * (1.0 + torch.from_numpy(np.convolve(rng.standard_normal(km.nknot), kern, mode="same")) * 1e-2)
                 for x in P0)
    obs = syn(*Pobs, mm0).detach()
    rho, vp, vs = (x.clone().requires_grad_() for x in P0)
    mm = mm0.clone().requires_grad_()
    loss = 0.5 * ((syn(rho, vp, vs, mm) - obs) ** 2).sum()
    loss.backward()
    assert syn.last_method == "adjoint"
    grad = (rho.grad, vp.grad, vs.grad, mm.grad)
    worst = 0.0
    for k in range(20):
        r = np.random.default_rng(100 + k)
        dk = tuple(torch.from_numpy(r.standard_normal(km.nknot)) * x * 1e-2 for x in P0)
        dm = torch.from_numpy(r.standard_normal(6)) * 1e18
        with torch.no_grad():
            lp = float(0.5 * ((syn(*(x + 1e-3 * y for x, y in zip(P0, dk)), mm0 + 1e-3 * dm) - obs) ** 2).sum())
            lm = float(0.5 * ((syn(*(x - 1e-3 * y for x, y in zip(P0, dk)), mm0 - 1e-3 * dm) - obs) ** 2).sum())
        fd = (lp - lm) / 2e-3
        ad = sum(float((g * y).sum()) for g, y in zip(grad, dk + (dm,)))
        worst = max(worst, abs(ad - fd) / abs(fd))
    assert worst <= 1e-6, worst
