"""The differentiable model chain (yspec_b200.model_chain) on the CPU.

KnotModel.arrays restates read_model (module_model.f90:175-383) in torch:
its arrays must equal the host chain's (ysh_read_model) to rounding on
every bundled deck, and its forward-mode derivative must agree with
central differences of the chain itself.
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN
from yspec_b200.model_chain import PARAMS, KnotModel

DECKS = ["model200.deck", "model200_fic.deck", "model200_ocean.deck", "model400.deck"]


@pytest.mark.parametrize("deck", DECKS)
def test_chain_equals_host(deck):
    km = KnotModel(GOLDEN / deck)
    arrs = km.arrays(*km.params())
    for name in PARAMS:
        scale = max(np.abs(km.host.array(name)).max(), 1e-300)
        for key in (name, name + "_cs"):
            err = np.abs(arrs[key].numpy() - km.host.array(key)).max()
            # second derivatives are compared on the scale of their values
            assert err <= 1e-12 * (scale if key == name else
                                   max(scale, np.abs(km.host.array(key)).max())), key
    alpha, beta = km.speeds(*km.params())
    np.testing.assert_allclose(alpha.numpy(), km.host.array("alpha"), rtol=1e-14, atol=0)
    np.testing.assert_allclose(beta.numpy(), km.host.array("beta"), rtol=1e-14, atol=1e-300)


@pytest.mark.parametrize("deck", ["model200.deck", "model400.deck"])
def test_chain_tangent_matches_differences(deck):
    km = KnotModel(GOLDEN / deck)
    rng = np.random.default_rng(0)
    p = km.params()
    d = tuple(torch.from_numpy(rng.standard_normal(km.nknot)) * x * 1e-2 for x in p)
    dm = km.tangent(d)
    eps = 1e-3
    ap = km.arrays(*(x + eps * y for x, y in zip(p, d)))
    am = km.arrays(*(x - eps * y for x, y in zip(p, d)))
    for i, name in enumerate(PARAMS):
        for key, tg in ((name, dm.val[i]), (name + "_cs", dm.cs[i])):
            fd = ((ap[key] - am[key]) / (2 * eps)).numpy()
            scale = max(np.abs(tg).max(), 1e-30)
            assert np.abs(fd - tg).max() <= 1e-6 * scale, key


def test_jacobian_columns_are_tangents():
    km = KnotModel(GOLDEN / "model200.deck")
    jac = km.jacobian()
    n = km.nknot
    for col in (0, n + 17, 2 * n + 150):
        e = torch.zeros(3 * n, dtype=torch.float64)
        e[col] = 1.0
        dm = km.tangent((e[:n], e[n:2 * n], e[2 * n:]))
        for i, name in enumerate(PARAMS):
            np.testing.assert_allclose(jac[name][:, col].numpy(), dm.val[i], rtol=1e-12, atol=1e-300)
            np.testing.assert_allclose(jac[name + "_cs"][:, col].numpy(), dm.cs[i], rtol=1e-12,
                                       atol=1e-12 * np.abs(dm.cs[i]).max() + 1e-300)


@pytest.mark.parametrize("deck", ["model200.deck", "model400.deck"])
def test_chain_transpose_by_autograd(deck):
    """The reverse-mode gradient's last step (adjoint.ModelSynthetics with
    method "adjoint"): dL/d(rho, Vp, Vs) from dL/d(knot arrays) by autograd
    through the chain equals the transpose of the complex-step Jacobian."""
    km = KnotModel(GOLDEN / deck)
    rng = np.random.default_rng(5)
    gval = rng.standard_normal((13, km.nknot))
    gcs = rng.standard_normal((13, km.nknot))
    pp = tuple(x.clone().requires_grad_() for x in km.params())
    arrs = km.arrays(*pp)
    s = sum((torch.from_numpy(gval[i]) * arrs[n]).sum() + (torch.from_numpy(gcs[i]) * arrs[n + "_cs"]).sum()
            for i, n in enumerate(PARAMS))
    gr = torch.autograd.grad(s, pp, allow_unused=True)
    got = torch.cat([g if g is not None else torch.zeros(km.nknot, dtype=torch.float64) for g in gr]).numpy()
    jac = km.jacobian()
    ref = sum(gval[i] @ jac[n].numpy() + gcs[i] @ jac[n + "_cs"].numpy() for i, n in enumerate(PARAMS))
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
