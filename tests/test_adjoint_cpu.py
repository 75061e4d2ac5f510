"""The autograd function of the differentiable path, on CPU: its backward is
the adjoint of its forward (torch.autograd.gradcheck on random Green's
functions), and the forward is the linear combination of the unit responses."""
import numpy as np
import torch

from yspec_b200 import adjoint


def test_moment_tensor_function_gradcheck():
    fn = adjoint._function()
    rng = np.random.default_rng(2)
    G = torch.from_numpy(rng.standard_normal((6, 3, 3, 11)))
    mm = torch.from_numpy(rng.standard_normal(6)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda m: fn.apply(m, G, 7.0), (mm,), eps=1e-6, atol=1e-9)
    out = fn.apply(mm, G, 7.0).detach().numpy()
    want = np.einsum("i,iktn->ktn", mm.detach().numpy(), G.numpy()) / 7.0
    np.testing.assert_allclose(out, want, rtol=1e-14, atol=0)
