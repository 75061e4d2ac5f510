"""Differentiable synthetics (yspec_b200.adjoint) on the GPU.

The forward of MomentTensorSynthetics must equal full solves of the event
with the same moment tensor (1e-9 relative L2 per trace).  The gradient of
an L2 waveform misfit with respect to the six moment-tensor components
must agree with central finite differences of the misfit.  The finite
differences use independent full solves through Engine.run, to 1e-6
relative (the bar for the differentiable path), per component and along
20 random directions.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, workloads as W
from yspec_b200 import adjoint

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("adj")
    p = W.config("c4", seed=3, lmax=60, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)[0]
    p.receivers = p.receivers[:12]
    pf = p.write(d / "c4.in")
    model = Model(p.model_file)
    eng = Engine(0)
    eng.upload(model)
    ev = Event(model, Params(pf))
    return p, eng, ev


def _misfit_full(eng, ev, mm, obs):
    tr = eng.run(adjoint.with_moment(ev, mm))[:, 1:4, :]
    return 0.5 * float(np.sum((tr - obs) ** 2))


def test_forward_equals_full_solves(case):
    p, eng, ev = case
    syn = adjoint.Synthetics(eng, ev)
    mm = torch.tensor(p.mm, dtype=torch.float64)
    got = syn(mm).numpy()
    want = eng.run(ev)
    np.testing.assert_array_equal(syn.time, want[0, 0])
    for k in range(ev.nr):
        for c in range(3):
            assert rel_l2(got[k, c], want[k, 1 + c]) <= 1e-9


def test_gradient_matches_finite_differences(case):
    p, eng, ev = case
    rng = np.random.default_rng(5)
    mm_obs = np.array(p.mm) + rng.normal(0.0, 3e19, 6)
    obs = eng.run(adjoint.with_moment(ev, mm_obs))[:, 1:4, :]
    obs = obs + 0.01 * np.std(obs) * rng.standard_normal(obs.shape)
    syn = adjoint.Synthetics(eng, ev)
    mm0 = np.array(p.mm)
    mm = torch.tensor(mm0, dtype=torch.float64, requires_grad=True)
    loss = 0.5 * ((syn(mm) - torch.from_numpy(obs)) ** 2).sum()
    loss.backward()
    grad = mm.grad.numpy()
    h = 1e-3 * np.max(np.abs(mm0))
    fd = np.zeros(6)
    for i in range(6):
        e = np.zeros(6)
        e[i] = h
        fd[i] = (_misfit_full(eng, ev, mm0 + e, obs) - _misfit_full(eng, ev, mm0 - e, obs)) / (2 * h)
    assert np.linalg.norm(grad - fd) <= 1e-6 * np.linalg.norm(fd)
    for _ in range(20):
        d = rng.standard_normal(6)
        d /= np.linalg.norm(d)
        dd = (_misfit_full(eng, ev, mm0 + h * d, obs) - _misfit_full(eng, ev, mm0 - h * d, obs)) / (2 * h)
        assert abs(grad @ d - dd) <= 1e-6 * np.linalg.norm(fd)
