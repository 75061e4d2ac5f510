"""Tangent-linear solver and model gradients on the GPU.

The tangent solver (k_solve_tangent.cu, Engine solver "tangent") returns
the derivative of the traces along one direction of the per-knot rho, Vp,
Vs.  Its derivatives are checked against central differences of full
primal solves, with the start levels and step counts of the deck held
fixed in both (model_chain.KnotModel.array_model freezes alpha and beta,
which steer only those integer decisions).  Central differences with step
1e-3 along a 1% direction carry a truncation error near 3e-8; the bar is
1e-6 relative L2 per trace, over the solver branches of the parity tests.

ModelSynthetics' backward (the gradient of a waveform misfit with respect
to all 3 x 200 knot parameters and the moment tensor) is checked against
central differences of the misfit along 20 random directions, to 1e-6.
"""
import numpy as np
import pytest
import torch

from yspec_b200 import Engine, Event, Params, workloads as W
from yspec_b200 import adjoint
from yspec_b200.model_chain import KnotModel

pytestmark = pytest.mark.gpu

TOL = 1e-6


def small(seed=3, **over):
    base = dict(lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)
    base.update(over)
    p = W.config("c1", seed=seed, **base)[0]
    p.receivers = p.receivers[:4]
    return p


SCENARIOS = {
    "grav2_atten": dict(ats=1),
    "grav2_atten_acc_cor": dict(ats=1, out=2, cor=1),
    "grav1_cowling": dict(grav=1, ats=1, out=1),
    "grav0_nogravity": dict(grav=0, ats=1, out=2),
    "receiver_below_source": dict(depth_s=20.0, depth_r=250.0, ats=1),
    "ocean_model": dict(model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_r=3.0, ats=1),
    "fic_model": dict(model_file=str(W.GOLDEN / "model200_fic.deck"), depth_r=3.0, ats=1),
}


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


def _direction(km, seed):
    rng = np.random.default_rng(seed)
    return tuple(torch.from_numpy(rng.standard_normal(km.nknot)) * x * 1e-2 for x in km.params())


def _primal(engine, km, ev, params):
    engine.set_solver("plain")
    engine.upload(km.array_model(*params))
    return engine.run(ev)[:, 1:4, :]


@pytest.mark.parametrize("name", list(SCENARIOS))
def test_tangent_matches_central_differences(engine, workdir, name):
    p = small(**SCENARIOS[name])
    pf = p.write(workdir / f"{name}.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    d = _direction(km, 1)
    T = adjoint.tangent_traces(engine, ev, km, d)
    P = km.params()
    eps = 1e-3
    up = _primal(engine, km, ev, tuple(x + eps * y for x, y in zip(P, d)))
    um = _primal(engine, km, ev, tuple(x - eps * y for x, y in zip(P, d)))
    fd = (up - um) / (2 * eps)
    assert np.linalg.norm(fd) > 0
    for k in range(T.shape[0]):
        for c in range(3):
            den = np.linalg.norm(fd[k, c])
            assert np.linalg.norm(T[k, c] - fd[k, c]) <= TOL * den, (k, c)


def test_tangent_is_linear_in_the_direction(engine, workdir):
    p = small(ats=1, out=2, cor=1)
    pf = p.write(workdir / "lin.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    d1, d2 = _direction(km, 4), _direction(km, 5)
    t1 = adjoint.tangent_traces(engine, ev, km, d1)
    t2 = adjoint.tangent_traces(engine, ev, km, d2)
    t12 = adjoint.tangent_traces(engine, ev, km, tuple(2.0 * a - 0.5 * b for a, b in zip(d1, d2)))
    assert np.linalg.norm(t12 - (2.0 * t1 - 0.5 * t2)) <= 1e-12 * np.linalg.norm(t12)
    zero = adjoint.tangent_traces(engine, ev, km, tuple(torch.zeros_like(a) for a in d1))
    assert not zero.any()


def test_directions_in_one_batch_equal_single_runs(engine, workdir):
    """Slot s of a tangent batch takes direction s: the batched derivatives
    equal one-direction runs."""
    p = small(ats=1, out=2, cor=1)
    pf = p.write(workdir / "many.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    dirs = [_direction(km, 20 + k) for k in range(5)]
    many = adjoint.tangent_traces_many(engine, ev, km, dirs)
    for k, d in enumerate(dirs):
        one = adjoint.tangent_traces(engine, ev, km, d)
        assert np.linalg.norm(many[k] - one) <= 1e-12 * np.linalg.norm(one), k


def test_direction_count_must_match_the_batch(engine, workdir):
    """Loaded directions must be one (shared by every slot) or one per slot;
    any other count is rejected before anything runs, and the engine keeps
    working afterwards."""
    p = small()
    pf = p.write(workdir / "count.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    dirs = [_direction(km, 30 + k) for k in range(3)]
    engine.set_solver("tangent")
    try:
        engine.upload(km.array_model())
        engine.upload_tangents([km.tangent(d) for d in dirs])
        with pytest.raises(Exception):
            engine.batch_run([ev, ev])
        engine.upload_tangents([km.tangent(d) for d in dirs[:2]])
        two = engine.batch_run([ev, ev])
    finally:
        engine.set_solver("batched")
    one = adjoint.tangent_traces(engine, ev, km, dirs[1])
    assert np.linalg.norm(two[1][:, 1:4, :] - one) <= 1e-12 * np.linalg.norm(one)


def test_tangent_needs_a_direction(engine, workdir):
    p = small()
    pf = p.write(workdir / "nodir.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    engine.set_solver("tangent")
    engine.upload(km.host)          # a new model discards any earlier direction
    with pytest.raises(Exception):
        engine.run(ev)
    engine.set_solver("batched")


@pytest.mark.parametrize("size", ["small", "c4"])
def test_model_gradient_matches_finite_differences(engine, workdir, size):
    """Misfit gradient over every knot parameter and the moment tensor,
    against central differences of the misfit along 20 random directions:
    on a small event, and on c4 as stated (lmax 300, 20 mHz, 60 min at 5 s,
    50 receivers, source at 150 km; 3 x 200 knot parameters)."""
    if size == "small":
        p = W.config("c4", seed=3, lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)[0]
        p.receivers = p.receivers[:6]
    else:
        p = W.config("c4", seed=0)[0]
    pf = p.write(workdir / "c4.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    syn = adjoint.ModelSynthetics(engine, ev, km)
    P0 = km.params()
    mm0 = torch.tensor(p.mm, dtype=torch.float64)
    # observed: a smoothed 1% perturbation of every knot parameter
    rng = np.random.default_rng(11)
    kern = np.exp(-0.5 * (np.arange(-9, 10) / 3.0) ** 2)
    smooth = lambda v: np.convolve(v, kern / kern.sum(), mode="same")
    Pobs = tuple(x * (1.0 + torch.from_numpy(smooth(rng.standard_normal(km.nknot))) * 1e-2) for x in P0)
    obs = syn(*Pobs, mm0).detach()

    rho, vp, vs = (x.clone().requires_grad_() for x in P0)
    mm = mm0.clone().requires_grad_()
    loss = 0.5 * ((syn(rho, vp, vs, mm) - obs) ** 2).sum()
    loss.backward()
    grad = (rho.grad, vp.grad, vs.grad, mm.grad)

    def misfit(q, m):
        with torch.no_grad():
            return float(0.5 * ((syn(*q, m) - obs) ** 2).sum())

    eps = 1e-3
    for k in range(20):
        dk = _direction(km, 100 + k)
        dm = torch.from_numpy(np.random.default_rng(200 + k).standard_normal(6)) * 1e18
        lp = misfit(tuple(x + eps * y for x, y in zip(P0, dk)), mm0 + eps * dm)
        lm = misfit(tuple(x - eps * y for x, y in zip(P0, dk)), mm0 - eps * dm)
        fd = (lp - lm) / (2 * eps)
        ad = sum(float((g * y).sum()) for g, y in zip(grad, dk + (dm,)))
        assert abs(ad - fd) <= TOL * abs(fd), (k, ad, fd)
