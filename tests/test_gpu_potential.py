"""Potential traces (ysg_event_potential, Engine.potential) against the CPU
oracle's potential mode (yo_set_potential).

The reference computes the pieces and never writes the result: the
spheroidal solution's third component (the potential, ysph(3,:)), the
l = 0 potential of rad_solver_wg (module_solver.f90:534-554) and the
four-component inverse transform ifft4 (module_fourier.f90:148-241).  The
potential traces put them together through the displacement's l-sum and
time stage.  Bar: 1e-9 relative L2 per trace, as for the displacement;
without gravity the potential is zero on both sides.
"""
import numpy as np
import pytest

import yo
from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-9


def small(seed=3, **over):
    base = dict(lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)
    base.update(over)
    p = W.config("c1", seed=seed, **base)[0]
    p.receivers = p.receivers[:4]
    return p


SCENARIOS = {
    "grav2_disp": dict(),
    "grav2_atten_acc_cor": dict(ats=1, out=2, cor=1),
    "grav2_vel_receiver_at_depth": dict(ats=1, out=1, depth_r=50.0),
    "receiver_below_source": dict(depth_s=20.0, depth_r=250.0, ats=1),
    "grav1_cowling": dict(grav=1, ats=1),
    "grav0_nogravity": dict(grav=0, ats=1, out=2),
    "fic_model": dict(model_file=str(W.GOLDEN / "model200_fic.deck"), depth_r=3.0, ats=1),
    "ocean_model": dict(model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_r=3.0, ats=1),
}


@pytest.mark.parametrize("solver", ["plain", "batched"])
@pytest.mark.parametrize("name", list(SCENARIOS))
def test_potential_traces_match_oracle(workdir, name, solver):
    p = small(**SCENARIOS[name])
    pf = p.write(workdir / f"pot_{name}.in")
    model = Model(p.model_file)
    ev = Event(model, Params(pf))
    eng = Engine(0, solver=solver)
    eng.upload(model)
    got = eng.potential(ev)
    want = yo.Problem(pf).potential_traces(nthreads=8)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got[:, 0], want[:, 0])
    if SCENARIOS[name].get("grav") == 0:
        assert np.all(got[:, 1] == 0.0) and np.all(want[:, 1] == 0.0)
        return
    assert np.abs(want[:, 1]).max() > 0.0
    for k in range(ev.nr):
        assert rel_l2(got[k, 1], want[k, 1]) <= TOL, (name, solver, k)


def test_potential_at_c1_size(workdir):
    """c1 as stated (lmax 150, 10 mHz, 10 receivers, 60 min at 10 s)."""
    p = W.config("c1", seed=0)[0]
    pf = p.write(workdir / "pot_c1.in")
    model = Model(p.model_file)
    ev = Event(model, Params(pf))
    eng = Engine(0)
    eng.upload(model)
    got = eng.potential(ev)
    want = yo.Problem(pf).potential_traces(nthreads=16)
    for k in range(ev.nr):
        assert rel_l2(got[k, 1], want[k, 1]) <= TOL, k


def test_potential_leaves_displacement_untouched(workdir):
    """A potential call between two displacement runs of the same event
    changes nothing in the second run."""
    p = small()
    pf = p.write(workdir / "pot_then_disp.in")
    model = Model(p.model_file)
    ev = Event(model, Params(pf))
    eng = Engine(0)
    eng.upload(model)
    a = eng.run(ev)
    eng.potential(ev)
    b = eng.run(ev)
    np.testing.assert_array_equal(a, b)
