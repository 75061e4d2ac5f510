"""GPU parity: the CUDA path through the C-ABI against the CPU oracle.

Bars (the reference path's own stated accuracy target): 1e-9 relative L2
per trace and per spectrum; the Legendre table is compared bit for bit; the
per-(omega,l) coefficients within 1e-9 of each coefficient row's norm.
"""
import numpy as np
import pytest

import yo
from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-9
SOLVERS = ["plain", "batched"]


def small(seed=3, **over):
    base = dict(lmax=40, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)
    base.update(over)
    p = W.config("c1", seed=seed, **base)[0]
    p.receivers = p.receivers[:4]
    return p


SCENARIOS = {
    "grav2_disp": dict(),
    "grav2_atten_acc_cor": dict(ats=1, out=2, cor=1),
    "grav2_vel": dict(ats=1, out=1),
    "grav1_cowling": dict(grav=1, ats=1),
    "grav0_nogravity": dict(grav=0, ats=1, out=2),
    "receiver_below_source": dict(depth_s=20.0, depth_r=250.0, ats=1),
    "deep_source": dict(depth_s=650.0, ats=1, out=2, cor=1),
    "ocean_model": dict(model_file=str(W.GOLDEN / "model200_ocean.deck"), depth_r=3.0, ats=1),
    "fic_model": dict(model_file=str(W.GOLDEN / "model200_fic.deck"), depth_r=3.0, ats=1),
    "fic_nogravity": dict(model_file=str(W.GOLDEN / "model200_fic.deck"), depth_r=3.0, grav=0),
    # sph_solver_cow_fic (module_solver.f90:1568-1740)
    "fic_cowling": dict(model_file=str(W.GOLDEN / "model200_fic.deck"), depth_r=3.0, grav=1,
                        ats=1),
    # receiver below the source on the fluid-inner-core deck: the low-degree
    # pairs start their solid minors inside the fluid inner core, as the
    # reference's fic solvers do on that branch
    "fic_receiver_below_source": dict(model_file=str(W.GOLDEN / "model200_fic.deck"),
                                      depth_s=20.0, depth_r=250.0, ats=1, out=2, cor=1),
    "fic_cowling_receiver_below": dict(model_file=str(W.GOLDEN / "model200_fic.deck"),
                                       depth_s=20.0, depth_r=250.0, grav=1),
    "fic_nogravity_receiver_below": dict(model_file=str(W.GOLDEN / "model200_fic.deck"),
                                         depth_s=20.0, depth_r=250.0, grav=0, ats=1),
    "lmin_band": dict(lmin=5, lmax=35),
}


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


def _case(workdir, name, over):
    p = small(**over)
    pf = p.write(workdir / f"{name}.in")
    model = Model(p.model_file)
    return p, pf, model, Event(model, Params(pf)), yo.Problem(pf)


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("name", list(SCENARIOS))
def test_traces_match_oracle(engine, workdir, name, solver):
    p, pf, model, ev, ref = _case(workdir, name, SCENARIOS[name])
    engine.set_solver(solver)
    engine.upload(model)
    got = engine.run(ev)
    want = ref.run(nthreads=8)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got[:, 0], want[:, 0])           # time column
    for k in range(got.shape[0]):
        for c in range(1, 4):
            err = rel_l2(got[k, c], want[k, c])
            assert err <= TOL, f"{name}/{solver}: receiver {k} comp {c}: {err:.3e}"


@pytest.mark.parametrize("solver", SOLVERS)
def test_spectra_match_oracle(engine, workdir, solver):
    p, pf, model, ev, ref = _case(workdir, "spec", dict(ats=1, out=2, cor=1))
    engine.set_solver(solver)
    engine.upload(model)
    gu, gt, gp = engine.spectra(ev)
    ru, rt, rp = ref.spectra(nthreads=8)
    for g, r in ((gu, ru), (gt, rt), (gp, rp)):
        for k in range(g.shape[0]):
            assert rel_l2(g[k], r[k]) <= TOL


@pytest.mark.parametrize("solver", SOLVERS)
def test_coefficients_match_oracle(engine, workdir, solver):
    p, pf, model, ev, ref = _case(workdir, "coef", dict(ats=1, out=2, cor=1, lmax=25))
    engine.set_solver(solver)
    engine.upload(model)
    got = engine.coef(ev)                       # (L, 15, nw)
    L, _, nw = got.shape
    want = np.zeros_like(got)
    for li in range(L):
        for j in range(1, nw + 1):
            want[li, :, j - 1] = ref.coef(p.lmin + li, j)
    for li in range(L):
        for q in range(15):
            n = np.linalg.norm(want[li, q])
            d = np.linalg.norm(got[li, q] - want[li, q])
            assert d <= TOL * max(n, 1e-300) or (n == 0 and d == 0), (li, q, d, n)


def test_legendre_bit_exact(engine):
    rng = np.random.default_rng(7)
    delta = np.concatenate([rng.uniform(0, np.pi, 29), [1e-6, 3e-6, 1e-5, np.pi - 1e-7, 0.5]])
    lmax = 300
    tab = engine.legendre(delta, lmax)          # (lmax+1, nr, 8)
    xa, xpa, xca = (np.zeros((delta.size, 3, lmax + 1)) for _ in range(3))
    yo.lib().yo_legendre_table(yo._p(delta), delta.size, lmax, yo._p(xa), yo._p(xpa), yo._p(xca))
    np.testing.assert_array_equal(tab[:, :, 0:3], np.transpose(xa, (2, 0, 1)))
    np.testing.assert_array_equal(tab[:, :, 3:6], np.transpose(xpa, (2, 0, 1)))
    np.testing.assert_array_equal(tab[:, :, 6:8], np.transpose(xca, (2, 0, 1))[:, :, 1:3])


def test_explosion_has_no_transverse_motion(engine, workdir):
    # an isotropic source excites no toroidal motion: E and N follow the
    # spheroidal field only, and receivers at equal distance record equal Z
    p = small(mm=[1e20, 0, 0, 1e20, 0, 1e20], lat_s=0.0, lon_s=0.0,
              receivers=[(0.0, 40.0), (0.0, -40.0)])
    pf = p.write(workdir / "expl.in")
    model = Model(p.model_file)
    engine.set_solver("batched")
    engine.upload(model)
    coef = engine.coef(Event(model, Params(pf)))
    assert np.abs(coef[:, 10:15]).max() == 0.0          # ww == 0
    tr = engine.run(Event(model, Params(pf)))
    z = tr[:, 1]
    assert rel_l2(z[1], z[0]) < 1e-10


@pytest.mark.parametrize("nrec", [45, 8])
def test_spectra_many_receivers_match_oracle(engine, workdir, nrec):
    """Receiver counts of 8 and more take the tensor-core l-sum (DMMA tiles of
    16 frequencies x 32 receivers): 45 receivers span a full and a partial
    receiver tile, and the band is not a multiple of the frequency tile."""
    import numpy as _np

    p = small(seed=9, ats=1, out=2, cor=1, lmax=37)
    p.receivers = W.sphere_points(_np.random.default_rng(77), nrec)
    pf = p.write(workdir / f"many{nrec}.in")
    model = Model(p.model_file)
    ev = Event(model, Params(pf))
    ref = yo.Problem(pf)
    assert ev.nw % 16 != 0 or nrec % 32 != 0
    for solver in SOLVERS:
        engine.set_solver(solver)
        engine.upload(model)
        gu, gt, gp = engine.spectra(ev)
        ru, rt, rp = ref.spectra(nthreads=8)
        for g, r in ((gu, ru), (gt, rt), (gp, rp)):
            for k in range(g.shape[0]):
                assert rel_l2(g[k], r[k]) <= TOL, (solver, k)
        got = engine.run(ev)
        want = ref.run(nthreads=8)
        for k in range(got.shape[0]):
            for c in range(1, 4):
                assert rel_l2(got[k, c], want[k, c]) <= TOL


def test_receivers_beyond_one_launch(engine, workdir):
    """More receivers than one launch of the time-series stage takes (21,845:
    three rows per receiver in grid.y): the stage runs in receiver chunks,
    and receivers on both sides of a chunk boundary must match the oracle
    run of those receivers alone."""
    import numpy as _np

    p = small(seed=12, lmax=20, fmax=4.0, f21=3.0, f22=3.8, dt=40.0, tout=40.0)
    p.receivers = W.sphere_points(_np.random.default_rng(5), 21900)
    pf = p.write(workdir / "wide.in")
    model = Model(p.model_file)
    engine.set_solver("batched")
    engine.upload(model)
    got = engine.run(Event(model, Params(pf)))
    pick = [0, 21844, 21845, 21899]
    p.receivers = [p.receivers[k] for k in pick]
    want = yo.Problem(p.write(workdir / "pick.in")).run(nthreads=8)
    for i, k in enumerate(pick):
        for c in range(1, 4):
            assert rel_l2(got[k, c], want[i, c]) <= TOL, (k, c)
