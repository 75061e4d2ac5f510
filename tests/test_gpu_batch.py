"""Several events in one batch (ysg_batch_run): one solve launch over the
items of every event, the whole batch captured in a CUDA graph.

Each event of an uneven batch (different frequency bands, degree ranges,
source depths, receiver counts, switches) must give the traces the CPU
oracle gives for that event alone, to 1e-9 relative L2 per trace, with the
batched and the plain solver; repeating a batch (the graph is updated in
place) and changing its shape (re-instantiated) must give the same result.
"""
import numpy as np
import pytest

import yo
from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-9

# uneven events sharing one model: bands, degrees, depths, switches, receivers
EVENTS = [
    dict(lmax=30, fmax=5.0, f21=4.0, f22=4.8, dt=20.0, tout=40.0, ats=1, nrec=3),
    dict(lmax=45, fmax=7.0, f21=5.5, f22=6.5, dt=20.0, tout=40.0, ats=1, out=2, cor=1,
         depth_s=500.0, nrec=1),
    dict(lmax=20, fmax=4.0, f21=3.0, f22=3.8, dt=40.0, tout=30.0, grav=1, depth_s=30.0, nrec=5),
    dict(lmin=3, lmax=25, fmax=5.0, f21=4.0, f22=4.8, dt=20.0, tout=40.0, grav=0, out=1, nrec=2),
    dict(lmax=35, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0, ats=1, depth_s=20.0,
         depth_r=250.0, nrec=2),
]


def _events(workdir, specs, seed0=11):
    out = []
    for i, spec in enumerate(specs):
        spec = dict(spec)
        nrec = spec.pop("nrec")
        p = W.config("c1", seed=seed0 + i, **spec)[0]
        p.receivers = p.receivers[:nrec]
        pf = p.write(workdir / f"b{i}.in")
        out.append((p, pf))
    return out


@pytest.fixture(scope="module")
def engine():
    return Engine(0)


@pytest.mark.parametrize("solver", ["batched", "plain"])
def test_batch_matches_oracle(engine, workdir, solver):
    cases = _events(workdir, EVENTS)
    model = Model(cases[0][0].model_file)
    engine.set_solver(solver)
    engine.upload(model)
    evs = [Event(model, Params(pf)) for _, pf in cases]
    got = engine.batch_run(evs)
    for i, ((p, pf), g) in enumerate(zip(cases, got)):
        want = yo.Problem(pf).run(nthreads=8)
        assert g.shape == want.shape
        np.testing.assert_array_equal(g[:, 0], want[:, 0])
        for k in range(g.shape[0]):
            for c in range(1, 4):
                err = rel_l2(g[k, c], want[k, c])
                assert err <= TOL, f"event {i} receiver {k} comp {c}: {err:.3e}"
    pairs, _ = engine.work()
    assert pairs == sum(e.L * e.nw for e in evs)


def test_batch_repeat_and_reshape(engine, workdir):
    # one fixed schedule: the autotuner may choose differently per batch shape
    cases = _events(workdir, EVENTS)
    model = Model(cases[0][0].model_file)
    engine.set_solver("batched")
    engine.set_schedule(1)
    engine.upload(model)
    evs = [Event(model, Params(pf)) for _, pf in cases]
    first = engine.batch_run(evs)
    again = engine.batch_run(evs)                 # same shape: graph updated in place
    for a, b in zip(first, again):
        np.testing.assert_array_equal(a, b)
    sub = engine.batch_run(evs[1:4])              # new shape: graph rebuilt
    for a, b in zip(first[1:4], sub):
        np.testing.assert_array_equal(a, b)
    single = engine.run(evs[2])                   # single-event path after a batch
    np.testing.assert_array_equal(single, first[2])
    rev = engine.batch_run(evs[::-1])             # order does not matter
    for a, b in zip(first[::-1], rev):
        np.testing.assert_array_equal(a, b)
    engine.set_schedule(-1)


def test_schedules_agree(engine, workdir):
    """Every work schedule (tiles, cost-sorted pair lists, the lists split
    into a spheroidal and a toroidal launch) and the autotuned choice give
    the same traces: each pair is computed by one thread with
    the same arithmetic whatever lane or warp it lands in.  The two kernel
    instantiations inline the pair code separately, so the compiler may
    round a few operations differently: agreement is to 1e-12 relative L2
    (far inside the 1e-9 bar), and each schedule is checked against the
    oracle on its own."""
    cases = _events(workdir, EVENTS)
    model = Model(cases[0][0].model_file)
    engine.set_solver("batched")
    engine.upload(model)
    evs = [Event(model, Params(pf)) for _, pf in cases]
    runs = {}
    for sched in (0, 1, 2, -1):
        engine.set_schedule(sched)
        runs[sched] = engine.batch_run(evs)
        used, _ = engine.last_schedule()
        assert used in (0, 1, 2) and (sched < 0 or used == sched)
    for s in (1, 2, -1):
        for a, b in zip(runs[0], runs[s]):
            np.testing.assert_array_equal(a[:, 0], b[:, 0])
            for k in range(a.shape[0]):
                for c in range(1, 4):
                    assert rel_l2(b[k, c], a[k, c]) <= 1e-12
    for (p, pf), g1, g2 in zip(cases, runs[1], runs[2]):
        want = yo.Problem(pf).run(nthreads=8)
        for g in (g1, g2):
            for k in range(g.shape[0]):
                for c in range(1, 4):
                    assert rel_l2(g[k, c], want[k, c]) <= TOL
    engine.set_schedule(1)
    single = engine.run(evs[1])
    np.testing.assert_array_equal(single, runs[1][1])
    engine.set_schedule(-1)


def test_c3_batch_at_size_matches_oracle(engine, workdir):
    """The benchmarked 64-event uneven batch (c3) in one ysg_batch_run; six
    of its events checked against the oracle run of each alone: the three
    lowest bands (10.3-10.9 mHz), a shallow 30 km source, a 13.7 mHz band,
    and the 48 mHz, lmax 722 event."""
    ps = W.config("c3", seed=0)
    model = Model(ps[0].model_file)
    pfs = [p.write(workdir / f"c3_{i}.in") for i, p in enumerate(ps)]
    engine.set_solver("batched")
    engine.upload(model)
    got = engine.batch_run([Event(model, Params(pf)) for pf in pfs])
    for i in (26, 62, 19, 10, 45, 4):
        want = yo.Problem(pfs[i]).run(nthreads=16)
        assert got[i].shape == want.shape, i
        np.testing.assert_array_equal(got[i][:, 0], want[:, 0])
        for k in range(want.shape[0]):
            for c in range(1, 4):
                assert rel_l2(got[i][k, c], want[k, c]) <= TOL, (i, k, c)
