"""Frequency shards on the GPU: shards computed one after the other on one
GPU interleave to the whole-band spectra bit for bit (omega is formed from
the full-band index; the solve schedule is fixed, since the two schedules'
kernels may round a few operations differently), and the sharded event
path gives the one-GPU traces."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from conftest import rel_l2
from yspec_b200 import Engine, Event, Model, Params, native as N, shard, workloads as W

pytestmark = pytest.mark.gpu


def _event(workdir):
    p = W.config("c1", seed=8, lmax=30, fmax=5.0, f21=3.5, f22=4.5, dt=20.0, tout=40.0, ats=1)[0]
    p.receivers = p.receivers[:5]
    pf = p.write(workdir / "sh.in")
    m = Model(p.model_file)
    return m, Event(m, Params(pf))


@pytest.mark.parametrize("world", [2, 3])
def test_shards_interleave_to_full_band(workdir, world):
    m, ev = _event(workdir)
    eng = Engine(0)
    eng.set_schedule(0)
    eng.upload(m)
    full = eng.spectra(ev)
    parts = [[], [], []]
    for r in range(world):
        sub = shard.shard_event(ev.raw.ev, world, r)
        bufs = [np.zeros((ev.nr, sub.nw, 2)) for _ in range(3)]
        N.check(N.lib().ysg_event_spectra(eng.h, C.byref(sub), *[N.dptr(b) for b in bufs]), "spectra")
        for c in range(3):
            parts[c].append(bufs[c][..., 0] + 1j * bufs[c][..., 1])
    for c in range(3):
        np.testing.assert_array_equal(shard.interleave(parts[c], ev.nw), full[c])


def test_sharded_event_path_single_rank(workdir):
    import torch.distributed as dist
    from datetime import timedelta

    s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        m, ev = _event(workdir)
        eng = Engine(0)
        eng.upload(m)
        want = eng.run(ev)
        got = shard.run_event_sharded(eng, ev)
        assert got.shape == want.shape
        for k in range(ev.nr):
            for c in range(1, 4):
                assert rel_l2(got[k, c], want[k, c]) <= 1e-9
    finally:
        dist.destroy_process_group()


def _shard_worker(rank, world, port, pf, model_file, out):
    import sys
    from datetime import timedelta

    import torch.distributed as dist
    from conftest import ROOT

    sys.path.insert(0, str(ROOT))
    from yspec_b200 import Engine, Event, Model, Params, shard as S

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        m = Model(model_file)
        ev = Event(m, Params(pf))
        eng = Engine(0)
        eng.set_schedule(0)
        eng.upload(m)
        got = S.run_event_sharded(eng, ev)
        if rank == 0:
            np.save(out, got)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_event_two_ranks_share_one_gpu(workdir, world):
    """run_event_sharded with world ranks (gloo, one process each, all on
    cuda:0): frequency shards, the receiver exchange, per-rank time series of
    its receivers and the row gather reproduce the one-rank sharded run bit
    for bit, and the one-GPU traces to 1e-9.  The ranks' kernels never wait
    on one another: the exchange runs on host copies."""
    import torch.multiprocessing as mp
    import torch.distributed as dist
    from datetime import timedelta

    p = W.config("c1", seed=8, lmax=30, fmax=5.0, f21=3.5, f22=4.5, dt=20.0, tout=40.0, ats=1)[0]
    p.receivers = W.sphere_points(np.random.default_rng(4), 7)
    pf = p.write(workdir / "sh2.in")
    port = _port()
    out = str(workdir / "sharded.npy")
    mp.start_processes(_shard_worker, args=(world, port, str(pf), p.model_file, out), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(out)
    m = Model(p.model_file)
    ev = Event(m, Params(pf))
    eng = Engine(0)
    eng.set_schedule(0)
    eng.upload(m)
    want = eng.run(ev)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_port())
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        one = shard.run_event_sharded(eng, ev)
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(got, one)
    for k in range(ev.nr):
        for c in range(1, 4):
            assert rel_l2(got[k, c], want[k, c]) <= 1e-9


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port
