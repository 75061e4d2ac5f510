"""Multi-rank frequency sharding on CPU: two gloo ranks each compute the
per-(omega,l) coefficients of their interleaved frequency shard (with the
oracle standing in for a GPU), all-gather them, and must reassemble exactly
the single-process result.  Covers the shard arithmetic, the padded
all-gather and the interleaving used by run_event_sharded."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, pf, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist
    from datetime import timedelta

    import yo
    from yspec_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    P = yo.Problem(pf)
    nw, L = P.nw, P.params.lmax + 1
    jofs, jstride, count = shard.shard_frequencies(nw, world, rank)
    local = np.zeros((L, 15, count), complex)
    for i, j0 in enumerate(range(jofs, nw, jstride)):
        for l in range(L):
            local[l, :, i] = P.coef(l, j0 + 1)
    full = shard.all_gather_interleaved(local, nw)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_frequency_shards(tmp_path):
    sys.path.insert(0, str(ROOT / "oracle"))
    import yo
    from yspec_b200 import workloads as W

    p = W.config("c1", seed=4, lmax=6, fmax=3.0, f21=2.0, f22=2.8, dt=40.0, tout=30.0)[0]
    p.receivers = p.receivers[:1]
    pf = str(p.write(tmp_path / "g.in"))
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, pf, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
        assert pr.exitcode == 0
    P = yo.Problem(pf)
    want = np.array([[P.coef(l, j) for j in range(1, P.nw + 1)] for l in range(P.params.lmax + 1)])
    want = np.transpose(want, (0, 2, 1))                    # (L, 15, nw)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        np.testing.assert_array_equal(got, want)


def test_shard_arithmetic():
    from yspec_b200 import native as N, shard

    for nw in (1, 2, 7, 820):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                jofs, js, cnt = shard.shard_frequencies(nw, world, r)
                seen += list(range(jofs, nw, js))[:cnt]
            assert sorted(seen) == list(range(nw))
    ev = N.YsgEvent(nw=820, jofs=0, jstride=1)
    sub = shard.shard_event(ev, 8, 3)
    assert (sub.jofs, sub.jstride, sub.nw) == (3, 8, 103)
    with pytest.raises(ValueError):
        shard.shard_event(sub, 2, 0)
    parts = [np.arange(r, 10, 3)[None, :].astype(float) for r in range(3)]
    np.testing.assert_array_equal(shard.interleave(parts, 10), np.arange(10)[None, :])
