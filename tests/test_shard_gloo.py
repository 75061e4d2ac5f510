"""Multi-rank sharding on CPU with gloo ranks (world sizes 2 and 3).

(1) The receiver exchange of run_event_sharded: every rank holds the
spectra of its interleaved frequency shard for all receivers; one
all-to-all must leave each rank with the whole band of its own receivers,
and the row gather must reassemble all receivers in order on rank 0 --
checked against a seeded full array.  (2) Frequency shards of the oracle's
per-(omega,l) coefficients (the oracle standing in for a GPU) reassemble
exactly into the single-process result."""
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


def _init(rank, world, port):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    return dist


def _full_spectra(nw, nr):
    rng = np.random.default_rng(1234)
    return rng.standard_normal((3, nr, nw, 2))          # (component, receiver, frequency, re/im)


def _exchange_worker(rank, world, port, nw, nr, out_dir):
    sys.path.insert(0, str(ROOT))
    import torch
    from yspec_b200 import shard

    dist = _init(rank, world, port)
    full = _full_spectra(nw, nr)
    local = torch.from_numpy(np.ascontiguousarray(full[:, :, rank::world]))
    mine = shard.exchange_to_receivers(local, nw, nr)
    np.save(os.path.join(out_dir, f"x{rank}.npy"), mine.numpy())
    rows = shard.gather_rows(torch.from_numpy(np.ascontiguousarray(full[0, rank::world])), nr)
    if rank == 0:
        np.save(os.path.join(out_dir, "rows.npy"), rows.numpy())
    dist.barrier()
    dist.destroy_process_group()


def _coef_worker(rank, world, port, pf, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch
    import yo
    from yspec_b200 import shard

    dist = _init(rank, world, port)
    P = yo.Problem(pf)
    nw, L = P.nw, P.params.lmax + 1
    jofs, jstride, count = shard.shard_frequencies(nw, world, rank)
    local = np.zeros((L, 15, count), complex)
    for i, j0 in enumerate(range(jofs, nw, jstride)):
        for l in range(L):
            local[l, :, i] = P.coef(l, j0 + 1)
    # one all-to-all round trip of the coefficient rows (treated as receivers)
    arr = np.stack([local.real, local.imag], -1).reshape(1, L * 15, count, 2)
    arr = np.concatenate([arr, arr, arr])
    mine = shard.exchange_to_receivers(torch.from_numpy(arr), nw, L * 15).numpy()
    rows = shard.gather_rows(torch.from_numpy(np.ascontiguousarray(mine[0])), L * 15)
    if rank == 0:
        full = rows.numpy()
        np.save(os.path.join(out_dir, "coef.npy"), (full[..., 0] + 1j * full[..., 1]).reshape(L, 15, nw))
    dist.barrier()
    dist.destroy_process_group()


def _spawn(target, world, *args):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port) + args) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
        assert pr.exitcode == 0


@pytest.mark.parametrize("world", [2, 3])
def test_receiver_exchange(tmp_path, world):
    nw, nr = 23, 7
    _spawn(_exchange_worker, world, nw, nr, str(tmp_path))
    full = _full_spectra(nw, nr)
    for r in range(world):
        got = np.load(tmp_path / f"x{r}.npy")
        np.testing.assert_array_equal(got, full[:, r::world])
    np.testing.assert_array_equal(np.load(tmp_path / "rows.npy"), full[0])


def test_two_rank_frequency_shards(tmp_path):
    sys.path.insert(0, str(ROOT / "oracle"))
    import yo
    from yspec_b200 import workloads as W

    p = W.config("c1", seed=4, lmax=6, fmax=3.0, f21=2.0, f22=2.8, dt=40.0, tout=30.0)[0]
    p.receivers = p.receivers[:1]
    pf = str(p.write(tmp_path / "g.in"))
    _spawn(_coef_worker, 2, pf, str(tmp_path))
    P = yo.Problem(pf)
    want = np.array([[P.coef(l, j) for j in range(1, P.nw + 1)] for l in range(P.params.lmax + 1)])
    want = np.transpose(want, (0, 2, 1))                    # (L, 15, nw)
    np.testing.assert_array_equal(np.load(tmp_path / "coef.npy"), want)


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
