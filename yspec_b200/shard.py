"""One event over several GPUs: frequency shards, then receiver shards.

Every (omega,l) solve is independent, so rank r of W takes the frequencies
j = r+1, r+1+W, ... (interleaved, which balances the cost that grows with
omega) and computes their spectra for every receiver on its own GPU.  The
ysg_event fields jofs and jstride carry the shard, so each GPU forms omega
exactly as a one-GPU run does.  One all-to-all over NCCL (NVLink /
NVSwitch) then transposes frequency shards into receiver shards: rank r
sends rank q the spectra of q's receivers (k = q, q+W, ...) at r's
frequencies, 3 nw nr complex values in total, and each rank runs the
time-series stage for its own receivers on its own GPU.  Rank 0 gathers
the traces.  Spectra stay in device memory from the solve to the
transform.  Batches of many events need none of this: events are split
between ranks (replicas, no collective).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


def shard_frequencies(nw: int, world: int, rank: int) -> tuple[int, int, int]:
    """(jofs, jstride, count) of rank's interleaved frequency shard."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    count = len(range(rank, nw, world))
    return rank, world, count


def shard_event(ev: N.YsgEvent, world: int, rank: int) -> N.YsgEvent:
    """Copy of a whole-band event restricted to rank's frequency shard."""
    if ev.jofs != 0 or ev.jstride != 1:
        raise ValueError("event is already a shard")
    jofs, jstride, count = shard_frequencies(ev.nw, world, rank)
    sub = type(ev).from_buffer_copy(ev)
    sub.jofs, sub.jstride, sub.nw = jofs, jstride, count
    return sub


def interleave(parts: list[np.ndarray], nw: int) -> np.ndarray:
    """Reassemble per-rank (..., count_r) arrays into (..., nw) in frequency order."""
    world = len(parts)
    out = np.zeros(parts[0].shape[:-1] + (nw,), dtype=parts[0].dtype)
    for r, p in enumerate(parts):
        out[..., r::world] = p[..., : len(range(r, nw, world))]
    return out


def exchange_to_receivers(local, nw: int, nr: int, group=None):
    """Transpose frequency shards into receiver shards with one all-to-all.

    local: real tensor (3, nr, count_r, 2) -- this rank's spectra (ur, ut,
    up; (re, im) pairs) for every receiver at its frequencies j = r, r+W, ...
    Returns (3, nr_mine, nw, 2) on local's device: the whole band for the
    receivers k = r, r+W, ...  Shards differ in length by at most one and
    are padded to equal blocks for the collective.
    """
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    cmax = -(-nw // world)
    kmax = -(-nr // world)
    cnt = local.shape[2]
    send = torch.zeros((world, 3, kmax, cmax, 2), dtype=local.dtype, device=local.device)
    for q in range(world):
        ks = torch.arange(q, nr, world, device=local.device)
        send[q, :, : ks.numel(), :cnt] = local[:, ks]
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    mine = len(range(rank, nr, world))
    out = torch.zeros((3, mine, nw, 2), dtype=local.dtype, device=local.device)
    for s in range(world):
        cs = len(range(s, nw, world))
        out[:, :, s::world] = recv[s, :, :mine, :cs]
    return out


def gather_rows(local, n: int, group=None, dst: int = 0):
    """All-gather per-rank rows k = r, r+W, ... (first axis) into n rows in k
    order; returns the full tensor on rank dst, None elsewhere."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    kmax = -(-n // world)
    pad = torch.zeros((kmax,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    if rank != dst:
        return None
    out = torch.zeros((n,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, g in enumerate(parts):
        m = len(range(r, n, world))
        out[r::world] = g[:m]
    return out


def run_event_sharded(engine, event, group=None) -> np.ndarray | None:
    """Traces of one event computed by all ranks of `group`; rank 0 returns
    (nr, 4, nout), the others None.  The engine's device is the rank's GPU
    (NCCL); with a gloo group the collectives run on host copies instead."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device())
    sub = shard_event(event.raw.ev, world, rank)
    nr, nw = event.nr, event.nw
    # this rank's frequency shard for every receiver, on the device
    spec = torch.zeros((3, nr, sub.nw, 2), dtype=torch.float64, device=dev)
    N.check(N.lib().ysg_event_spectra_device(engine.h, C.byref(sub), spec[0].data_ptr(),
                                             spec[1].data_ptr(), spec[2].data_ptr()), "spectra")
    coll = spec if on_gpu else spec.cpu()
    mine_spec = exchange_to_receivers(coll, nw, nr, group).to(dev).contiguous()
    # time series of this rank's receivers
    mine = np.arange(rank, nr, world)
    tm = N.YsgTime.from_buffer_copy(event.raw.tm)
    tm.nr = len(mine)
    nout = N.lib().ysg_trace_rows(C.byref(tm))
    azep = np.ctypeslib.as_array(event.raw.azep, (nr,))[mine].copy()
    d_az = torch.from_numpy(azep).to(dev)
    d_out = torch.zeros((len(mine), 4, nout), dtype=torch.float64, device=dev)
    if len(mine):
        n = C.c_int()
        N.check(N.lib().ysg_traces_noalloc(C.byref(tm), mine_spec[0].data_ptr(), mine_spec[1].data_ptr(),
                                           mine_spec[2].data_ptr(), d_az.data_ptr(), d_out.data_ptr(),
                                           C.byref(n), None), "traces")
        torch.cuda.synchronize(dev)
    full = gather_rows(d_out if on_gpu else d_out.cpu(), nr, group)
    return None if full is None else full.cpu().numpy()
