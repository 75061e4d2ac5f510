"""One event over several GPUs: frequency shards, then receiver shards.

Every (omega,l) solve is independent, so rank r of W takes the frequencies
j = r+1, r+1+W, ... (interleaved, which balances the cost that grows with
omega) and computes their spectra for every receiver on its own GPU.  One
all-gather over NCCL (NVLink / NVSwitch) gives every rank the whole
(nw, nr) spectra; each rank then runs the time-series stage for its own
receivers and rank 0 gathers the traces.  The ysg_event fields jofs and
jstride carry the shard, so each GPU forms omega exactly as a one-GPU run
does.  Batched workloads of many events need none of this: events are
simply split between ranks (replicas, no collective).
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


def all_gather_interleaved(local: np.ndarray, nw: int, group=None, device=None) -> np.ndarray:
    """Gather every rank's frequency shard (last axis) and interleave them.

    Shards differ in length by at most one; they are padded to the longest
    for the collective.  Complex arrays travel as (re, im) float64 pairs.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    width = -(-nw // world)
    cplx = np.iscomplexobj(local)
    arr = np.stack([local.real, local.imag], -1) if cplx else local[..., None]
    pad = np.zeros(arr.shape[:-2] + (width, arr.shape[-1]))
    pad[..., : arr.shape[-2], :] = arr
    t = torch.from_numpy(pad)
    if device is not None:
        t = t.to(device)
    bufs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(bufs, t, group=group)
    parts = []
    for b in bufs:
        b = b.cpu().numpy()
        parts.append(b[..., 0] + 1j * b[..., 1] if cplx else b[..., 0])
    return interleave(parts, nw)


def run_event_sharded(engine, event, group=None, device=None) -> np.ndarray | None:
    """Traces of one event computed by all ranks of `group`; rank 0 returns
    (nr, 4, nout), the others None.  `device` holds the collective buffers
    (the rank's CUDA device for NCCL, None for CPU tensors with gloo); the
    time-series stage always runs on the current CUDA device."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    sub = shard_event(event.raw.ev, world, rank)
    nr, nw = event.nr, event.nw
    bufs = [np.zeros((nr, sub.nw, 2)) for _ in range(3)]
    N.check(N.lib().ysg_event_spectra(engine.h, C.byref(sub), *[N.dptr(b) for b in bufs]), "spectra")
    local = [b[..., 0] + 1j * b[..., 1] for b in bufs]
    full = [all_gather_interleaved(x, nw, group, device) for x in local]     # (nr, nw) each
    # receiver shard for the time-series stage
    mine = np.arange(rank, nr, world)
    tm = N.YsgTime.from_buffer_copy(event.raw.tm)
    tm.nr = len(mine)
    nout = N.lib().ysg_trace_rows(C.byref(tm))
    dev = torch.device("cuda", torch.cuda.current_device())
    coll = device if device is not None else torch.device("cpu")
    def dspec(a):
        return torch.from_numpy(np.ascontiguousarray(np.stack([a[mine].real, a[mine].imag], -1))).to(dev)
    azep = np.ctypeslib.as_array(event.raw.azep, (nr,))[mine].copy()
    d_az = torch.from_numpy(azep).to(dev)
    d_out = torch.zeros((len(mine), 4, nout), dtype=torch.float64, device=dev)
    if len(mine):
        d = [dspec(a) for a in full]
        f = N.lib().ysg_traces_noalloc
        f.argtypes = [C.POINTER(N.YsgTime)] + [C.c_void_p] * 5 + [C.POINTER(C.c_int), C.c_void_p]
        n = C.c_int()
        N.check(f(C.byref(tm), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d_az.data_ptr(),
                  d_out.data_ptr(), C.byref(n), None), "traces")
        torch.cuda.synchronize(dev)
    local_tr = d_out.cpu().numpy()                                          # (count, 4, nout)
    width = -(-nr // world)
    pad = torch.zeros((width, 4, nout), dtype=torch.float64, device=coll)
    pad[: len(mine)] = torch.from_numpy(local_tr).to(coll)
    gathered = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(gathered, pad, group=group)
    if rank != 0:
        return None
    out = np.zeros((nr, 4, nout))
    for r, g in enumerate(gathered):
        idx = np.arange(r, nr, world)
        out[idx] = g.cpu().numpy()[: len(idx)]
    return out
