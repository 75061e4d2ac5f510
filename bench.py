"""Benchmark: (omega,l) radial solves per second on the single-event-at-scale workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--solver batched|plain]

One step = the whole hot path for one event: Legendre table, every
(omega,l) radial solve, the receiver l-sum, filter + inverse FFT +
post-processing.  Workload (synthetic, seeded): lmax 750, fmax 50 mHz,
120 min at 1 s, 100 receivers uniform on the sphere, attenuation and full
self-gravitation, acceleration output with potential/tilt corrections,
200-knot PREM-like model, source depth U(0, 700) km: 615,820 (omega,l) pairs.

Multi-GPU: every rank runs its own copy of the event (replicas, weak scaling;
the pairs are independent, no collective is on the data path).  With
--shard, one event is split over the ranks instead: frequency shards, one
NCCL all-to-all to receiver shards, a row gather of the traces (strong
scaling).  Timing is on
the device with CUDA events on the engine's stream, max over ranks.
The reference arm (--impl reference) times the CPU restatement of the
reference path on all host cores over the whole event, every step.

On one GPU the line also carries "batched_vs_plain": the 64-event uneven
batch (fmax U(10, 50) mHz, lmax 15 fmax, depth U(0, 700) km, 1-1000
receivers) run once as one batched solve launch inside a CUDA graph and
once event by event with the plain one-thread-per-pair solver, one launch
per event; "c5_batch": the largest configuration (16 events x 10,000
receivers) as one batch; "parity": the timed event's traces against the
oracle's; "stage_roofline": the l-sum and time-series stages against their
peaks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "(omega,l) radial solves/s"
UNIT = "solves/s"
WORKLOAD = ("single event at scale: lmax 750, fmax 50 mHz, 120 min @ 1 s, 100 receivers, "
            "attenuation + self-gravitation, acceleration with potential/tilt corrections, "
            "200-knot model")


def make_event(tmp: Path, seed: int = 0):
    from yspec_b200 import workloads as W

    p = W.config("c2", seed=seed)[0]
    pf = p.write(tmp / "c2.in")
    return p, pf


def batch_compare(local: int, reps: int = 2) -> dict:
    """c3 (64 uneven events): batched graph vs plain per-event launches."""
    from yspec_b200 import Engine, Event, Model, Params, workloads as W

    tmp = Path(tempfile.mkdtemp(prefix="ysbatch_"))
    ps = W.config("c3", seed=0)
    model = Model(ps[0].model_file)
    evs = [Event(model, Params(p.write(tmp / f"e{i}.in"))) for i, p in enumerate(ps)]
    pairs = float(sum(e.L * e.nw for e in evs))
    traces = float(sum(e.nr for e in evs))
    eng = Engine(local, solver="batched")
    eng.upload(model)
    res = {}
    for solver in ("batched", "plain"):
        eng.set_solver(solver)
        if solver == "batched":
            eng.batch_run(evs)                                   # warm-up, graph instantiation
        else:
            eng.run(evs[0])
        best = None
        for _ in range(reps):
            t0 = time.perf_counter()
            solve = dev = 0.0
            launches = 0
            if solver == "batched":
                eng.batch_run(evs)
                ms = eng.timings()
                solve, dev = ms[1], sum(ms)
                launches = eng.launches()
            else:
                for e in evs:
                    eng.run(e)
                    ms = eng.timings()
                    solve += ms[1]
                    dev += sum(ms)
                    launches += eng.launches()
            wall = time.perf_counter() - t0
            r = {"solve_ms": solve, "device_ms": dev, "wall_ms": 1e3 * wall, "gpu_launches": launches,
                 "solves_per_s": pairs / (solve / 1e3),
                 "pipeline_solves_per_s": pairs / (dev / 1e3),
                 "e2e_solves_per_s": pairs / wall, "traces_per_s": traces / (dev / 1e3)}
            if solver == "batched":
                r["schedule"], r["autotune_solve_ms"] = eng.last_schedule()
            if best is None or r["device_ms"] < best["device_ms"]:
                best = r
        res[solver] = best
    res["workload"] = ("64 uneven events (c3, seed 0): fmax U(10,50) mHz, lmax 15 fmax, "
                       "depth U(0,700) km, receivers log-uniform 1..1000, 60 min")
    res["pairs"] = int(pairs)
    res["traces"] = int(traces)
    res["ratio_solve"] = res["batched"]["solves_per_s"] / res["plain"]["solves_per_s"]
    res["ratio_pipeline"] = res["batched"]["pipeline_solves_per_s"] / res["plain"]["pipeline_solves_per_s"]
    res["ratio_e2e"] = res["batched"]["e2e_solves_per_s"] / res["plain"]["e2e_solves_per_s"]
    res["timing"] = ("device: CUDA events around each stage group on the engine stream; "
                     "plain = sum over events; best of %d" % reps)
    return res


def cpu_sample(pf: Path, stride: int, threads: int, keep: bool = False):
    """Oracle on every stride-th frequency of the event: (pairs, seconds, nw, L),
    and with keep=True also the oracle problem and its spectra."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import yo  # the CPU restatement of the reference path (test oracle / baseline only)

    P = yo.Problem(pf)
    nj = (P.nw - 1) // stride + 1
    L = P.params.lmax - P.params.lmin + 1
    t0 = time.perf_counter()
    spec = P.spectra(nthreads=threads, jsub=-stride)
    dt = time.perf_counter() - t0
    if keep:
        return nj * L, dt, P.nw, L, P, spec
    return nj * L, dt, P.nw, L


def trace_parity(got, P, spec) -> dict:
    """Largest relative L2 error per trace of the device traces (nr, 4, nout)
    against the oracle's traces of the same event, and whether the time
    columns are equal."""
    import numpy as np

    want = P.traces(*spec)
    worst = 0.0
    for k in range(want.shape[0]):
        for c in range(1, 4):
            den = float(np.linalg.norm(want[k, c]))
            num = float(np.linalg.norm(got[k, c] - want[k, c]))
            worst = max(worst, num / den if den > 0 else num)
    return {"max_rel_l2_per_trace": worst, "bar": 1e-9, "ok": bool(worst <= 1e-9),
            "time_column_equal": bool(np.array_equal(got[:, 0], want[:, 0])),
            "checked": "traces of the timed end-to-end run against the oracle's traces of the "
                       "whole event (every receiver and component)"}


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [l.split(",") for l in open(self.path).read().splitlines() if l.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of the solve kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(f.read_text())
        return d.get(kernel)
    except Exception:
        return None


def gradient_check(local: int) -> dict:
    """The differentiable path at the c4 size: misfit gradient with respect to
    3 x 200 knot parameters and the moment tensor (adjoint.ModelSynthetics:
    forward = six unit responses in one batch; backward = reverse mode, one
    Engine.gradient call -- time-stage and l-sum transposes, the reverse
    sweep of every (omega, l) solve -- then autograd through the model
    chain), wall-clock timed on the host with a device sync (the best of
    three backward passes), and the gradient checked along 20 random
    directions against central differences of the misfit."""
    import numpy as np
    import torch
    from yspec_b200 import Engine, Event, Params, adjoint, workloads as W
    from yspec_b200.model_chain import KnotModel

    tmp = Path(tempfile.mkdtemp(prefix="ysgrad_"))
    p = W.config("c4", seed=0)[0]
    pf = p.write(tmp / "c4.in")
    km = KnotModel(p.model_file)
    ev = Event(km.host, Params(pf))
    eng = Engine(local)
    syn = adjoint.ModelSynthetics(eng, ev, km)
    P0 = km.params()
    mm0 = torch.tensor(p.mm, dtype=torch.float64)
    # observed traces: the model with seeded 1% Gaussian-smoothed (3 knots)
    # perturbations of rho, Vp and Vs at every knot
    rng = np.random.default_rng(11)
    kern = np.exp(-0.5 * (np.arange(-9, 10) / 3.0) ** 2)
    kern /= kern.sum()
    Pobs = tuple(x * (1.0 + torch.from_numpy(np.convolve(rng.standard_normal(km.nknot), kern, mode="same")) * 1e-2)
                 for x in P0)
    obs = syn(*Pobs, mm0).detach()
    syn(*P0, mm0)                                   # warm-up (module loading, graphs)
    fwd, bwd, sweeps = [], [], []
    for rep in range(3):
        rho, vp, vs = (x.clone().requires_grad_() for x in P0)
        mm = mm0.clone().requires_grad_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = 0.5 * ((syn(rho, vp, vs, mm) - obs) ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        fwd.append(t1 - t0)
        bwd.append(t2 - t1)
        sweeps.append(eng.timings()[1])
    grad = (rho.grad, vp.grad, vs.grad, mm.grad)
    errs = []
    for k in range(20):
        r = np.random.default_rng(100 + k)
        dk = tuple(torch.from_numpy(r.standard_normal(km.nknot)) * x * 1e-2 for x in P0)
        dm = torch.from_numpy(r.standard_normal(6)) * 1e18
        with torch.no_grad():
            lp = float(0.5 * ((syn(*(x + 1e-3 * y for x, y in zip(P0, dk)), mm0 + 1e-3 * dm) - obs) ** 2).sum())
            lm = float(0.5 * ((syn(*(x - 1e-3 * y for x, y in zip(P0, dk)), mm0 - 1e-3 * dm) - obs) ** 2).sum())
        fd = (lp - lm) / 2e-3
        ad = sum(float((g * y).sum()) for g, y in zip(grad, dk + (dm,)))
        errs.append(abs(ad - fd) / abs(fd))
    return {"workload": "c4: lmax 300, fmax 20 mHz, 60 min @ 5 s, 50 receivers, source 150 km, "
                        "200-knot model, misfit gradient over 3 x 200 knot parameters + 6 moment components",
            "pairs": ev.L * ev.nw, "params": 3 * km.nknot + 6,
            "forward_s": min(fwd), "gradient_s": min(bwd), "gradient_over_forward": min(bwd) / min(fwd),
            "reverse_sweeps_ms": min(sweeps), "backend": syn.last_method,
            "method": "reverse mode: trace adjoint through the time-stage and l-sum transposes, discrete "
                      "adjoint of every (omega, l) solve (k_solve_adjoint), autograd through the model chain",
            "fd_rel_err": max(errs), "fd_check": "central differences along 20 random directions, step 1e-3"}


def measured_peaks() -> dict:
    """The pool's measured HBM copy bandwidth (GB/s), if the file is present."""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "MEASURED_PEAKS.json (measured)"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback: earlier measurement on this pool"}


def c5_batch(local: int) -> dict:
    """c5: 16 events x 10,000 receivers on the 400-knot model, lmax 1500,
    100 mHz, 120 min at 0.5 s, as one ysg_batch_run (one solve stage over
    39.4 M pairs, per-event l-sum and time series, one CUDA graph).  The
    traces (74 GB) exceed the host's memory beside everything else, so every
    event writes into one shared pinned host buffer; all device-to-host
    copies are still made and timed.  One warm-up batch, then one timed
    batch."""
    import numpy as np
    from yspec_b200 import Engine, Event, Model, Params, workloads as W

    tmp = Path(tempfile.mkdtemp(prefix="ysc5_"))
    ps = W.config("c5", seed=0)
    model = Model(ps[0].model_file)
    t0 = time.perf_counter()
    evs = [Event(model, Params(p.write(tmp / f"e{i}.in"))) for i, p in enumerate(ps)]
    setup_s = time.perf_counter() - t0
    eng = Engine(local, solver="batched")
    eng.set_schedule(2)
    eng.upload(model)
    import torch

    # one pinned host buffer shared by every event (page-locked copies)
    buf = torch.empty((evs[0].nr, 4, evs[0].nout()), dtype=torch.float64, pin_memory=True).numpy()
    eng.batch_run(evs, outs=[buf] * len(evs))           # warm-up: graph capture
    t0 = time.perf_counter()
    eng.batch_run(evs, outs=[buf] * len(evs))
    wall = time.perf_counter() - t0
    ms = eng.timings()
    pairs = float(sum(e.L * e.nw for e in evs))
    nrec = sum(e.nr for e in evs)
    return {"workload": "c5: 16 events x 10,000 receivers, 400-knot model, lmax 1500, 100 mHz, "
                        "120 min @ 0.5 s, attenuation + self-gravitation, one batch",
            "pairs": int(pairs), "traces": nrec,
            # a batch runs each event's l-sum and time series back to back,
            # so the two share one interval
            "stage_ms": {"legendre": ms[0], "solve": ms[1], "lsum_and_ifft": ms[2] + ms[3]},
            "wall_s": wall, "traces_per_s": nrec / wall, "solves_per_s_device": pairs / (ms[1] / 1e3),
            "event_setup_s": setup_s,
            "timing": "wall clock of one ysg_batch_run after a warm-up batch, including the "
                      "device-to-host copy of every event's traces (73.7 GB), each started "
                      "when its event's time series is complete"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        _, pf = make_event(Path(d))
        stride = 1                                   # the whole event, every step
        for _ in range(args.warmup):
            cpu_sample(pf, stride, threads)
        times, pairs = [], 0
        for _ in range(args.steps):
            n, dt, nw, L = cpu_sample(pf, stride, threads)
            times.append(dt)
            pairs = n
    total = sum(times)
    value = pairs * args.steps / total
    sample = f"the whole event per step: {nw} frequencies x {L} degrees ({pairs} pairs)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PREM-like model, receivers, moment tensor)",
        "config": {"workload": WORKLOAD, "pairs_per_event": pairs, "sample": sample,
                   "same_config": True},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_sharded(args) -> None:
    """One c2 event split over the ranks (yspec_b200.shard.run_event_sharded):
    each rank solves an interleaved frequency shard for every receiver, one
    NCCL all-to-all moves the spectra to receiver shards, each rank runs the
    time series of its receivers, rank 0 gathers the traces.  Total work is
    fixed as N grows (strong scaling).  A step is one whole event; the
    timed span is bracketed by barriers and device synchronisations and
    measured with CUDA events, max over ranks."""
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from yspec_b200 import Engine, Event, Model, Params, shard as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world == 1 and "MASTER_PORT" not in os.environ:
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(sk.getsockname()[1])
        sk.close()
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    tmp = Path(tempfile.mkdtemp(prefix=f"ysshard{rank}_"))
    p, pf = make_event(tmp)
    model = Model(p.model_file)
    eng = Engine(local, solver="batched")
    eng.set_schedule(2)
    eng.upload(model)
    ev = Event(model, Params(pf))
    pairs = float(ev.L * ev.nw)
    for _ in range(args.warmup):
        S.run_event_sharded(eng, ev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        out = S.run_event_sharded(eng, ev)
    torch.cuda.synchronize()
    e1.record()
    e1.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms = float(ms.item())
    if rank == 0:
        line = {
            "metric": METRIC, "value": pairs * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PREM-like model, receivers, moment tensor)",
            "config": {"workload": WORKLOAD, "pairs_per_event": int(pairs), "receivers": ev.nr,
                       "parallelism": f"frequency shards x{world}, NCCL all-to-all to receiver shards, "
                                      "row gather of the traces on rank 0"},
            "e2e": {"value": pairs * args.steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(out.nbytes) if out is not None else 0},
        }
        print(json.dumps(line), flush=True)
    dist.destroy_process_group()


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    from yspec_b200 import Engine, Event, Model, Params, fp64_peak_tflops

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    tmp = Path(tempfile.mkdtemp(prefix=f"ysbench{rank}_"))
    p, pf = make_event(tmp)
    model = Model(p.model_file)
    eng = Engine(local, solver=args.solver)
    eng.set_schedule(args.schedule)
    eng.upload(model)
    ev = Event(model, Params(pf))
    nr, nout = ev.nr, ev.nout()
    pairs = float(ev.L * ev.nw)
    peak = fp64_peak_tflops(local)

    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    out_pinned = torch.empty(nr * 4 * nout, dtype=torch.float64, pin_memory=True)

    # inputs resident on the device for the kernel-throughput value
    eng.prepare(ev)
    for _ in range(args.warmup):
        eng.execute()
        eng.fetch(None)

    # --- device-timed steps: flush L2, then the whole hot path of one event
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    solve_ms, flops = [], 0.0
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    launches0 = eng.launches()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev0[k].record(stream)
        eng.execute()
        with torch.cuda.stream(stream):
            ev1[k].record(stream)
        eng.fetch(None)                   # host sync; reads the stage timings
        solve_ms.append(eng.timings()[1])
        flops = eng.work()[1]
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = eng.launches() - launches0
    sched = eng.last_schedule()[0] if args.solver == "batched" else None
    barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    dev_ms = allmax(dev_ms)
    value = world * pairs * args.steps / (dev_ms / 1e3)

    # --- end to end through the public C-ABI with host buffers
    e_ms = 0.0
    h2d = d2h = 0.0
    barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        t0 = time.perf_counter()
        eng.prepare(ev)
        eng.execute()
        eng.fetch(out_ptr=out_pinned.data_ptr())
        e_ms += 1e3 * (time.perf_counter() - t0)
        h2d, d2h = eng.bytes_moved()
    barrier()
    e_ms = allmax(e_ms)
    e2e = world * pairs * args.steps / (e_ms / 1e3)
    traces_last = out_pinned.numpy().reshape(nr, 4, nout).copy()

    if rank == 0:
        mean_solve = statistics.mean(solve_ms)
        achieved = flops / (mean_solve / 1e3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PREM-like model, receivers, moment tensor)",
            "config": {"workload": WORKLOAD, "pairs_per_event": int(pairs), "receivers": nr,
                       "nt": ev.tm.nt, "trace_rows": nout, "solver": args.solver,
                       "schedule": sched,
                       "l2": "flushed between timed steps (256 MB write, untimed)",
                       "parallelism": f"replicas x{world}"},
            "traces_per_s": world * nr * args.steps / (dev_ms / 1e3),
            "stage_ms": dict(zip(["legendre", "solve", "lsum", "ifft"], eng.timings())),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e_ms / args.steps},
            "gpu_launches": launches,
            "roofline": {"bound": "fp64", "pipe": "FP64 CUDA-core FMA pipe (the radial solves use no tensor cores)",
                         "kernel": "k_solve_batched" if args.solver == "batched" else "k_solve_plain",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None,
                         "peak_source": "measured: FP64 FMA microbenchmark run by this bench on this GPU",
                         "flops_per_launch": flops, "launch_ms": mean_solve,
                         "traffic": traffic_from_profiles(
                             "k_solve_batched" if args.solver == "batched" else "k_solve_plain")},
            "clocks": clk,
        }
        st = dict(zip(["legendre", "solve", "lsum", "ifft"], eng.timings()))
        hbm = measured_peaks()
        L, nw, nt = ev.L, ev.nw, ev.tm.nt
        lsum_flops = 4.0 * nw * nr * (22 * (L - 2) + 9)
        ifft_bytes = 3.0 * nr * (nw * 16 + nout * 8)
        ifft_flops = 3.0 * nr * 5.0 * nt * (nt.bit_length() - 1)
        line["stage_roofline"] = {
            "lsum": {"kernel": "k_lsum_mma", "bound": "fp64 tensor (DMMA)",
                     "achieved_tflops": lsum_flops / (st["lsum"] / 1e3) / 1e12,
                     "frac_of_fp64_peak": lsum_flops / (st["lsum"] / 1e3) / 1e12 / peak,
                     "flops": lsum_flops},
            "ifft": {"kernels": "k_ifft_a2, k_ifft_b2, k_rotate",
                     "achieved_gbs": ifft_bytes / (st["ifft"] / 1e3) / 1e9,
                     "frac_of_hbm": ifft_bytes / (st["ifft"] / 1e3) / 1e9 / hbm["hbm_gbs"],
                     "hbm_peak_gbs": hbm["hbm_gbs"], "hbm_peak_source": hbm["source"],
                     "fft_tflops": ifft_flops / (st["ifft"] / 1e3) / 1e12,
                     "fft_frac_of_fp64_peak": ifft_flops / (st["ifft"] / 1e3) / 1e12 / peak,
                     "bytes": ifft_bytes, "fft_flops_5nlog2n": ifft_flops}}
        if world == 1 and not args.no_batch:
            line["batched_vs_plain"] = batch_compare(local)
        if world == 1 and not args.no_grad:
            line["gradient"] = gradient_check(local)
        if world == 1 and not args.no_c5:
            line["c5_batch"] = c5_batch(local)
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            n, dt, nw, L, P, spec = cpu_sample(pf, 1, threads, keep=True)
            line["parity"] = trace_parity(traces_last, P, spec)
            n1, dt1, _, _ = cpu_sample(pf, 41, 1)
            line["cpu_baseline"] = {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": f"the whole event: {nw} frequencies x {L} degrees "
                                              f"({n} pairs, {dt:.1f} s on {threads} threads)",
                                    "single_thread": {"value": n1 / dt1, "unit": UNIT, "cores": 1,
                                                      "sample": f"every 41st of {nw} frequencies x "
                                                                f"{L} degrees ({n1} pairs, {dt1:.1f} s)"}}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--solver", default="batched", choices=["batched", "plain"])
    ap.add_argument("--schedule", type=int, default=-1,
                    help="batched-solver schedule: 0 tiles, 1 pair lists, 2 split pair lists, -1 autotuned")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain comparison")
    ap.add_argument("--no-grad", action="store_true", help="skip the c4 model-gradient timing")
    ap.add_argument("--no-c5", action="store_true", help="skip the c5 16-event batch")
    ap.add_argument("--shard", action="store_true",
                    help="one event split over the N GPUs (frequency shards, all-to-all) instead of replicas")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.shard:
        run_sharded(args)
    else:
        run_b200(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
