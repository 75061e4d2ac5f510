"""Benchmark: (omega,l) radial solves per second on the single-event-at-scale workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--solver batched|plain]

One step = the whole hot path for one event: Legendre table, every
(omega,l) radial solve, the receiver l-sum, filter + inverse FFT +
post-processing.  Workload (synthetic, seeded): lmax 750, fmax 50 mHz,
120 min at 1 s, 100 receivers uniform on the sphere, attenuation and full
self-gravitation, acceleration output with potential/tilt corrections,
200-knot PREM-like model, source depth U(0, 700) km: 615,820 (omega,l) pairs.

Multi-GPU: every rank runs its own copy of the event (replicas, weak scaling;
the pairs are independent, no collective is on the data path).  Timing is on
the device with CUDA events on the engine's stream, max over ranks.
The reference arm (--impl reference) times the CPU restatement of the
reference path on all host cores over a bounded frequency sample.

On one GPU the line also carries "batched_vs_plain": the 64-event uneven
batch (fmax U(10, 50) mHz, lmax 15 fmax, depth U(0, 700) km, 1-1000
receivers) run once as one batched solve launch inside a CUDA graph and
once event by event with the plain one-thread-per-pair solver, one launch
per event.
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


def cpu_sample(pf: Path, stride: int, threads: int):
    """Oracle on every stride-th frequency of the event: (pairs, seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import yo  # the CPU restatement of the reference path (test oracle / baseline only)

    P = yo.Problem(pf)
    nj = (P.nw - 1) // stride + 1
    L = P.params.lmax - P.params.lmin + 1
    t0 = time.perf_counter()
    P.spectra(nthreads=threads, jsub=-stride)
    dt = time.perf_counter() - t0
    return nj * L, dt, P.nw, L


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
    forward = six unit responses in one batch, backward = one tangent-linear
    solve per knot parameter, batches of 64), wall-clock timed on the host
    with a device sync, and the gradient checked along two random directions
    against central differences of the misfit."""
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
    rng = np.random.default_rng(11)
    obs = syn(*(x * (1.0 + torch.from_numpy(rng.standard_normal(km.nknot)) * 1e-3) for x in P0), mm0).detach()
    syn(*P0, mm0)                                   # warm-up (module loading, graphs)
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
    grad = (rho.grad, vp.grad, vs.grad, mm.grad)
    errs = []
    for k in range(2):
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
            "forward_s": t1 - t0, "gradient_s": t2 - t1,
            "method": "forward mode: tangent-linear solve per knot parameter, 64 per batched launch",
            "fd_rel_err": max(errs), "fd_check": "central differences along 2 random directions, step 1e-3"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        _, pf = make_event(Path(d))
        stride = 8                                   # 103 of 820 frequencies per step
        for _ in range(args.warmup):
            cpu_sample(pf, stride, threads)
        times, pairs = [], 0
        for _ in range(args.steps):
            n, dt, nw, L = cpu_sample(pf, stride, threads)
            times.append(dt)
            pairs = n
    total = sum(times)
    value = pairs * args.steps / total
    sample = f"every {stride}th of {nw} frequencies x all {L} degrees ({pairs} pairs) per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PREM-like model, receivers, moment tensor)",
        "config": {"workload": WORKLOAD, "pairs_per_event": 615820, "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
            "roofline": {"bound": "tensor", "pipe": "fp64 (CUDA-core FMA rate = FP64 tensor rate on B200)",
                         "kernel": "k_solve_batched" if args.solver == "batched" else "k_solve_plain",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None,
                         "peak_source": "measured: FP64 FMA microbenchmark run by this bench on this GPU",
                         "flops_per_launch": flops, "launch_ms": mean_solve,
                         "traffic": traffic_from_profiles(
                             "k_solve_batched" if args.solver == "batched" else "k_solve_plain")},
            "clocks": clk,
        }
        if world == 1 and not args.no_batch:
            line["batched_vs_plain"] = batch_compare(local)
        if world == 1 and not args.no_grad:
            line["gradient"] = gradient_check(local)
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            n, dt, nw, L = cpu_sample(pf, 1, threads)
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
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
