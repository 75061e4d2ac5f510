"""Time the device stages of a synthetic workload configuration.

    python -m yspec_b200.stages c2 [--solver batched|plain] [--schedule 0|1|2] [--reps 3]
                                   [--seed 0] [--set lmax=300 --set fmax=20.0] [--batch]
    python -m yspec_b200.stages c5 --batch --reuse-output --schedule 2 --reps 2
    python -m yspec_b200.stages c4 --gradient --reps 2

Runs the configuration's first event through `Engine.run` (or, with
--batch, all its events through one `Engine.batch_run`) `reps` times and
prints, per run, the device time of each stage (Legendre table, solves,
l-sum, filter + inverse FFT) measured with CUDA events on the engine's
stream, the number of (omega,l) solves and the counted FP64 work of the
solve stage.  A batch of several events runs each event's l-sum and time
series back to back, so its "lsum" time covers both and "ifft" is zero.
With --gradient it runs the reverse mode instead
(Engine.gradient of a seeded random trace adjoint) and prints its stages
(Legendre table, reverse sweeps, l-sum transpose, time-stage transpose).
It is also the small, self-contained command used for ncu captures of one
kernel.
"""
from __future__ import annotations

import argparse
import tempfile
import time
from pathlib import Path

import numpy as np

from . import Engine, Event, Model, Params, workloads as W


def _parse_set(items: list[str]) -> dict:
    out = {}
    for kv in items:
        k, v = kv.split("=", 1)
        out[k] = int(v) if k == "nrec" else type(getattr(W.Params(), k))(v)
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("config", help="c1 .. c5")
    ap.add_argument("--solver", default="batched", choices=["batched", "plain"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--event", type=int, default=0, help="event index within the configuration")
    ap.add_argument("--schedule", type=int, default=-1,
                    help="batched-solver schedule: 0 tiles, 1 pair lists, 2 split pair lists, -1 autotuned")
    ap.add_argument("--batch", action="store_true", help="run every event of the configuration as one batch")
    ap.add_argument("--reuse-output", action="store_true",
                    help="with --batch: one host trace buffer for every event (c5's traces exceed host memory)")
    ap.add_argument("--gradient", action="store_true",
                    help="time the reverse-mode gradient of the event (Engine.gradient) instead")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="override a parameter of the configuration")
    a = ap.parse_args(argv)
    ps = W.config(a.config, seed=a.seed, **_parse_set(a.set))
    if not a.batch:
        ps = [ps[a.event]]
    eng = Engine(0, solver=a.solver)
    eng.set_schedule(a.schedule)
    with tempfile.TemporaryDirectory() as tmp:
        m = Model(ps[0].model_file)
        eng.upload(m)
        evs = [Event(m, Params(p.write(Path(tmp) / f"{a.config}_{i}.in"))) for i, p in enumerate(ps)]
        if a.gradient:
            ev = evs[0]
            gout = np.random.default_rng(a.seed).standard_normal((ev.nr, 4, ev.nout()))
            gout[:, 0, :] = 0.0
            for rep in range(a.reps):
                t = time.perf_counter()
                gval, _ = eng.gradient(ev, gout)
                wall = time.perf_counter() - t
                ms = eng.timings()
                print(f"{a.config} gradient rep{rep}: wall {wall:.3f} s  stages (ms) legendre {ms[0]:.3f} "
                      f"sweeps {ms[1]:.3f} lsum-T {ms[2]:.3f} time-T {ms[3]:.3f}  pairs {ev.L * ev.nw}  "
                      f"|dL/dval|_1 {float(np.abs(gval).sum()):.6e}", flush=True)
            return
        outs = None
        if a.batch and a.reuse_output:
            if any((e.nr, e.nout()) != (evs[0].nr, evs[0].nout()) for e in evs):
                raise SystemExit("--reuse-output needs events of one trace shape")
            shared = np.ones((evs[0].nr, 4, evs[0].nout()))      # pages touched before timing
            outs = [shared] * len(evs)
        for rep in range(a.reps):
            t = time.perf_counter()
            if a.batch:
                eng.batch_run(evs, outs=outs)
            else:
                eng.run(evs[0])
            wall = time.perf_counter() - t
            ms = eng.timings()
            pairs, fl = eng.work()
            sched = eng.last_schedule()[0] if a.solver == "batched" else "-"
            print(f"{a.config} {a.solver} sched {sched} rep{rep}: wall {wall:.3f} s  stages (ms) "
                  f"legendre {ms[0]:.3f} solve {ms[1]:.3f} lsum {ms[2]:.3f} ifft {ms[3]:.3f}  "
                  f"pairs {pairs:.0f}  solves/s {pairs / (ms[1] / 1e3):.4g}  "
                  f"solve FP64 {fl / (ms[1] / 1e3) / 1e12:.3f} TFLOP/s", flush=True)


if __name__ == "__main__":
    main()
