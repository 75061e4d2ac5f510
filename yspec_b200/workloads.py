"""Synthetic workloads: yspec parameter files for the benchmark configurations.

The reference publishes no benchmark data; these are seeded synthetic
stand-ins with the shapes the configurations name.  Receivers are uniform on
the sphere (lat = asin(2u-1), lon = 360u - 180), moment-tensor entries are
N(0, 1e20) N m, source depths uniform where a range is given.

    c1  plain, small: lmax 150, fmax 10 mHz, 60 min @ 10 s, 10 receivers,
        displacement, full gravity, attenuation off, source at 100 km
    c2  single event at scale: lmax 750, fmax 50 mHz, 120 min @ 1 s,
        100 receivers, acceleration with potential/tilt corrections,
        attenuation on, full gravity, source depth U(0, 700) km
    c3  64 uneven events: fmax U(10, 50) mHz, lmax 15 fmax, depth U(0, 700),
        receivers log-uniform 1..1000, 60 min, dt = 1/(2.2 fmax) rounded
        down to 0.5 s, filter 0.1-0.2 / 0.9-0.98 fmax
    c4  adjoint config: lmax 300, fmax 20 mHz, 60 min @ 5 s, 50 receivers,
        source at 150 km
    c5  16 events: lmax 1500, fmax 100 mHz, 120 min @ 0.5 s, 10000
        receivers, 400-knot model
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent.parent / "tests" / "golden"
MODEL200 = GOLDEN / "model200.deck"
MODEL400 = GOLDEN / "model400.deck"


@dataclass
class Params:
    pref_out: str = "yspec.out"
    model_file: str = str(MODEL200)
    ats: int = 0
    grav: int = 2
    out: int = 0
    cor: int = 0
    lmin: int = 0
    lmax: int = 150
    fmin: float = 0.1
    fmax: float = 10.0
    tout: float = 60.0
    dt: float = 10.0
    f11: float = 0.1
    f12: float = 0.2
    f21: float = 8.0
    f22: float = 9.5
    depth_s: float = 100.0
    lat_s: float = 0.0
    lon_s: float = 0.0
    mm: list = field(default_factory=lambda: [1e20, 0, 0, 0, 0, 0])
    depth_r: float = 0.0
    receivers: list = field(default_factory=lambda: [(0.0, 30.0)])

    def text(self) -> str:
        """The parameter file in the reference's positional layout
        (yspec.f90:88-137; comment-line counts as examples/input.txt)."""
        def q(s: str) -> str:
            # list-directed reads stop at '/', so paths are quoted
            return f"'{s}'" if ("/" in s or " " in s) else s
        L = ["# yspec parameter file", "# (synthetic workload)", "",
             "# prefix for output files", f"  {q(self.pref_out)}", "",
             "# Earth model", f"  {q(self.model_file)}", "",
             "# attenuation switch: 1 = on, 0 = off", f"{self.ats}", "",
             "# gravitation: 0 = none, 1 = cowling, 2 = self", f"{self.grav}", "",
             "# output: 0 = displacement, 1 = velocity, 2 = acceleration", f"{self.out}", "",
             "# potential and tilt corrections: 0 = no, 1 = yes", f"{self.cor}", "",
             "# lmin", f"  {self.lmin}", "", "# lmax", f"  {self.lmax}", "",
             "# fmin (mHz)", f"  {self.fmin!r}", "", "# fmax (mHz)", f"  {self.fmax!r}", "",
             "# length of time series (min)", f"  {self.tout!r}", "",
             "# time step (sec)", f"  {self.dt!r}", "",
             "# f11 filter (mHz)", f"  {self.f11!r}", "", "# f12 filter (mHz)", f"  {self.f12!r}", "",
             "# f21 filter (mHz)", f"  {self.f21!r}", "", "# f22 filter (mHz)", f"  {self.f22!r}", "",
             "# source depth (km)", f"  {self.depth_s!r}", "",
             "# source latitude (deg)", f"  {self.lat_s!r}", "",
             "# source longitude (deg)", f"  {self.lon_s!r}", ""]
        names = ["M_{r,r}", "M_{r,theta}", "M_{r,phi}", "M_{theta,theta}", "M_{theta,phi}", "M_{phi,phi}"]
        for n, v in zip(names, self.mm):
            L += [f"# {n} (Nm)", f"  {float(v)!r}", ""]
        L += ["# receiver depth", f"  {self.depth_r!r}", "",
              "# number of receivers", f"{len(self.receivers)}", "",
              "# receiver latitudes and longitudes"]
        L += [f"  {la!r}  {lo!r}" for la, lo in self.receivers]
        return "\n".join(L) + "\n"

    def write(self, path: str | os.PathLike) -> Path:
        path = Path(path)
        path.write_text(self.text())
        return path


def sphere_points(rng: np.random.Generator, n: int) -> list[tuple[float, float]]:
    u, v = rng.random(n), rng.random(n)
    lat = np.degrees(np.arcsin(2 * u - 1))
    lon = 360 * v - 180
    return [(float(a), float(b)) for a, b in zip(lat, lon)]


def moment_tensor(rng: np.random.Generator) -> list[float]:
    return [float(x) for x in rng.normal(0.0, 1e20, 6)]


def config(name: str, seed: int = 0, **over) -> list[Params]:
    """Parameter sets of a configuration (one per event).  `over` sets
    Params fields; nrec=n keeps each event's first n receivers."""
    rng = np.random.default_rng(seed)
    nrec = over.pop("nrec", None)
    if name == "c1":
        (ls, lo), = sphere_points(rng, 1)
        p = Params(ats=0, grav=2, out=0, cor=0, lmax=150, fmin=0.1, fmax=10.0, tout=60.0, dt=10.0,
                   f11=0.1, f12=0.2, f21=8.0, f22=9.5, depth_s=100.0, lat_s=ls, lon_s=lo,
                   mm=moment_tensor(rng), receivers=sphere_points(rng, 10))
        ps = [p]
    elif name == "c2":
        (ls, lo), = sphere_points(rng, 1)
        p = Params(ats=1, grav=2, out=2, cor=1, lmax=750, fmin=0.1, fmax=50.0, tout=120.0, dt=1.0,
                   f11=0.1, f12=0.2, f21=45.0, f22=49.0, depth_s=float(rng.uniform(0, 700)),
                   lat_s=ls, lon_s=lo, mm=moment_tensor(rng), receivers=sphere_points(rng, 100))
        ps = [p]
    elif name == "c3":
        ps = []
        for _ in range(64):
            fmax = float(rng.uniform(10.0, 50.0))
            nr = int(round(math.exp(rng.uniform(0.0, math.log(1000.0)))))
            dt = math.floor(1.0 / (2.2 * fmax * 1e-3) / 0.5) * 0.5
            (ls, lo), = sphere_points(rng, 1)
            ps.append(Params(ats=1, grav=2, out=0, cor=0, lmax=int(round(15 * fmax)), fmin=0.1,
                             fmax=fmax, tout=60.0, dt=dt, f11=0.1, f12=0.2, f21=0.9 * fmax,
                             f22=0.98 * fmax, depth_s=float(rng.uniform(0, 700)), lat_s=ls, lon_s=lo,
                             mm=moment_tensor(rng), receivers=sphere_points(rng, max(1, nr))))
    elif name == "c4":
        (ls, lo), = sphere_points(rng, 1)
        p = Params(ats=1, grav=2, out=0, cor=0, lmax=300, fmin=0.1, fmax=20.0, tout=60.0, dt=5.0,
                   f11=0.1, f12=0.2, f21=18.0, f22=19.5, depth_s=150.0, lat_s=ls, lon_s=lo,
                   mm=moment_tensor(rng), receivers=sphere_points(rng, 50))
        ps = [p]
    elif name == "c5":
        ps = []
        for _ in range(16):
            (ls, lo), = sphere_points(rng, 1)
            ps.append(Params(model_file=str(MODEL400), ats=1, grav=2, out=0, cor=0, lmax=1500,
                             fmin=0.1, fmax=100.0, tout=120.0, dt=0.5, f11=0.1, f12=0.2, f21=90.0,
                             f22=98.0, depth_s=float(rng.uniform(0, 700)), lat_s=ls, lon_s=lo,
                             mm=moment_tensor(rng), receivers=sphere_points(rng, 10000)))
    else:
        raise ValueError(name)
    for p in ps:
        for k, v in over.items():
            setattr(p, k, v)
        if nrec is not None:
            p.receivers = p.receivers[: int(nrec)]
    return ps
