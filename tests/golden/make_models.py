"""Generate the synthetic earth-model decks used by the tests and the benchmark,
and copy the reference's own example inputs beside them.

    python tests/golden/make_models.py <reference examples directory>

The decks are resamplings of the PREM decks bundled with the reference
(examples/prem.200.isotropic, prem.200, prem.200.fic).  Each layer between
repeated-radius discontinuities keeps its end radii; its knot count is the
reference count scaled to the target total (at least 2); the knots are
spaced uniformly in radius and every column is evaluated with a natural
cubic spline through the reference knots of that layer.  Written in the
9-column deck format (anisotropy flag 1; an isotropic source gets
Vph = Vpv, Vsh = Vsv, eta = 1).

Outputs (committed; the generator only runs where the reference is mounted):
    model200.deck        200 knots, no ocean, solid inner core  (configs 1-4)
    model400.deck        400 knots, same structure               (config 5)
    model200_ocean.deck  200 knots, transversely isotropic, 3 km ocean
    model200_fic.deck    200 knots, fluid inner core, ocean
    examples/            the reference's examples/input.txt and its five
                         prem.200* decks, copied byte for byte (the only
                         fixtures the reference ships)
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import numpy as np
from scipy.interpolate import CubicSpline

HERE = Path(__file__).resolve().parent


EXAMPLES = ["input.txt", "prem.200", "prem.200.no", "prem.200.fic", "prem.200.isotropic",
            "prem.200.noiso"]


def read_deck(path: Path):
    lines = path.read_text().splitlines()
    title = lines[0].strip()
    ians = int(lines[1].split()[0])
    tref = float(lines[1].split()[1])
    n = int(lines[2].split()[0])
    rows = np.array([[float(x) for x in l.split()] for l in lines[3:3 + n]])
    if ians != 1:   # isotropic: append Vph = Vpv, Vsh = Vsv, eta = 1
        rows = np.column_stack([rows, rows[:, 2], rows[:, 3], np.ones(n)])
    return title, tref, rows


def layers(r: np.ndarray):
    cuts = [0] + [i for i in range(1, r.size) if r[i] == r[i - 1]] + [r.size]
    return list(zip(cuts[:-1], cuts[1:]))


def resample(rows: np.ndarray, total: int) -> tuple[np.ndarray, list[int]]:
    lay = layers(rows[:, 0])
    counts = np.array([b - a for a, b in lay], float)
    want = np.maximum(2, np.round(counts * total / counts.sum())).astype(int)
    order = np.argsort(-counts)
    k = 0
    while want.sum() != total:           # adjust the thickest layers
        i = order[k % len(order)]
        if want.sum() > total and want[i] > 2:
            want[i] -= 1
        elif want.sum() < total:
            want[i] += 1
        k += 1
    out = []
    for (a, b), m in zip(lay, want):
        r0, r1 = rows[a, 0], rows[b - 1, 0]
        rn = np.linspace(r0, r1, m)
        block = np.empty((m, rows.shape[1]))
        block[:, 0] = rn
        for c in range(1, rows.shape[1]):
            if b - a >= 3:
                block[:, c] = CubicSpline(rows[a:b, 0], rows[a:b, c], bc_type="natural")(rn)
            else:
                block[:, c] = np.interp(rn, rows[a:b, 0], rows[a:b, c])
        out.append(block)
    return np.vstack(out), list(want)


def write_deck(path: Path, title: str, tref: float, rows: np.ndarray, counts: list[int]):
    nic = counts[0]
    noc = counts[0] + counts[1]
    with path.open("w") as f:
        f.write(f" {title}\n 1 {tref:.1f} 1\n {rows.shape[0]} {nic} {noc}\n")
        for row in rows:
            f.write(f"{row[0]:11.2f}{row[1]:10.3f}{row[2]:10.3f}{row[3]:10.3f}{row[4]:10.1f}"
                    f"{row[5]:9.1f}{row[6]:10.3f}{row[7]:10.3f}{row[8]:9.5f}\n")


def main(argv: list[str]) -> int:
    if len(argv) != 2:
        print(__doc__)
        return 2
    ex = Path(argv[1])
    jobs = [("prem.200.isotropic", "model200.deck", 200, "synthetic200"),
            ("prem.200.isotropic", "model400.deck", 400, "synthetic400"),
            ("prem.200", "model200_ocean.deck", 200, "synthetic200_ocean"),
            ("prem.200.fic", "model200_fic.deck", 200, "synthetic200_fic")]
    for src, dst, n, title in jobs:
        _, tref, rows = read_deck(ex / src)
        new, counts = resample(rows, n)
        write_deck(HERE / dst, title, tref, new, counts)
        print(f"{dst}: {new.shape[0]} knots, layers {counts}")
    (HERE / "examples").mkdir(exist_ok=True)
    for name in EXAMPLES:
        shutil.copyfile(ex / name, HERE / "examples" / name)
        print(f"examples/{name}: copied")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
