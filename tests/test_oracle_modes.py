"""The oracle's ODE core against published normal-mode eigenfrequencies.

The response of the two-point solvers (oracle/yo_solver.c through
yo_green) to a source near the surface has poles at the eigenfrequencies of
the earth model.  On the reference's own PREM deck (tests/golden/examples/
prem.200: ocean, transverse isotropy, attenuation with physical dispersion
at the deck's reference period), scanned along the real frequency axis with
a small damping, the response of each solver must peak at the PREM
eigenfrequencies of Dziewonski & Anderson (1981, Phys. Earth Planet.
Inter. 25:297-356), quoted here to four digits:

    0S0 814.7, 0S2 309.3, 1S2 679.9, 0S3 468.6, 0S4 647.1 microhertz
    (spheroidal: the self-gravitating minor and b-vector systems, and the
    l = 0 radial solver with gravity),
    0T2 379.2, 0T3 586.2 microhertz (toroidal).

The peaks of the oracle are within 0.05% of these (within 0.01% for all
but 0S0).  This checks the gravitating equations, start values and
boundary conditions of the oracle against physics it was not transcribed
from; the device solvers are checked against the oracle elsewhere."""
from __future__ import annotations

import numpy as np
import pytest

import yo
from yspec_b200 import workloads as W

# (name, solver kind of yo_green, l, PREM eigenfrequency in mHz)
MODES = [
    ("0S0", 2, 0, 0.8147),
    ("0S2", 3, 2, 0.3093),
    ("1S2", 3, 2, 0.6799),
    ("0S3", 3, 3, 0.4686),
    ("0S4", 3, 4, 0.6471),
    ("0T2", 0, 2, 0.3792),
    ("0T3", 0, 3, 0.5862),
]


@pytest.fixture(scope="module")
def prem(tmp_path_factory):
    d = tmp_path_factory.mktemp("modes")
    deck = W.GOLDEN / "examples" / "prem.200"
    # receiver at 3 km depth (below the sea floor), source at 30 km
    p = W.config("c1", seed=0, model_file=str(deck), depth_r=3.0, depth_s=30.0, ats=1)[0]
    P = yo.Problem(p.write(d / "modes.in"))
    assert P.setup_rc == 0
    return P


def _response(P, kind, l, f_mhz, rr=0.998, rs=0.99, damp=2e-4):
    """|G| at the real frequency f_mhz with a relative damping damp."""
    w = 2.0 * np.pi * f_mhz * 1e-3 * P.norms.t_norm * (1.0 - 1j * damp)
    return np.linalg.norm(P.green(kind, l, w, rr, rs, 1))


def _peak(P, kind, l, f0, span=0.03, n=61):
    """Frequency of the largest response within f0 (1 +- span): the grid
    maximum refined by a parabola through log |G| at it and its neighbours,
    and its height over the median of the scan."""
    fs = np.linspace(f0 * (1.0 - span), f0 * (1.0 + span), n)
    a = np.array([_response(P, kind, l, f) for f in fs])
    i = int(np.argmax(a))
    assert 0 < i < n - 1, "maximum at the edge of the scan"
    y0, y1, y2 = np.log(a[i - 1:i + 2])
    shift = 0.5 * (y0 - y2) / (y0 - 2.0 * y1 + y2)
    return fs[i] + shift * (fs[1] - fs[0]), a[i] / np.median(a)


@pytest.mark.parametrize("name,kind,l,f0", MODES, ids=[m[0] for m in MODES])
def test_response_peaks_at_prem_eigenfrequency(prem, name, kind, l, f0):
    f, contrast = _peak(prem, kind, l, f0)
    assert contrast > 5.0, (name, contrast)            # a resonance, not a slope
    assert abs(f - f0) / f0 < 1e-3, (name, f, f0)
