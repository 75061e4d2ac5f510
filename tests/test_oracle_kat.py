"""Known-answer tests of the CPU oracle (the restatement the GPU is checked against).

The reference ships no tests or golden outputs, so the oracle is pinned here
by independent mathematics: natural cubic splines, Legendre functions,
spherical-Bessel logarithmic derivatives, the frequency grid, the gravity
integral, linearity of the whole path in the moment tensor, and the
radix-2 transform with the reference's single-precision pi.
"""
import numpy as np
import pytest
from scipy import special
from scipy.interpolate import CubicSpline

import yo
from yspec_b200 import workloads as W

PI_D = float(np.float32(np.pi))
FOURPI_D = 12.56637061


def test_frequency_grid_table():
    # nt, i2, nw of the benchmark configurations (module_fourier.f90:362-397)
    tn = 1.0 / (6.371e6 * np.sqrt(PI_D * 6.6723e-11 * 5.515e3) / 6.371e6)
    cases = {  # fmin, fmax (mHz), length (min), dt (s): nt, i2, nw
        "c1": (0.1, 10.0, 60.0, 10.0, 512, 53, 52),
        "c2": (0.1, 50.0, 120.0, 1.0, 16384, 821, 820),
        "c4": (0.1, 20.0, 60.0, 5.0, 1024, 104, 103),
        "c5": (0.1, 100.0, 120.0, 0.5, 32768, 1640, 1639),
        "example": (0.2, 40.0, 60.0, 1.0, 8192, 329, 328),
    }
    for name, (f1, f2, tout, dt, nt, i2, nw) in cases.items():
        rc, nt_, i1_, i2_, df, ep = yo.fcal(f1 * tn / 1000, f2 * tn / 1000, dt / tn, tout * 60 / tn)
        assert rc == 0
        assert (nt_, i2_, i2_ - i1_ + 1) == (nt, i2, nw), name


def test_fcal_nyquist_stop():
    rc, *_ = yo.fcal(0.001, 10.0, 1.0, 100.0)      # 1/(2 dt) = 0.5 < f2
    assert rc == 5


def test_natural_spline_matches_scipy():
    rng = np.random.default_rng(1)
    x = np.sort(rng.uniform(0, 1, 30))
    y = np.sin(5 * x) + x ** 2
    y2 = yo.spline(x, y)
    ref = CubicSpline(x, y, bc_type="natural")
    np.testing.assert_allclose(y2, ref(x, 2), rtol=1e-11, atol=1e-11)
    for k in (1, 7, 29):
        xv = 0.5 * (x[k - 1] + x[k])
        assert abs(yo.splint(x, y, y2, xv, k) - ref(xv)) < 1e-12
    lin = 3 * x - 2
    assert np.allclose(yo.spline(x, lin), 0.0, atol=1e-9)   # rounding of slope differences


@pytest.mark.parametrize("l", [2, 3, 17, 120, 600])
def test_legendre_against_scipy(l):
    theta = np.array([0.3, 1.1, 2.5])
    for th in theta:
        x, xp, xc = yo.legendre(th, l, 2)
        norm = np.sqrt((2 * l + 1) / FOURPI_D)
        # X_l0 (exact FP64 path of the recursion)
        assert abs(x[0] - norm * special.eval_legendre(l, np.cos(th))) <= 1e-9 * norm
        # |X_lm| for m = 1, 2 (single-precision sqrt factors in the reference)
        for m in (1, 2):
            fac = np.sqrt(special.factorial(l - m, exact=False) / special.factorial(l + m, exact=False)) \
                if l < 150 else np.exp(0.5 * (special.gammaln(l - m + 1) - special.gammaln(l + m + 1)))
            want = norm * fac * abs(special.lpmv(m, l, np.cos(th)))
            assert abs(abs(x[m]) - want) <= 1e-6 * norm, (m, x[m], want)
            assert abs(xc[m] - x[m] / np.sin(th)) <= 1e-12 * abs(x[m] / np.sin(th)) + 1e-300


def test_legendre_normalisation_sum():
    # sum over all m of X_lm^2 is (2l+1)/(4 pi) (the reference's own check,
    # module_function.f90:62-64,112,123); complete for l <= 2
    for l in (0, 1, 2):
        for th in (0.2, 1.3, 2.9):
            x, _, _ = yo.legendre(th, l, min(l, 2))
            s = x[0] ** 2 + 2 * np.sum(x[1:] ** 2)
            assert abs(s - (2 * l + 1) / FOURPI_D) < 1e-6


@pytest.mark.parametrize("l", [0, 1, 5, 30])
def test_bessel_log_derivative(l):
    # continued fraction (Re x^2 > 0) against x j_l'(x)/j_l(x)
    for x in (0.3, 2.0, 7.5):
        fp = yo.bfs(l, complex(x * x, 0.0))
        want = x * special.spherical_jn(l, x, derivative=True) / special.spherical_jn(l, x)
        assert abs(fp - want) < 1e-7 * max(1.0, abs(want))
    # series (Re x^2 <= 0): j_l(i y) ~ i_l(y), the same ratio in y
    for y in (0.3, 2.0, 6.0):
        fp = yo.bfs(l, complex(-y * y, 0.0))
        want = y * special.spherical_in(l, y, derivative=True) / special.spherical_in(l, y)
        assert abs(fp - want) < 1e-7 * max(1.0, abs(want))


def test_delaz_equator():
    d = np.zeros(1); ae = np.zeros(1); ast = np.zeros(1)
    yo.lib().yo_delaz(0.0, 30.0, 0.0, 0.0, yo._p(d), yo._p(ae), yo._p(ast))
    assert abs(d[0] - 30 * 0.0174533) < 1e-12
    assert abs(ae[0] - 1.5 * PI_D) < 1e-6 or abs(ae[0] - 0.5 * PI_D) < 1e-6


def _problem(tmp_path, **over):
    base = dict(lmax=12, fmax=4.0, f21=3.0, f22=3.8, dt=30.0, tout=30.0, ats=1)
    base.update(over)
    p = W.config("c1", seed=11, **base)[0]
    p.receivers = p.receivers[:2]
    return p


def test_model_arrays_independent(tmp_path):
    p = _problem(tmp_path)
    pf = p.write(tmp_path / "m.in")
    P = yo.Problem(pf)
    raw = np.loadtxt(W.MODEL200, skiprows=3)
    norms = P.norms
    r = raw[:, 0] / norms.r_norm
    rho = raw[:, 1] / norms.rho_norm
    vp, vs = raw[:, 2] / norms.vel_norm, raw[:, 3] / norms.vel_norm
    np.testing.assert_allclose(P.array("r"), r, rtol=0, atol=0)
    np.testing.assert_allclose(P.array("kappa"), rho * (vp ** 2 - 4.0 / 3.0 * vs ** 2), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(P.array("mu"), rho * vs ** 2, rtol=1e-13, atol=1e-15)
    # gravity: 4/r^2 * integral of the natural spline of r^2 rho per layer (exact for Gauss-Legendre 5)
    cuts = [0] + [i for i in range(1, r.size) if r[i] == r[i - 1]] + [r.size]
    fint, g = 0.0, np.zeros_like(r)
    for a, b in zip(cuts[:-1], cuts[1:]):
        if b - a >= 2:
            cs = CubicSpline(r[a:b], r[a:b] ** 2 * rho[a:b], bc_type="natural")
            for i in range(a, b - 1):
                fint += cs.integrate(r[i], r[i + 1])
                g[i + 1] = fint
        if b < r.size:
            g[b] = fint
    g[1:] = 4 * g[1:] / r[1:] ** 2
    np.testing.assert_allclose(P.array("grav"), g, rtol=1e-10, atol=1e-14)


def test_lsum_matches_coefficients(tmp_path):
    # the oracle's spectra equal an independent numpy l-sum of its own
    # per-(omega,l) coefficients and Legendre table (yspec.f90:291-419)
    p = _problem(tmp_path)
    pf = p.write(tmp_path / "s.in")
    P = yo.Problem(pf)
    ur, ut, up = P.spectra(nthreads=2)
    xa, xpa, xca = P.legendre_table()
    _, _, azst = P.geometry()
    nw, nr, lmax = P.nw, P.nr, P.params.lmax
    coef = np.array([[P.coef(l, j) for j in range(1, nw + 1)] for l in range(0, lmax + 1)])
    e = np.exp(1j * azst)
    UR = np.zeros((nr, nw), complex); UT = np.zeros_like(UR); UP = np.zeros_like(UR)
    for l in range(lmax + 1):
        for m in range(-2, 3):
            a = abs(m); s = (-1.0) ** m if m < 0 else 1.0
            x, xp, xc = s * xa[:, a, l], s * xpa[:, a, l], s * xca[:, a, l]
            uu, vv, ww = coef[l, :, m + 2], coef[l, :, 5 + m + 2], coef[l, :, 10 + m + 2]
            ph = e ** m
            if l == 0:
                if m == 0:
                    UR += np.outer(x, uu)
                continue
            UR += np.outer(x * ph, uu)
            UT += np.outer(xp * ph, vv) + np.outer(1j * m * x * ph, ww)
            UP += np.outer(1j * m * xc * ph, vv) - np.outer(xp * ph, ww)
    for a, b in ((UR, ur), (UT, ut), (UP, up)):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())


def test_linear_in_moment_tensor(tmp_path):
    ma = [1e20, 2e19, -3e19, 5e19, 0.0, -4e19]
    mb = [-2e19, 0.0, 6e19, 1e19, 3e19, 2e19]
    outs = []
    for mm in (ma, mb, list(np.add(ma, mb))):
        p = _problem(tmp_path, mm=mm)
        outs.append(yo.Problem(p.write(tmp_path / "l.in")).run(nthreads=2))
    np.testing.assert_allclose(outs[0][:, 1:] + outs[1][:, 1:], outs[2][:, 1:], rtol=1e-10,
                               atol=1e-10 * np.abs(outs[2][:, 1:]).max())


def _network(row, pi):
    """Radix-2 decimation-in-time with twiddles exp(i m pi / mmax) (fourrow_dp, isign = +1)."""
    n = row.size
    p = int(np.log2(n))
    idx = np.array([int(format(i, f"0{p}b")[::-1], 2) for i in range(n)])
    d = row[idx].astype(complex)
    mmax = 1
    while mmax < n:
        for m in range(mmax):
            w = np.exp(1j * m * pi / mmax)
            t = w * d[m + mmax::2 * mmax].copy()
            d[m + mmax::2 * mmax] = d[m::2 * mmax] - t
            d[m::2 * mmax] = d[m::2 * mmax] + t
        mmax *= 2
    return d


def test_fft_network_single_precision_pi():
    # with exact pi the network is the DFT; with the reference's pi_f it
    # departs from it at ~1e-7, so the traces must reproduce the network
    rng = np.random.default_rng(3)
    row = rng.normal(size=64) + 1j * rng.normal(size=64)
    exact = np.fft.ifft(row) * 64
    assert np.max(np.abs(_network(row, np.pi) - exact)) < 1e-12 * np.abs(exact).max()
    diff = np.max(np.abs(_network(row, PI_D) - exact)) / np.abs(exact).max()
    assert 1e-10 < diff < 1e-5


def test_traces_match_independent_ifft(tmp_path):
    # the oracle's ifft + post-processing (module_fourier.f90:55-145,
    # yspec.f90:432-486) against a numpy restatement on random spectra
    p = _problem(tmp_path, out=2)
    P = yo.Problem(p.write(tmp_path / "f.in"))
    g, n = P.grid, P.norms
    rng = np.random.default_rng(4)
    nr, nw, nt = P.nr, P.nw, g.nt
    spec = [rng.normal(size=(nr, nw)) + 1j * rng.normal(size=(nr, nw)) for _ in range(3)]
    got = P.traces(*spec)
    nout = got.shape[2]
    _, azep, _ = P.geometry()
    w = np.arange(nt // 2 + 1) * g.df
    filt = np.zeros_like(w)
    for i, wi in enumerate(w):
        if wi < g.f11: f = 0.0
        elif wi < g.f12: f = 0.5 * (1 - np.cos(PI_D * (wi - g.f11) / (g.f12 - g.f11)))
        elif wi < g.f21: f = 1.0
        elif wi < g.f22: f = 0.5 * (1 - np.cos(PI_D * (g.f22 - wi) / (g.f22 - g.f21)))
        else: f = 0.0
        filt[i] = f
    t = np.arange(nt) * g.dt
    for k in range(nr):
        comp = []
        for c in range(3):
            d = np.zeros(nt, complex)
            d[g.i1 - 1:g.i2] = spec[c][k]
            d[: nt // 2 + 1] *= filt
            d[nt // 2 + 1:] = np.conj(d[1: nt // 2][::-1])
            d = _network(d, PI_D) / (g.dt * nt) * np.exp(g.ep * t) * n.acl_norm
            comp.append(d.real[:nout])
        N_ = -comp[1] * np.cos(azep[k]) + comp[2] * np.sin(azep[k])
        E_ = comp[1] * np.sin(azep[k]) + comp[2] * np.cos(azep[k])
        for c, want in ((1, comp[0]), (2, N_), (3, E_)):
            np.testing.assert_allclose(got[k, c], want, rtol=1e-11, atol=1e-11 * np.abs(want).max())


def test_shard_and_pair_list_equal_full_runs(tmp_path):
    # the sampled forms the size tests compare against are the same solves
    p = W.config("c1", seed=3, lmax=30, fmax=6.0, f21=4.5, f22=5.5, dt=20.0, tout=40.0)[0]
    p.receivers = p.receivers[:3]
    P = yo.Problem(p.write(tmp_path / "s.in"))
    nw = P.nw
    full = P.spectra(nthreads=4)
    count = len(range(2, nw, 3))
    for a, b in zip(full, P.spectra_shard(2, 3, count, nthreads=3)):
        np.testing.assert_array_equal(a[:, 2::3], b)
    ls = np.array([0, 1, 2, 30, 17])
    js = np.array([1, 2, nw, 5, 9])
    got = P.coef_list(ls, js, nthreads=3)
    for k in range(ls.size):
        np.testing.assert_array_equal(got[k], P.coef(int(ls[k]), int(js[k])))
    with pytest.raises(ValueError):
        P.coef_list([3], [nw + 1])
