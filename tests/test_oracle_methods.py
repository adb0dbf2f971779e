"""Pins the oracle's Yukawa3D and Stokeslet3D harmonic methods to the reference's own tests
(CPU only): test/test_harmonics_yukawa.jl (the radial factors against the modified spherical
Bessel functions at rtol 1e-12, the generating identity at p = 30, the sphere rule, the Laplace
limit, the FMM end to end against direct sums) and test/test_harmonics_stokes.jl (the FMM end to
end against direct Stokeslet sums at p = 16: 1e-5, pressure 1e-4), plus the Stokes blocks as
Laplace expansions (harmonics_stokes.jl's decomposition)."""
import numpy as np
import pytest
from scipy import special

from helpers import DISTRIBUTIONS3, mrd, stokes_direct_all, yukawa_direct


def _u_series(n, z):
    """u_n(z) = (2n+1)!! i_n(z)/z^n = Σ_k (z²/2)^k / (k! Π_{j=1..k} (2n+2j+1)): positive terms only"""
    s, t, k = 0.0, 1.0, 0
    while True:
        s += t
        k += 1
        t *= (z * z / 2) / (k * (2 * n + 2 * k + 1))
        if t < 1e-18 * s:
            return s + t


def _v_closed(n, z):
    """v_n(z) = (2/π) z^{n+1} k_n(z) / (2n−1)!! from the finite sum of k_n:
    e^{−z} Σ_{k≤n} (n+k)!/(k!(n−k)!) z^{n−k} 2^{−k} / (2n−1)!!, positive terms only"""
    from math import factorial
    df = float(np.prod(np.arange(1, 2 * n, 2, dtype=float))) if n > 0 else 1.0
    s = sum(factorial(n + k) / (factorial(k) * factorial(n - k)) * z ** (n - k) * 2.0 ** (-k) for k in range(n + 1))
    return np.exp(-z) * s / df


def test_yukawa_radial_factors(oracle):
    """test/test_harmonics_yukawa.jl:14-26 (the modified spherical Bessel functions as their
    positive series, in place of SpecialFunctions)"""
    for z in (1e-6, 0.03, 0.7, 2.5, 9.0, 40.0):
        u, v = oracle.yukawa_radial(z, 20)
        for n in range(21):
            assert u[n] == pytest.approx(_u_series(n, z), rel=1e-12)
            assert v[n] == pytest.approx(_v_closed(n, z), rel=1e-12)
    # against scipy's Bessel functions where they are accurate
    z = 2.5
    u, v = oracle.yukawa_radial(z, 10)
    for n in range(11):
        i_n = np.sqrt(np.pi / (2 * z)) * special.iv(n + 0.5, z)
        k_n = np.sqrt(np.pi / (2 * z)) * special.kv(n + 0.5, z)
        assert u[n] == pytest.approx(float(np.prod(np.arange(1, 2 * n + 2, 2, dtype=float))) * i_n / z ** n, rel=1e-10)
        assert v[n] == pytest.approx((2 / np.pi) * z ** (n + 1) * k_n / (float(np.prod(np.arange(1, 2 * n, 2, dtype=float))) if n else 1.0), rel=1e-10)


def test_yukawa_generating_identity(oracle):
    """test/test_harmonics_yukawa.jl:39-56: Σ over the real bases equals e^{−κ|x−y|}/|x−y|."""
    kappa, p = 2.0, 30
    x, y = np.array([0.6, -0.5, 0.8]), np.array([0.1, 0.2, -0.05])
    br, bi = oracle.yukawa_bases(y, x, kappa, p)
    s = 0.0
    for n in range(p + 1):
        s += br[n * n] * bi[n * n]
        for m in range(1, n + 1):
            s += (br[n * n + 2 * m - 1] * bi[n * n + 2 * m - 1] - br[n * n + 2 * m] * bi[n * n + 2 * m]) / 2
    r = np.linalg.norm(x - y)
    assert s == pytest.approx(np.exp(-kappa * r) / r, rel=1e-12)


def test_sphere_rule(oracle):
    t, w = oracle.gauss_legendre(2 * 8 + 10)
    assert np.all(np.diff(t) > 0) and np.sum(w) == pytest.approx(2.0, rel=1e-14)
    # exact for polynomials of degree 2n − 1
    assert np.sum(w * t ** 50) == pytest.approx(2 / 51, rel=1e-13)


def test_yukawa_laplace_limit(oracle):
    """A tiny κ reproduces the Laplace3D FMM (test/test_harmonics_yukawa.jl:87-95)."""
    rng = np.random.default_rng(3)
    pts = rng.random((6000, 3))
    tau = rng.standard_normal(6000)
    out = []
    for kernel in ("yukawa", "laplace"):
        O = oracle.FMM(8, pts, 64, kernel=kernel, kappa=1e-10)
        O.build_expansions(pts, tau)
        out.append(O.evaluate_at_sources())
    assert mrd(out[0][0], out[1][0]) < 1e-9 and mrd(out[0][1], out[1][1]) < 1e-9


@pytest.mark.parametrize("name", ["uniform", "helix", "mixed"])
def test_yukawa_fmm_against_direct(oracle, name):
    """test/test_harmonics_yukawa.jl:104-121: κ = 4, p = 16, ppl = 40, 5000 points."""
    rng = np.random.default_rng(52)
    kappa, n = 4.0, 5000
    pts = DISTRIBUTIONS3[name](rng, n)
    tau = rng.standard_normal(n)
    tg = rng.random((400, 3))
    O = oracle.FMM(16, pts, 40, kernel="yukawa", kappa=kappa)
    O.build_expansions(pts, tau)
    u, _ = O.evaluate_at_sources()
    assert mrd(u, yukawa_direct(pts, tau, pts, kappa, self_excluded=True)) < 1e-5
    ut, gt = O.evaluate(tg)
    dp, dg = yukawa_direct(pts, tau, tg, kappa, gradient=True)
    assert mrd(ut, dp) < 1e-5 and mrd(gt, dg) < 1e-4


@pytest.mark.parametrize("name", ["uniform", "helix", "mixed"])
def test_stokes_fmm_against_direct(oracle, name):
    """test/test_harmonics_stokes.jl:46-60: Stokeslets, p = 16, ppl = 40, 5000 points: velocity
    at the sources and at targets within 1e-5, pressure at targets within 1e-4."""
    rng = np.random.default_rng(34)
    n = 5000
    pts = DISTRIBUTIONS3[name](rng, n)
    tg = rng.random((400, 3))
    f = rng.standard_normal((n, 3))
    O = oracle.FMM(16, pts, 40, kernel="stokes")
    O.build_expansions(pts, f)
    v, _ = O.evaluate_at_sources_stokes()
    assert mrd(v, stokes_direct_all(pts, np.arange(n), f=f)) < 1e-5
    vt, pt = O.evaluate_stokes(tg)
    assert mrd(vt, stokes_direct_all(pts, None, f=f, tgt=tg)) < 1e-5
    assert mrd(pt, stokes_direct_all(pts, None, f=f, tgt=tg, output="pressure")) < 1e-4


def test_stokes_blocks_are_laplace_expansions(oracle):
    """Φ_k are the Laplace expansions of the charges f_k, and Ψ̂ = (E[y·f] − c·E[f]) / w
    (harmonics_stokes.jl:14-21), at every node."""
    rng = np.random.default_rng(7)
    n, p = 8000, 8
    pts = rng.random((n, 3))
    f = rng.standard_normal((n, 3))
    O = oracle.FMM(p, pts, 40, kernel="stokes")
    O.build_expansions(pts, f)
    SM, SL = O.expansions()
    N = (p + 1) ** 2
    E = []
    for q in [f[:, 0], f[:, 1], f[:, 2], np.einsum("ij,ij->i", pts, f)]:
        Lp = oracle.FMM(p, pts, 40)
        Lp.build_expansions(pts, q)
        E.append(Lp.expansions())
    T = O.tree
    for k in range(3):
        for i in range(2):
            ref = E[k][i]
            got = (SM, SL)[i][:, k * N:(k + 1) * N]
            assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))
    wl = 1.0 / 2.0 ** T.level
    cen = (T.cell + 0.5) * wl[:, None]
    for i, sel in ((0, np.ones(T.n, bool)), (1, T.leaf.astype(bool))):
        ref = (E[3][i] - sum(cen[:, k:k + 1] * E[k][i] for k in range(3))) / wl[:, None]
        got = (SM, SL)[i][:, 3 * N:]
        assert np.max(np.abs(got[sel] - ref[sel])) < 1e-12 * np.max(np.abs(ref[sel]))
