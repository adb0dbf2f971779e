"""Dipole densities with SphericalHarmonics(Laplace3D) on the device, alone and with charges (τ as
the tuple (charge, Dipole), src/sources.jl:16-31,137-155): the P2M's dipole terms from the
derivative identities (src/operators/harmonics.jl:708-738) and the dipole near field, against FP64
direct sums of q/(4πr) + d·v/(4πr³) and their gradients, on both precision paths, at the sources
and at targets (the reference checks its dipole FMM the same way, test/test_harmonics.jl:129-152)."""
import numpy as np
import pytest

from helpers import clustered3, rel_l2, uniform3

pytestmark = pytest.mark.gpu
KC = 1 / (4 * np.pi)


def direct(src, q, d, tgt, self_idx=None):
    pot = np.zeros(len(tgt))
    grad = np.zeros((len(tgt), 3))
    for a in range(0, len(tgt), 128):
        v = tgt[a:a + 128, None, :] - src[None, :, :]
        r2 = np.einsum("tsk,tsk->ts", v, v)
        if self_idx is not None:
            r2[np.arange(len(r2)), self_idx[a:a + 128]] = np.inf
        ir = 1 / np.sqrt(r2)
        ir3 = ir ** 3
        dv = np.einsum("tsk,sk->ts", v, d)
        pot[a:a + 128] = KC * ((q[None, :] * ir).sum(1) + (dv * ir3).sum(1))
        c = q[None, :] * ir3 + 3 * dv * ir3 * ir * ir
        grad[a:a + 128] = KC * (-np.einsum("ts,tsk->tk", c, v) + np.einsum("ts,sk->tk", ir3, d))
    return pot, grad


@pytest.mark.parametrize("gen", [uniform3, clustered3])
@pytest.mark.parametrize("with_charges", [False, True])
@pytest.mark.parametrize("precision,p,tol", [("fp64", 14, 2e-6), ("mixed", 11, 2e-5)])
def test_dipoles_against_direct(fmmb, gen, with_charges, precision, p, tol):
    rng = np.random.default_rng(11)
    n = 20000
    pts = gen(rng, n)
    d = rng.standard_normal((n, 3))
    q = rng.standard_normal(n) if with_charges else np.zeros(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=p), pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
    assert f.nlevels >= 4
    dens = (q, fmmb.Dipoles(d)) if with_charges else fmmb.Dipoles(d)
    st = fmmb.build_expansions(f, pts, dens, precision=precision)
    u, g = fmmb.evaluate_at_sources_both(f, st)
    sel = np.sort(rng.choice(n, 300, replace=False))
    du, dg = direct(pts, q, d, pts[sel], sel)
    assert rel_l2(u[sel], du) < tol, (gen.__name__, with_charges, precision, rel_l2(u[sel], du))
    assert rel_l2(g[sel], dg) < 10 * tol, (gen.__name__, with_charges, precision, rel_l2(g[sel], dg))
    tg = rng.random((300, 3))
    ut = fmmb.evaluate(f, st, tg)
    gt = fmmb.evaluate(f, st, tg, output=fmmb.Gradient())
    dut, dgt = direct(pts, q, d, tg)
    assert rel_l2(ut, dut) < 3 * tol and rel_l2(gt, dgt) < 30 * tol, (rel_l2(ut, dut), rel_l2(gt, dgt))


def test_dipoles_charges_only_state_back(fmmb, oracle):
    """A state rebuilt with charges alone drops the dipoles (and matches the charge-only path)."""
    rng = np.random.default_rng(12)
    n = 8000
    pts = uniform3(rng, n)
    q = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=8), pts, ppl=64)
    st = fmmb.FMMState(f, "fp64")
    fmmb.build_expansions_(st, f, pts, fmmb.Dipoles(rng.standard_normal((n, 3))))
    fmmb.build_expansions_(st, f, pts, q)
    u = fmmb.evaluate_at_sources(f, st)
    u0 = fmmb.evaluate_at_sources(f, fmmb.build_expansions(f, pts, q))
    assert np.array_equal(u, u0)
    # charges given as the tuple with zero moments equal the charge path to rounding
    u2 = fmmb.evaluate_at_sources(f, fmmb.build_expansions(f, pts, (q, fmmb.Dipoles(np.zeros((n, 3))))))
    assert rel_l2(u2, u0) < 1e-13


def test_dipole_errors(fmmb):
    rng = np.random.default_rng(13)
    pts = uniform3(rng, 3000)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=6), pts, ppl=64)
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.build_expansions(f, pts, fmmb.Dipoles(np.zeros((2999, 3))))
    fy = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Yukawa3D(2.0), p=6), pts, ppl=64)
    with pytest.raises(fmmb.Unsupported):
        fmmb.build_expansions(fy, pts, fmmb.Dipoles(np.zeros((3000, 3))))
