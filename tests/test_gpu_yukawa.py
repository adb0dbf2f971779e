"""SphericalHarmonics(Yukawa3D(κ); p) on the device (FP64 path), as the reference's Yukawa
tests check it (test/test_harmonics_yukawa.jl): the FMM end to end against FP64 direct sums of
e^{−κr}/(4πr) (κ = 4, p = 16, ppl = 40, N = 5000 in the unit box: potential at the sources and
at targets within 1e-5, gradient at targets within 1e-4, max-norm relative), and the Laplace
limit (a tiny κ reproduces the Laplace3D FMM, whose path is pinned to the oracle)."""
import numpy as np
import pytest

from helpers import clustered3, helix3, mrd, uniform3, yukawa_direct

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gen", [uniform3, helix3, clustered3])
def test_yukawa_fmm_against_direct(fmmb, gen):
    rng = np.random.default_rng(52)
    n, kappa = 5000, 4.0
    pts = gen(rng, n)
    tau = rng.standard_normal(n)
    tg = rng.random((400, 3))
    m = fmmb.SphericalHarmonics(fmmb.Yukawa3D(kappa), p=16)
    f = fmmb.FMM(m, pts, ppl=40, bbox=((0.0, 0.0, 0.0), 1.0))
    assert f.nlevels >= 3
    st = fmmb.build_expansions(f, pts, tau)
    u = fmmb.evaluate_at_sources(f, st)
    assert mrd(u, yukawa_direct(pts, tau, pts, kappa, self_excluded=True)) < 1e-5
    ut = fmmb.evaluate(f, st, tg)
    gt = fmmb.evaluate(f, st, tg, output=fmmb.Gradient())
    dp, dg = yukawa_direct(pts, tau, tg, kappa, gradient=True)
    assert mrd(ut, dp) < 1e-5
    assert mrd(gt, dg) < 1e-4


def test_yukawa_gradient_at_sources(fmmb):
    rng = np.random.default_rng(4)
    n, kappa = 20000, 5.0                                               # p = 12: the order of tol 1e-6
    pts = uniform3(rng, n)
    tau = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Yukawa3D(kappa), p=12), pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
    st = fmmb.build_expansions(f, pts, tau)
    u, g = fmmb.evaluate_at_sources_both(f, st)
    sel = np.sort(rng.choice(n, 200, replace=False))
    d = pts[sel, None, :] - pts[None, :, :]
    r = np.sqrt(np.einsum("tsk,tsk->ts", d, d))
    r[np.arange(len(sel)), sel] = 1.0                                  # the self terms, dropped below
    e = np.exp(-kappa * r) / r
    e[np.arange(len(sel)), sel] = 0.0
    du = e @ tau / (4 * np.pi)
    dg = np.einsum("ts,tsk->tk", -(e * (1 + kappa * r) / r ** 2) * tau[None, :], d) / (4 * np.pi)
    assert mrd(u[sel], du) < 5e-6
    assert mrd(g[sel], dg) < 5e-5


def test_yukawa_laplace_limit(fmmb):
    """κ = 1e-10: the Yukawa operators (built by projection on the device) and radial weights
    reduce to the exact Laplace ones; the FMMs agree to the kernels' own difference."""
    rng = np.random.default_rng(3)
    n = 20000
    pts = uniform3(rng, n)
    tau = rng.standard_normal(n)
    out = []
    for k in (fmmb.Yukawa3D(1e-10), fmmb.Laplace3D()):
        f = fmmb.FMM(fmmb.SphericalHarmonics(k, p=8), pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
        assert f.nlevels >= 4
        out.append(fmmb.evaluate_at_sources_both(f, fmmb.build_expansions(f, pts, tau)))
    assert mrd(out[0][0], out[1][0]) < 1e-9
    assert mrd(out[0][1], out[1][1]) < 1e-9


def test_yukawa_errors(fmmb):
    with pytest.raises(fmmb.ArgumentError):
        fmmb.OperatorCache(fmmb.SphericalHarmonics(fmmb.Yukawa3D(-1.0), p=6))
    pts = np.random.default_rng(1).random((3000, 3))
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Yukawa3D(2.0), p=12), pts, ppl=64)
    with pytest.raises(fmmb.Unsupported):                               # the tensor-core M2L takes p ≤ 11
        fmmb.FMMState(f, "mixed")


@pytest.mark.parametrize("p,kappa,gen", [(11, 5.0, uniform3), (8, 10.0, clustered3), (6, 2.0, helix3)])
def test_yukawa_mixed_path(fmmb, p, kappa, gen):
    """The mixed path of Yukawa3D: the tensor-core M2L with each level width's class operators split
    into FP16 head and tail (the rest of the matvec in FP64) against the FP64 path on the same
    tree: potential within 1e-6 and gradient within 1e-5 relative L2 (the mixed path's stated
    tolerance); the FP64 path's own error against direct sums bounds the mixed one's too."""
    rng = np.random.default_rng(90 + p)
    n = 40000
    pts = gen(rng, n)
    tau = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Yukawa3D(kappa), p=p), pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
    assert f.nlevels >= 4
    ud, gd = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions(f, pts, tau, precision="fp64"))
    um, gm = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions(f, pts, tau, precision="mixed"))
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel(um, ud) < 1e-6
    assert rel(gm, gd) < 1e-5
    sel = np.sort(rng.choice(n, 300, replace=False))
    d = pts[sel, None, :] - pts[None, :, :]
    r = np.sqrt(np.einsum("tsk,tsk->ts", d, d))
    r[np.arange(len(sel)), sel] = np.inf                                 # the self terms
    dp = (np.exp(-kappa * r) / r) @ tau / (4 * np.pi)
    assert rel(um[sel], dp) < rel(ud[sel], dp) + 2e-6


YK_PARITY = [("uniform", 20000, 40, 12, 5.0, 61), ("clustered", 8000, 30, 16, 4.0, 62), ("helix", 6000, 30, 8, 10.0, 63)]


@pytest.mark.parametrize("name,n,ppl,p,kappa,seed", YK_PARITY)
def test_yukawa_fp64_path_matches_oracle(oracle, fmmb, name, n, ppl, p, kappa, seed):
    """The device path against the oracle's restatement of harmonics_yukawa.jl on the same tree:
    potential and gradient at the sources and at targets within 1e-12 / 1e-11 (max-norm
    relative); multipoles and locals within 1e-9. Both sides build the per-width operators by
    projection with the same rule, but the quadrature nodes (Newton's iteration here, the
    Golub–Welsch eigenvalues in the oracle, as the reference) and the products' summation orders
    differ by rounding, and the projection amplifies that in the highest degrees: on the oracle
    alone, nodes moved by 3e-16 move the p = 16 multipoles of the clustered case by 1.9e-10
    relative and its potentials by 2.9e-13."""
    from helpers import DISTRIBUTIONS3
    rng = np.random.default_rng(seed)
    pts = DISTRIBUTIONS3[name](rng, n)
    tau = rng.standard_normal(n)
    tg = rng.random((500, 3))
    O = oracle.FMM(p, pts, ppl, kernel="yukawa", kappa=kappa)
    O.build_expansions(pts, tau)
    ou, og = O.evaluate_at_sources()
    tu, tgr = O.evaluate(tg)
    OM, OL = O.expansions()
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Yukawa3D(kappa), p=p), pts, ppl=ppl, bbox=((0.0, 0.0, 0.0), 1.0))
    assert f.nnodes == O.tree.n and f.nlevels >= 4
    st = fmmb.build_expansions(f, pts, tau)
    M, Lc = st.expansions()
    assert np.max(np.abs(M - OM)) < 1e-9 * np.max(np.abs(OM))
    assert np.max(np.abs(Lc - OL)) < 1e-9 * np.max(np.abs(OL))
    u, g = fmmb.evaluate_at_sources_both(f, st)
    assert mrd(u, ou) < 1e-12 and mrd(g, og) < 1e-11
    assert mrd(fmmb.evaluate(f, st, tg), tu) < 1e-12
    assert mrd(fmmb.evaluate(f, st, tg, output=fmmb.Gradient()), tgr) < 1e-11
