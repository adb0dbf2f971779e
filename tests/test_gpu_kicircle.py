"""KernelIndependent(Laplace2D(); nequiv) on the device (the 2D circle method of
src/operators/kifmm.jl), points in the plane z = 0 of the octree, FP64: against FP64 direct sums
of c·log r², c = −1/(4π), as the reference checks it (test/test_operators_kifmm.jl; accuracy
~(0.547)^N per translation, docs/kifmm.md: 2e-8 at N = 30, rounding-limited near 1e-13 at
N = 60): at the sources and at targets, uniform and clustered points."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu
C2 = -1 / (4 * np.pi)


def direct2(src, tau, tgt, self_idx=None):
    pot = np.zeros(len(tgt))
    grad = np.zeros((len(tgt), 2))
    for a in range(0, len(tgt), 512):
        d = tgt[a:a + 512, None, :] - src[None, :, :]
        r2 = np.einsum("tsk,tsk->ts", d, d)
        if self_idx is not None:
            r2[np.arange(len(r2)), self_idx[a:a + 512]] = 1.0
        lr = np.log(r2)
        g = 2 * C2 * tau[None, :] / r2
        if self_idx is not None:
            lr[np.arange(len(r2)), self_idx[a:a + 512]] = 0.0
            g[np.arange(len(r2)), self_idx[a:a + 512]] = 0.0
        pot[a:a + 512] = C2 * lr @ tau
        grad[a:a + 512] = np.einsum("ts,tsk->tk", g, d)
    return pot, grad


def clustered2(rng, n):
    c = 0.1 + 0.8 * rng.random((6, 2))
    return np.clip(c[np.arange(n) % 6] + 0.02 * rng.standard_normal((n, 2)), 0.0, 1.0)


@pytest.mark.parametrize("dist", ["uniform", "clustered"])
def test_circle_ki_against_direct(fmmb, dist):
    rng = np.random.default_rng(1)
    n = 20000
    pts = rng.random((n, 2)) if dist == "uniform" else clustered2(rng, n)
    tau = rng.standard_normal(n)
    m = fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=60)
    f = fmmb.FMM(m, pts, ppl=50, bbox=((0.0, 0.0), 1.0))
    assert f.nlevels >= 4
    st = fmmb.build_expansions(f, pts, tau)
    u, g = fmmb.evaluate_at_sources_both(f, st)
    assert g.shape == (n, 2)
    sel = np.sort(rng.choice(n, 400, replace=False))
    du, dg = direct2(pts, tau, pts[sel], sel)
    assert rel_l2(u[sel], du) < 1e-11, (dist, rel_l2(u[sel], du))
    assert rel_l2(g[sel], dg) < 1e-10, (dist, rel_l2(g[sel], dg))
    tg = rng.random((2000, 2))
    ut = fmmb.evaluate(f, st, tg)
    gt = fmmb.evaluate(f, st, tg, output=fmmb.Gradient())
    dut, dgt = direct2(pts, tau, tg)
    assert rel_l2(ut, dut) < 1e-11 and rel_l2(gt, dgt) < 1e-10


def test_circle_ki_order(fmmb):
    """Fewer points per circle: the error follows (r₁/r₂)^N, 2e-8 at N = 30 in the reference."""
    rng = np.random.default_rng(2)
    n = 20000
    pts = rng.random((n, 2))
    tau = rng.standard_normal(n)
    sel = np.sort(rng.choice(n, 300, replace=False))
    du, _ = direct2(pts, tau, pts[sel], sel)
    errs = []
    for N in (16, 30, 60):
        f = fmmb.FMM(fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=N), pts, ppl=50, bbox=((0.0, 0.0), 1.0))
        u = fmmb.evaluate_at_sources(f, fmmb.build_expansions(f, pts, tau))
        errs.append(rel_l2(u[sel], du))
    assert errs[0] > errs[1] > errs[2] and errs[1] < 1e-6, errs


def test_circle_ki_errors(fmmb):
    with pytest.raises(fmmb.ArgumentError):
        fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=3)
    m = fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=20)
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.FMM(m, np.zeros((10, 3)))


@pytest.mark.parametrize("dist,nequiv", [("uniform", 16), ("clustered", 16), ("uniform", 32), ("clustered", 60)])
def test_circle_ki_matches_oracle(oracle, fmmb, dist, nequiv):
    """The device path against the oracle's restatement of the method (oracle/ki_oracle.py) on
    the same tree: the device tree equals the oracle's (the embedded octree, perm included), and
    potentials and gradients agree far inside the method's own truncation error (1.8e-5 against
    direct sums at N = 16): the same approximation, not only two close to the truth. The bar is
    relative L2, 1e-10: the two sides' pseudo-inverses come from different SVDs (one-sided
    Jacobi here, LAPACK in the oracle), whose roundings the truncated modes amplify."""
    import ki_oracle as K
    rng = np.random.default_rng(40 + nequiv)
    n = 3000
    pts = rng.random((n, 2)) if dist == "uniform" else clustered2(rng, n)
    tau = rng.standard_normal(n)
    m = fmmb.KernelIndependent(fmmb.Laplace2D(), nequiv=nequiv)
    f = fmmb.FMM(m, pts, ppl=30, bbox=((0.0, 0.0), 1.0))
    u, g = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions(f, pts, tau))
    ou, og, T = K.circle_fmm(pts, tau, nequiv, 30, (0.0, 0.0), 1.0)
    t = f.tree()
    assert f.nnodes == T.n
    for k in ("cell", "level", "parent", "child_first", "colleagues", "perm"):
        assert np.array_equal(t[k], getattr(T, k)), k
    assert rel_l2(u, ou) < 1e-10
    assert rel_l2(g, og) < 1e-10
