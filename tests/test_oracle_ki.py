"""The oracle's restatement of the circle kernel-independent method (oracle/ki_oracle.py) pinned
as the reference pins the method: against FP64 direct sums of c·log r², the error falling with
the circle's points to the reference's stated levels (src/operators/kifmm.jl:7-10: the global
relative error on uniform data 6e-9 at N = 32, a rounding floor near 1e-14 at N = 64), on
uniform and clustered (adaptive, ghosted) points."""
import numpy as np
import pytest


def _direct(pts, tau):
    import ki_oracle as K
    d = pts[:, None, :] - pts[None, :, :]
    r2 = np.einsum("tsk,tsk->ts", d, d)
    np.fill_diagonal(r2, 1.0)
    g = K.C2 * np.log(r2)
    np.fill_diagonal(g, 0.0)
    gr = 2 * K.C2 / r2
    np.fill_diagonal(gr, 0.0)
    return g @ tau, np.einsum("ts,tsk->tk", gr * tau[None, :], d)


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_circle_oracle_against_direct(oracle, kind):
    import ki_oracle as K
    rng = np.random.default_rng(31)
    n = 2500
    if kind == "uniform":
        pts = rng.random((n, 2))
    else:
        c = 0.1 + 0.8 * rng.random((5, 2))
        pts = np.clip(c[np.arange(n) % 5] + 0.01 * rng.standard_normal((n, 2)), 0.0, 1.0)
    tau = rng.standard_normal(n)
    ud, gd = _direct(pts, tau)
    errs = []
    for ne, bar in ((16, 1e-4), (32, 5e-8), (48, 1e-10), (60, 1e-12)):
        u, g, T = K.circle_fmm(pts, tau, ne, 30, (0.0, 0.0), 1.0)
        e = np.linalg.norm(u - ud) / np.linalg.norm(ud)
        eg = np.linalg.norm(g - gd) / np.linalg.norm(gd)
        assert e < bar and eg < 100 * bar, (ne, e, eg)
        errs.append(e)
    assert errs == sorted(errs, reverse=True)              # falls with the circle's points
    if kind == "clustered":
        assert T.ghost.any() and T.L >= 5                  # an adaptive tree with ghosts


def test_circle_oracle_operators(oracle):
    """The folded M2M reproduces, on the parent's large circle, the check potentials of the
    children's equivalent densities (the identity it is built from), and the pseudo-inverse of
    the upward check map recovers an equivalent density from its own check potentials."""
    import ki_oracle as K
    op = K.CircleLevel(32, 0.25, 50 * np.finfo(float).eps)
    rng = np.random.default_rng(2)
    q = rng.standard_normal(4 * 32)
    centers = [(np.array([k & 1, (k >> 1) & 1], float) - 0.5) * 0.125 for k in range(4)]
    child_small = K.circle_points(32, K.SMALL * 0.125)
    check = sum(K.kernel_matrix(child_small + c, op.large) @ q[32 * k:32 * (k + 1)] for k, c in enumerate(centers))
    parent = op.m2m @ q
    assert np.linalg.norm(K.kernel_matrix(op.small, op.large) @ parent - check) < 1e-12 * np.linalg.norm(check)
    x = rng.standard_normal(32)
    A = K.kernel_matrix(op.small, op.large)
    assert np.linalg.norm(op.up.apply(A @ x) - x) < 1e-9 * np.linalg.norm(x)


def test_cube_oracle_against_direct(oracle):
    """The oracle's cube KI method (dense M2L) against FP64 direct sums of 1/(4πr): the error falls
    with p to the floor the reference's default truncation for Laplace3D(Float32) sets
    (50·eps(Float32) on the check maps: ≈ 1e-6, docs/kifmm.md's Float32 figures)."""
    import ki_oracle as K
    rng = np.random.default_rng(33)
    n = 2500
    pts = rng.random((n, 3))
    tau = rng.standard_normal(n)
    d = pts[:, None, :] - pts[None, :, :]
    r = np.sqrt(np.einsum("tsk,tsk->ts", d, d))
    np.fill_diagonal(r, np.inf)
    ud = (K.C3 / r) @ tau
    errs = []
    for p, bar in ((4, 3e-4), (6, 5e-6), (8, 3e-6)):
        u, g, M, Lc, T = K.cube_fmm(pts, tau, p, 64, (0.0, 0.0, 0.0), 1.0)
        errs.append(np.linalg.norm(u - ud) / np.linalg.norm(ud))
        assert errs[-1] < bar, (p, errs[-1])
    assert errs[0] > errs[1] > errs[2] * 0.5


@pytest.mark.parametrize("p", [4, 6, 8])
def test_cube_spectral_m2l_equals_the_dense_product(oracle, p):
    """The oracle's restatement of the spectral M2L (zero-padded lattice, circulant kernel tables,
    FFTs) equals the dense kernel-matrix translation K(small + o·w → small) it replaces, in FP64,
    for far offsets of every kind and two widths (the reference's own check of the spectral
    operator, test/test_cubeki.jl:43-69)."""
    import ki_oracle as K
    rng = np.random.default_rng(40 + p)
    d = 0.1
    for w in (1.0, 0.25):
        lv = K.CubeLevel(p, 16, d, w, 50 * np.finfo(np.float32).eps)
        a = (1 + d) * w / 2
        for off in ((2, 0, 0), (3, -2, 1), (-3, 3, 3), (0, 2, -3), (-2, -2, 2)):
            sigma = rng.standard_normal(lv.ns)
            dense = lv.m2l(off) @ sigma
            spec = K.spectral_m2l(p, a, off, w, sigma)
            assert np.linalg.norm(spec - dense) < 1e-12 * np.linalg.norm(dense), (w, off)
