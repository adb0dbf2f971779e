"""StokesHarmonics(Stokeslet3D(); p) on the device (FP64 path) through the Stokes plan API,
against FP64 direct Stokeslet sums (1/8π)Σ_{j≠i}[f_j/r + d(d·f_j)/r³] (src/kernels.jl:253-272),
as the reference's own Stokes harmonics test does (test/test_harmonics_stokes.jl:50-66: Stokeslets
within 1e-5 of direct sums at p = 16). Tolerances: a single-leaf tree (all near field) within 1e-13; the FMM at
p = 8 / 12 / 16 within 3e-3 / 1e-4 / 1e-5 relative L2 of the velocities at sampled sources,
and the error falling with p."""
import numpy as np
import pytest

from helpers import rel_l2, sphere_points, stokes_direct

pytestmark = pytest.mark.gpu


def test_single_leaf_is_the_direct_sum(fmmb):
    rng = np.random.default_rng(1)
    pts = rng.random((150, 3))
    f = rng.standard_normal((150, 3))
    plan = fmmb.StokesFMMPlan(pts, p=6, ppl=200)                     # the root is a leaf: no far field
    u = fmmb.stokes_fmm_eval(plan, f)
    ud = stokes_direct(pts, f, np.arange(150))
    assert rel_l2(u, ud) < 1e-13


@pytest.mark.parametrize("dist", ["uniform", "sphere"])
def test_stokes_harmonics_against_direct(fmmb, dist):
    rng = np.random.default_rng(2)
    n = 40000
    pts = rng.random((n, 3)) if dist == "uniform" else sphere_points(rng, n)
    f = rng.standard_normal((n, 3))
    sel = np.sort(rng.choice(n, 300, replace=False))
    ud = stokes_direct(pts, f, sel)
    errs = {}
    for p, tol in ((8, 3e-3), (12, 1e-4), (16, 1e-5)):
        plan = fmmb.StokesFMMPlan(pts, p=p, ppl=64)
        u = fmmb.stokes_fmm_eval(plan, f)
        errs[p] = rel_l2(u[sel], ud)
        assert errs[p] < tol, (dist, p, errs[p])
        if p == 16:
            assert np.array_equal(fmmb.stokes_fmm_eval(plan, f), u)   # deterministic
    assert errs[16] < errs[12] < errs[8]


def test_stokes_errors(fmmb):
    rng = np.random.default_rng(3)
    pts = rng.random((2000, 3))
    plan = fmmb.StokesFMMPlan(pts, p=8, ppl=64)
    with pytest.raises(fmmb.Unsupported):
        fmmb.FMMState(plan.fmm, "mixed")
    with pytest.raises(fmmb.Unsupported):
        fmmb.device_matvec(plan.fmm, plan.state, pts, np.ones(2000))
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.stokes_fmm_eval(plan, np.ones((1999, 3)))


@pytest.mark.parametrize("dist", ["uniform", "sphere"])
def test_stokes_blocks_are_laplace_expansions(fmmb, dist):
    """The four Stokes blocks against FP64 Laplace FMMs on the same tree (the Laplace path is
    pinned to the oracle): Φ_k are the expansions of the charges f_k; Ψ̂ at each node is
    (E[y·f] − c·E[f]) / w for both the multipoles and the leaves' locals (harmonics_stokes.jl's
    coupling, exact by linearity up to rounding)."""
    rng = np.random.default_rng(7)
    n, p = 20000, 10
    pts = rng.random((n, 3)) if dist == "uniform" else sphere_points(rng, n)
    f = rng.standard_normal((n, 3))
    plan = fmmb.StokesFMMPlan(pts, p=p, ppl=64)
    fmmb.stokes_fmm_eval(plan, f)
    SM, SL = plan.state.expansions()
    lm = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=p)
    lf = fmmb.FMM(lm, pts, ppl=64, bbox=fmmb.square_bbox(pts))
    t = lf.tree()
    assert lf.nlevels >= 4 and np.array_equal(plan.fmm.tree()["cell"], t["cell"])

    def lap(q):
        return fmmb.build_expansions(lf, pts, q).expansions()

    E = [lap(f[:, k]) for k in range(3)]
    for k in range(3):
        assert np.array_equal(SM[:, k], E[k][0]) and np.array_equal(SL[:, k], E[k][1])
    E0 = lap(np.einsum("ij,ij->i", pts, f))
    wl = lf.width / 2.0 ** t["level"]
    cen = lf.origin[None, :] + (t["cell"] + 0.5) * wl[:, None]
    leaf = t["leaf"].astype(bool)
    for i, sel in ((0, np.ones(lf.nnodes, bool)), (1, leaf)):
        ref = (E0[i] - sum(cen[:, k:k + 1] * E[k][i] for k in range(3))) / wl[:, None]
        got = (SM if i == 0 else SL)[:, 3]
        assert np.max(np.abs(got[sel] - ref[sel])) < 1e-12 * np.max(np.abs(ref[sel])), (dist, i)
