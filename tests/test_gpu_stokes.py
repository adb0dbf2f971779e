"""StokesHarmonics(Stokeslet3D(); p) on the device (FP64 path) through the Stokes plan API,
against FP64 direct Stokeslet sums (1/8π)Σ_{j≠i}[f_j/r + d(d·f_j)/r³] (src/kernels.jl:253-272),
as the reference's own Stokes harmonics tests do (test/test_harmonics.jl, Stokeslet checks
against direct sums). Tolerances: a single-leaf tree (all near field) within 1e-13; the FMM at
p = 8 / 12 / 16 within 3e-3 / 1e-4 / 1e-5 relative L2 of the velocities at sampled sources,
and the error falling with p."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def stokes_direct(src, f, sel):
    """Velocities at the sources `sel` (self excluded), FP64, vectorised in chunks."""
    out = np.zeros((len(sel), 3))
    for a in range(0, len(sel), 64):
        idx = sel[a:a + 64]
        d = src[idx, None, :] - src[None, :, :]                     # (t, s, 3)
        r2 = np.einsum("tsk,tsk->ts", d, d)
        r2[np.arange(len(idx)), idx] = np.inf                         # the i = j term
        ir = 1.0 / np.sqrt(r2)
        df = np.einsum("tsk,sk->ts", d, f) * ir ** 3
        out[a:a + 64] = (np.einsum("ts,sk->tk", ir, f) + np.einsum("ts,tsk->tk", df, d)) / (8 * np.pi)
    return out


def sphere_points(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None] + rng.uniform(-0.01, 0.01, (n, 3))


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
