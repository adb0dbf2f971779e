"""StokesHarmonics(Stokeslet3D(); p) on the device (FP64 path) through the Stokes plan API,
against FP64 direct Stokeslet sums (1/8π)Σ_{j≠i}[f_j/r + d(d·f_j)/r³] (src/kernels.jl:253-272),
as the reference's own Stokes harmonics test does (test/test_harmonics_stokes.jl:50-66: Stokeslets
within 1e-5 of direct sums at p = 16). Tolerances: a single-leaf tree (all near field) within 1e-13; the FMM at
p = 8 / 12 / 16 within 3e-3 / 1e-4 / 1e-5 relative L2 of the velocities at sampled sources,
and the error falling with p."""
import numpy as np
import pytest

from helpers import mrd, rel_l2, sphere_points, stokes_direct, stokes_direct_all

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


# ---------------------------------------------------------------- stresslets, doublets, pressure
def _mixed(rng, n):
    """Stokeslets, unit stressvecs with their strengths, doublets and weights (the densities of
    test/test_harmonics_stokes.jl:10-12)."""
    nu = rng.standard_normal((n, 3))
    nu /= np.linalg.norm(nu, axis=1)[:, None]
    return dict(stokeslets=rng.standard_normal((n, 3)), stresslets=rng.standard_normal((n, 3)), stressvecs=nu,
                doublets=rng.standard_normal((n, 3)), weights=rng.random(n) + 0.5)


def _direct(pts, sel, d, output):
    return stokes_direct_all(pts, sel, f=d.get("stokeslets"), fs=d.get("stresslets"), nu=d.get("stressvecs"),
                             g=d.get("doublets"), w=d.get("weights"), output=output)


def test_single_leaf_densities_are_the_direct_sum(fmmb):
    rng = np.random.default_rng(11)
    pts = rng.random((150, 3))
    d = _mixed(rng, 150)
    plan = fmmb.StokesFMMPlan(pts, p=6, ppl=200)
    for output in ("velocity", "pressure", "gradient"):
        u = fmmb.stokes_fmm_eval(plan, output=output, **d)
        assert rel_l2(u, _direct(pts, np.arange(150), d, output)) < 1e-13, output


@pytest.mark.parametrize("dist", ["uniform", "sphere"])
def test_stresslets_doublets_against_direct(fmmb, dist):
    """test/test_harmonics_stokes.jl:48-60: mixed densities at p = 16 within 1e-4 (max-norm
    relative, velocity) and 1e-3 (pressure) of direct sums; here each kind alone as well."""
    rng = np.random.default_rng(12)
    n = 20000
    pts = rng.random((n, 3)) if dist == "uniform" else sphere_points(rng, n)
    d = _mixed(rng, n)
    sel = np.sort(rng.choice(n, 300, replace=False))
    plan = fmmb.StokesFMMPlan(pts, p=16, ppl=40)
    for output, tol in (("velocity", 1e-4), ("pressure", 1e-3)):
        u = fmmb.stokes_fmm_eval(plan, output=output, **d)
        assert mrd(u[sel], _direct(pts, sel, d, output)) < tol, (dist, output)
    for kind in ({"stresslets": d["stresslets"], "stressvecs": d["stressvecs"]}, {"doublets": d["doublets"]}):
        u = fmmb.stokes_fmm_eval(plan, **kind)
        assert mrd(u[sel], _direct(pts, sel, kind, "velocity")) < 1e-4, (dist, list(kind))


def test_densities_are_linear(fmmb):
    """The evaluation is linear in the densities: the sum of the three kinds evaluated apart is
    the evaluation of all three (up to rounding), and the weights scale each source."""
    rng = np.random.default_rng(13)
    n = 20000
    pts = sphere_points(rng, n)
    d = _mixed(rng, n)
    plan = fmmb.StokesFMMPlan(pts, p=12, ppl=64)
    w = d.pop("weights")
    for output in ("velocity", "pressure"):
        whole = fmmb.stokes_fmm_eval(plan, output=output, **d)
        parts = (fmmb.stokes_fmm_eval(plan, output=output, stokeslets=d["stokeslets"])
                 + fmmb.stokes_fmm_eval(plan, output=output, stresslets=d["stresslets"], stressvecs=d["stressvecs"])
                 + fmmb.stokes_fmm_eval(plan, output=output, doublets=d["doublets"]))
        assert rel_l2(parts, whole) < 1e-12, output
        pre = {k: (v * w[:, None] if k != "stressvecs" else v) for k, v in d.items()}
        assert rel_l2(fmmb.stokes_fmm_eval(plan, output=output, weights=w, **d),
                      fmmb.stokes_fmm_eval(plan, output=output, **pre)) < 1e-13, output


def test_stokeslets_with_small_doublets(fmmb):
    """test/test_harmonics_stokes.jl:72-77: the Stokes plan with stokeslets and doublets 0.01·g
    on a helix-like curve within 1e-5 of direct sums (here at the sources)."""
    rng = np.random.default_rng(14)
    n = 3000
    t = np.sort(rng.random(n)) * 8 * np.pi
    pts = np.stack([0.5 + 0.3 * np.cos(t), 0.5 + 0.3 * np.sin(t), 0.1 + 0.8 * t / t[-1]], axis=1)
    pts += 1e-3 * rng.standard_normal(pts.shape)
    d = dict(stokeslets=rng.standard_normal((n, 3)), doublets=0.01 * rng.standard_normal((n, 3)))
    plan = fmmb.StokesFMMPlan(pts, p=16, ppl=30)
    u = fmmb.stokes_fmm_eval(plan, **d)
    assert mrd(u, _direct(pts, np.arange(n), d, "velocity")) < 1e-5


def test_density_errors(fmmb):
    rng = np.random.default_rng(15)
    pts = rng.random((2000, 3))
    plan = fmmb.StokesFMMPlan(pts, p=8, ppl=64)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_fmm_eval(plan, stresslets=np.ones((2000, 3)))
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_fmm_eval(plan)
    with pytest.raises(fmmb.Unsupported):
        fmmb.stokes_fmm_eval(plan, stokeslets=np.ones((2000, 3)), output="hessian")


# ---------------------------------------------------------------- targets
@pytest.mark.parametrize("dist", ["uniform", "helix"])
def test_stokes_at_targets(fmmb, dist):
    """test/test_harmonics_stokes.jl:48-60 at targets: a plan with targets (its box covers both),
    Stokeslets within 1e-5 and mixed densities within 1e-4 (velocity) / 1e-3 (pressure) max-norm
    relative of direct sums at 400 uniform targets; stokes_fmm_eval_src_trg gives the same values
    at the sources and at the targets as the two separate evaluations."""
    rng = np.random.default_rng(16)
    n = 5000
    if dist == "uniform":
        pts = rng.random((n, 3))
    else:
        t = np.sort(rng.random(n)) * 6 * np.pi
        pts = np.stack([0.5 + 0.3 * np.cos(t), 0.5 + 0.3 * np.sin(t), 0.1 + 0.8 * t / t[-1]], axis=1)
    tg = rng.random((400, 3)) * 1.2 - 0.1                     # some outside the sources' cube
    d = _mixed(rng, n)
    plan = fmmb.StokesFMMPlan(pts, targets=tg, p=16, ppl=40)
    f = {"stokeslets": d["stokeslets"]}
    ref = stokes_direct_all(pts, None, f=d["stokeslets"], tgt=tg)
    assert mrd(fmmb.stokes_fmm_eval(plan, **f), ref) < 1e-5
    for output, tol in (("velocity", 1e-4), ("pressure", 1e-3)):
        u = fmmb.stokes_fmm_eval(plan, output=output, **d)
        ref = stokes_direct_all(pts, None, f=d["stokeslets"], fs=d["stresslets"], nu=d["stressvecs"],
                                g=d["doublets"], w=d["weights"], output=output, tgt=tg)
        assert mrd(u, ref) < tol, (dist, output)
        us, ut = fmmb.stokes_fmm_eval_src_trg(plan, output=output, **d)
        assert np.array_equal(ut, u)
        self_plan = fmmb.StokesFMMPlan(pts, p=16, ppl=40, bbox=fmmb.square_bbox(np.concatenate([pts, tg])))
        assert np.array_equal(us, fmmb.stokes_fmm_eval(self_plan, output=output, **d))


def test_stokes_target_errors(fmmb):
    rng = np.random.default_rng(17)
    pts = rng.random((2000, 3))
    plan = fmmb.StokesFMMPlan(pts, p=8, ppl=64)
    f = rng.standard_normal((2000, 3))
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_fmm_eval_src_trg(plan, stokeslets=f)                  # no targets
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_fmm_eval(plan, stokeslets=f, targets=np.array([[2.0, 0.5, 0.5]]))   # outside the box
    tg = pts[:50] * 0.99 + 0.005                                      # near the sources, inside the box
    u = fmmb.stokes_fmm_eval(plan, stokeslets=f, targets=tg)
    ref = stokes_direct_all(pts, None, f=f, tgt=tg)
    assert mrd(u, ref) < 3e-3


@pytest.mark.parametrize("dist", ["uniform", "sphere"])
def test_velocity_gradient(fmmb, dist):
    """test/test_harmonics_stokes.jl:48-60's Gradient() bars (10·tol: 1e-4 for Stokeslets, 1e-3
    for mixed densities, max-norm relative of the 3 × 3 matrices) at the sources and at targets,
    p = 16; the far-field gradient is the Hessians of the four local blocks (degree-(p−1) L2Ps of
    their gradient expansions). The trace of a Stokeslet velocity gradient vanishes (∇·u = 0)."""
    rng = np.random.default_rng(18)
    n = 20000
    pts = rng.random((n, 3)) if dist == "uniform" else sphere_points(rng, n)
    tg = rng.random((300, 3))
    d = _mixed(rng, n)
    plan = fmmb.StokesFMMPlan(pts, targets=tg, p=16, ppl=40)
    sel = np.sort(rng.choice(n, 200, replace=False))
    f = {"stokeslets": d["stokeslets"]}
    for dens, tol in ((f, 1e-4), (d, 1e-3)):
        gs, gt = fmmb.stokes_fmm_eval_src_trg(plan, output="gradient", **dens)
        kw = dict(f=dens.get("stokeslets"), fs=dens.get("stresslets"), nu=dens.get("stressvecs"),
                  g=dens.get("doublets"), w=dens.get("weights"), output="gradient")
        es = np.max(np.linalg.norm(gs[sel] - stokes_direct_all(pts, sel, **kw), axis=(1, 2)))
        rs = np.max(np.linalg.norm(stokes_direct_all(pts, sel, **kw), axis=(1, 2)))
        ref_t = stokes_direct_all(pts, None, tgt=tg, **kw)
        et = np.max(np.linalg.norm(gt - ref_t, axis=(1, 2))) / np.max(np.linalg.norm(ref_t, axis=(1, 2)))
        assert es / rs < tol and et < tol, (dist, list(dens), es / rs, et)
        if dens is f:
            tr = np.abs(np.trace(gt, axis1=1, axis2=2))
            assert np.max(tr) < 1e-4 * np.max(np.linalg.norm(gt, axis=(1, 2)))


ST_PARITY = [("uniform", 20000, 64, 12, 71), ("sphere", 20000, 64, 16, 72), ("helix", 8000, 30, 8, 73)]


@pytest.mark.parametrize("name,n,ppl,p,seed", ST_PARITY)
def test_stokes_fp64_path_matches_oracle(oracle, fmmb, name, n, ppl, p, seed):
    """The device's Stokes harmonics against the oracle's restatement of harmonics_stokes.jl
    on the same box and tree: the four expansion blocks of every node (multipoles and leaf
    locals), the velocities and pressures at the sources and at targets, max-norm relative."""
    from helpers import DISTRIBUTIONS3
    rng = np.random.default_rng(seed)
    pts = sphere_points(rng, n) if name == "sphere" else DISTRIBUTIONS3[name](rng, n)
    f = rng.standard_normal((n, 3))
    plan = fmmb.StokesFMMPlan(pts, p=p, ppl=ppl)
    lo = plan.fmm.origin
    O = oracle.FMM(p, pts, ppl, origin=tuple(lo), width=plan.fmm.width, kernel="stokes")
    assert plan.fmm.nnodes == O.tree.n and plan.fmm.nlevels >= 4
    O.build_expansions(pts, f)
    ov, op = O.evaluate_at_sources_stokes()
    u = fmmb.stokes_fmm_eval(plan, f)
    pr = fmmb.stokes_fmm_eval(plan, f, output="pressure")
    M, Lc = plan.state.expansions()
    OM, OL = O.expansions()
    M, Lc = M.reshape(OM.shape), Lc.reshape(OL.shape)
    assert np.max(np.abs(M - OM)) < 1e-12 * np.max(np.abs(OM))
    assert np.max(np.abs(Lc - OL)) < 1e-11 * np.max(np.abs(OL))
    assert mrd(u, ov) < 1e-12 and mrd(pr, op) < 1e-11
    tg = pts[rng.choice(n, 300, replace=False)] + 1e-3 * rng.standard_normal((300, 3))
    tg = np.clip(tg, lo + 1e-9, lo + plan.fmm.width - 1e-9)
    tv, tp = O.evaluate_stokes(tg)
    assert mrd(fmmb.stokes_fmm_eval(plan, f, targets=tg), tv) < 1e-12
    assert mrd(fmmb.stokes_fmm_eval(plan, f, targets=tg, output="pressure"), tp) < 1e-11
