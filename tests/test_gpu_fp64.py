"""The device tree and the plain FP64 path against the CPU oracle.

Mirrors the reference's device tests: test/test_device_tree.jl (the tree equal to the host
tree field by field), test/test_device_passes.jl (lists as sets, robustness) and
test/test_device_harmonics.jl (multipoles < 1e-13, locals < 1e-11, matvec and evaluation
at targets < 1e-11, gradient < 1e-10). The FP64 path's bar here is 1e-12 (max-norm relative)
on potentials.
"""
import numpy as np
import pytest

from helpers import (DISTRIBUTIONS3, check_coverage, check_tree_invariants, gaussian_cloud, mrd, oracle_tree_dict,
                     pairs_equal_as_sets, same_structure)

pytestmark = pytest.mark.gpu
BOX = ((0.0, 0.0, 0.0), 1.0)

TREE_CASES = [("uniform", 20000, 40, 1), ("mixed", 8000, 40, 2), ("sphere", 8000, 60, 3), ("helix", 8000, 50, 4),
              ("clustered", 6000, 30, 5), ("one_octant", 5000, 20, 6), ("mixed", 3000, 8, 7)]


def _method(F, p):
    return F.SphericalHarmonics(F.Laplace3D(), p=p)


@pytest.mark.parametrize("name,n,ppl,seed", TREE_CASES)
def test_device_tree_equals_host_tree(oracle, fmmb, name, n, ppl, seed):
    rng = np.random.default_rng(seed)
    pts = DISTRIBUTIONS3[name](rng, n)
    T = oracle.Tree.build(pts, ppl)
    f = fmmb.FMM(_method(fmmb, 4), pts, ppl=ppl, bbox=BOX)
    t = f.tree()
    ref = oracle_tree_dict(T)
    assert f.nlevels == T.L and f.nnodes == T.n
    assert same_structure(t, ref) is None, same_structure(t, ref)
    # the order of the points within the childless nodes too (the host tree's perm)
    assert np.array_equal(t["perm"], ref["perm"])
    # the far pairs of every level, as sets of (target, source, far offset)
    for l in range(T.L):
        a = sorted(zip(*[x.tolist() for x in f.pairs(l)]))
        b = sorted(zip(*[x.tolist() for x in T.pairs(l)]))
        assert a == b, f"level {l}"


def test_device_tree_equals_host_tree_adaptive_cloud(oracle, fmmb):
    """The adaptive configuration's point cloud (16 Gaussians, sigma 0.01) at 5e5 points and
    ppl = 64: 10 levels, ghosts and 2:1 restriction at scale; every field, perm and the far
    pairs of every level equal the oracle's."""
    pts = gaussian_cloud(500_000)
    T = oracle.Tree.build(pts, 64)
    f = fmmb.FMM(_method(fmmb, 4), pts, ppl=64, bbox=BOX)
    assert T.L >= 10 and f.nlevels == T.L and f.nnodes == T.n and T.ghost.sum() > 0
    t = f.tree()
    ref = oracle_tree_dict(T)
    assert same_structure(t, ref) is None, same_structure(t, ref)
    assert np.array_equal(t["perm"], ref["perm"])
    for l in range(T.L):
        assert pairs_equal_as_sets(f.pairs(l), T.pairs(l)), f"level {l}"


@pytest.mark.parametrize("name", sorted(DISTRIBUTIONS3))
def test_device_lists_coverage(oracle, fmmb, name):
    """test/test_coverage.jl:86-96 on the device tree and the device far pairs."""
    rng = np.random.default_rng(4)
    pts = DISTRIBUTIONS3[name](rng, 400)
    f = fmmb.FMM(_method(fmmb, 4), pts, ppl=4, bbox=BOX)
    check_coverage(f.tree(), [f.pairs(l) for l in range(f.nlevels)], oracle.far_offsets())


def test_device_lists_coverage_larger(oracle, fmmb):
    rng = np.random.default_rng(5)
    for pts, ppl in ((DISTRIBUTIONS3["mixed"](rng, 800), 3), (DISTRIBUTIONS3["uniform"](rng, 12), 12),
                     (DISTRIBUTIONS3["clustered"](rng, 10000), 30), (DISTRIBUTIONS3["sphere"](rng, 10000), 16)):
        f = fmmb.FMM(_method(fmmb, 4), pts, ppl=ppl, bbox=BOX)
        check_coverage(f.tree(), [f.pairs(l) for l in range(f.nlevels)], oracle.far_offsets())


def test_device_tree_invariants(fmmb):
    rng = np.random.default_rng(11)
    pts = DISTRIBUTIONS3["mixed"](rng, 2500)
    f = fmmb.FMM(_method(fmmb, 4), pts, ppl=10, bbox=BOX)
    t = f.tree()
    assert t["ghost"].sum() > 0 and t["xlist"].sum() > 0 and f.nlevels >= 5
    check_tree_invariants(t, pts)


def test_device_tree_deterministic(fmmb):
    rng = np.random.default_rng(12)
    pts = DISTRIBUTIONS3["sphere"](rng, 20000)
    m = _method(fmmb, 4)
    a = fmmb.FMM(m, pts, ppl=30, bbox=BOX).tree()
    b = fmmb.FMM(m, pts, ppl=30, bbox=BOX).tree()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_small_trees(oracle, fmmb):
    rng = np.random.default_rng(13)
    m = _method(fmmb, 6)
    for n, ppl in ((1, 5), (10, 50), (64, 64), (65, 64), (300, 4)):
        pts = rng.random((n, 3))
        tau = rng.standard_normal(n)
        f = fmmb.FMM(m, pts, ppl=ppl, bbox=BOX)
        T = oracle.Tree.build(pts, ppl)
        assert same_structure(f.tree(), oracle_tree_dict(T)) is None
        st = fmmb.build_expansions(f, pts, tau)
        u, g = fmmb.evaluate_at_sources_both(f, st)
        du, dg = oracle.direct(pts, tau)
        if n == 1:
            assert u[0] == 0 and np.all(g == 0)
            continue
        O = oracle.FMM(6, pts, ppl)
        O.build_expansions(pts, tau)
        ou, og = O.evaluate_at_sources()
        assert mrd(u, ou) < 1e-12 and mrd(g, og) < 1e-11
        assert mrd(u, du) < 1e-3 and mrd(g, dg) < 1e-2


PARITY_CASES = [("uniform", 30000, 40, 10, 21), ("mixed", 12000, 40, 10, 22), ("helix", 8000, 30, 8, 23),
                ("sphere", 10000, 60, 12, 24), ("clustered", 8000, 30, 16, 25)]


@pytest.mark.parametrize("name,n,ppl,p,seed", PARITY_CASES)
def test_fp64_path_matches_oracle(oracle, fmmb, name, n, ppl, p, seed):
    rng = np.random.default_rng(seed)
    pts = DISTRIBUTIONS3[name](rng, n)
    tau = rng.standard_normal(n)
    targets = rng.random((500, 3))
    O = oracle.FMM(p, pts, ppl)
    O.build_expansions(pts, tau)
    ou, og = O.evaluate_at_sources()
    tu, tg = O.evaluate(targets)
    OM, OL = O.expansions()
    f = fmmb.FMM(_method(fmmb, p), pts, ppl=ppl, bbox=BOX)
    st = fmmb.build_expansions(f, pts, tau)
    M, Lc = st.expansions()
    assert np.max(np.abs(M - OM)) < 1e-13 * np.max(np.abs(OM))
    assert np.max(np.abs(Lc - OL)) < 1e-11 * np.max(np.abs(OL))
    u, g = fmmb.evaluate_at_sources_both(f, st)
    assert mrd(u, ou) < 1e-12
    assert mrd(g, og) < 1e-11
    assert mrd(fmmb.evaluate(f, st, targets), tu) < 1e-12
    assert mrd(fmmb.evaluate(f, st, targets, output=fmmb.Gradient()), tg) < 1e-11
    # the separate-output calls agree with the combined one bitwise
    assert np.array_equal(fmmb.evaluate_at_sources(f, st), u)
    assert np.array_equal(fmmb.evaluate_at_sources(f, st, output=fmmb.Gradient()), g)


def test_fp64_accuracy_vs_direct(oracle, fmmb):
    """test/test_harmonics.jl:129-152: p = 16, 6000 points, potential < 1e-5, gradient < 1e-4."""
    rng = np.random.default_rng(31)
    for name in DISTRIBUTIONS3:
        pts = DISTRIBUTIONS3[name](rng, 6000)
        tau = rng.standard_normal(6000)
        targets = rng.random((500, 3))
        f = fmmb.FMM(_method(fmmb, 16), pts, ppl=40, bbox=BOX)
        st = fmmb.build_expansions(f, pts, tau)
        du, _ = oracle.direct(pts, tau)
        tu, tg = oracle.direct(pts, tau, targets)
        assert mrd(fmmb.evaluate_at_sources(f, st), du) < 1e-5, name
        assert mrd(fmmb.evaluate(f, st, targets), tu) < 1e-5, name
        assert mrd(fmmb.evaluate(f, st, targets, output=fmmb.Gradient()), tg) < 1e-4, name


def test_device_direct(oracle, fmmb):
    import ctypes as C
    import torch
    rng = np.random.default_rng(41)
    src = rng.random((3000, 3))
    tau = rng.standard_normal(3000)
    tg = rng.random((700, 3))
    du, dg = oracle.direct(src, tau, tg)
    ctx = fmmb.default_context()
    s_d = torch.from_numpy(src).cuda()
    t_d = torch.from_numpy(tau).cuda()
    g_d = torch.from_numpy(tg).cuda()
    pot = torch.zeros(700, dtype=torch.float64, device="cuda")
    grad = torch.zeros((700, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = fmmb.lib().fmmb_direct_dev(ctx._h, C.c_void_p(s_d.data_ptr()), C.c_void_p(t_d.data_ptr()), 3000,
                                    C.c_void_p(g_d.data_ptr()), None, 700, C.c_void_p(pot.data_ptr()),
                                    C.c_void_p(grad.data_ptr()))
    assert rc == 0
    assert mrd(pot.cpu().numpy(), du) < 1e-13 and mrd(grad.cpu().numpy(), dg) < 1e-13


def test_errors(fmmb):
    rng = np.random.default_rng(51)
    m = _method(fmmb, 6)
    pts = rng.random((3000, 3))
    tau = rng.standard_normal(3000)
    for bad in ((np.nan, 0.5, 0.5), (0.5, np.inf, 0.5)):
        q = pts.copy()
        q[17] = bad
        with pytest.raises(fmmb.ArgumentError, match="finite"):
            fmmb.FMM(m, q, ppl=40, bbox=BOX)
    with pytest.raises(fmmb.ArgumentError, match="outside"):
        fmmb.FMM(m, pts, ppl=40, bbox=((0.5, 0.5, 0.5), 1.0))
    with pytest.raises(fmmb.ArgumentError, match="max_levels"):
        fmmb.FMM(m, np.full((20, 3), 0.3), ppl=5, bbox=BOX, max_levels=10)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.FMM(m, pts, ppl=0, bbox=BOX)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.FMM(m, np.zeros((0, 3)), ppl=5, bbox=BOX)
    f = fmmb.FMM(m, pts, ppl=40, bbox=BOX)
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.build_expansions(f, pts[:-1], tau[:-1])
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.build_expansions(f, pts, tau[:-1])
    with pytest.raises(fmmb.ArgumentError):
        fmmb.build_expansions(f, pts, tau.astype(np.complex128))
    st = fmmb.FMMState(f)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.evaluate_at_sources(f, st)
    fmmb.build_expansions_(st, f, pts, tau)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.evaluate_at_sources(f, st, output="pressure")
    with pytest.raises(fmmb.ArgumentError, match="outside"):
        fmmb.evaluate(f, st, np.array([[1.0 + 1e-12, 0.5, 0.5]]))
    with pytest.raises(fmmb.ArgumentError):
        fmmb.OperatorCache(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=0))
    other = fmmb.OperatorCache(_method(fmmb, 6))
    with pytest.raises(fmmb.ArgumentError, match="different method"):
        fmmb.FMM(m, pts, ppl=40, cache=other)


def test_nan_density_poisons_one_application(fmmb):
    """test/test_device_passes.jl:187-196: a plan recovers bitwise after a non-finite density."""
    rng = np.random.default_rng(61)
    pts = DISTRIBUTIONS3["mixed"](rng, 5000)
    tau = rng.standard_normal(5000)
    f = fmmb.FMM(_method(fmmb, 8), pts, ppl=40, bbox=BOX)
    st = fmmb.FMMState(f)
    u0 = fmmb.device_matvec(f, st, pts, tau)
    bad = tau.copy()
    bad[5] = np.nan
    assert np.any(np.isnan(fmmb.device_matvec(f, st, pts, bad)))
    assert np.array_equal(fmmb.device_matvec(f, st, pts, tau), u0)
    # a fresh plan gives the same result bitwise (determinism)
    f2 = fmmb.FMM(_method(fmmb, 8), pts, ppl=40, bbox=BOX)
    assert np.array_equal(fmmb.device_matvec(f2, fmmb.FMMState(f2), pts, tau), u0)


def test_shared_cache_snaps_boxes(oracle, fmmb):
    """src/operators/cache.jl:57-83: the second box is snapped to ldexp(W0, e)."""
    rng = np.random.default_rng(71)
    m = _method(fmmb, 8)
    cache = fmmb.OperatorCache(m)
    pts = rng.random((4000, 3))
    tau = rng.standard_normal(4000)
    f1 = fmmb.FMM(m, pts, ppl=40, bbox=BOX, cache=cache)
    assert cache.W0 == 1.0
    pts2 = 0.2 + 0.3 * rng.random((4000, 3))
    f2 = fmmb.FMM(m, pts2, ppl=40, cache=cache)          # square_bbox then snapped
    assert f2.width in (0.25, 0.5)
    st = fmmb.build_expansions(f2, pts2, tau)
    du, _ = oracle.direct(pts2, tau)
    assert mrd(fmmb.evaluate_at_sources(f2, st), du) < 2e-4            # p = 8
    O = oracle.FMM(8, pts2, 40, origin=tuple(f2.origin), width=f2.width, ref_width=1.0)
    O.build_expansions(pts2, tau)
    assert mrd(fmmb.evaluate_at_sources(f2, st), O.evaluate_at_sources()[0]) < 1e-12
    del f1


def test_handles_destroyed_in_any_order(fmmb):
    """A garbage collector finalises in any order: destroying a context, cache or plan before
    the handles built on it must defer their release, not crash."""
    import ctypes as C
    L = fmmb.lib()
    rng = np.random.default_rng(81)
    pts = rng.random((5000, 3))
    tau = rng.standard_normal(5000)
    for order in ("ctx_first", "plan_first", "cache_first"):
        ctx = C.c_void_p()
        assert L.fmmb_ctx_create(0, C.byref(ctx)) == 0
        d = fmmb._MethodDesc(1, 1, 6, 0, 0.0)
        cache = C.c_void_p()
        assert L.fmmb_cache_create(ctx, C.byref(d), C.byref(cache)) == 0
        o = fmmb._TreeOpts()
        o.ppl, o.max_levels, o.has_bbox, o.width = 40, 30, 1, 1.0
        plan = C.c_void_p()
        assert L.fmmb_plan_create(cache, fmmb._ptr(pts), 5000, C.byref(o), C.byref(plan)) == 0
        st = C.c_void_p()
        assert L.fmmb_state_create(plan, 0, C.byref(st)) == 0
        if order == "ctx_first":
            assert L.fmmb_ctx_destroy(ctx) == 0
        elif order == "plan_first":
            assert L.fmmb_plan_destroy(plan) == 0
        else:
            assert L.fmmb_cache_destroy(cache) == 0
        u = np.zeros(5000)
        assert L.fmmb_matvec(st, fmmb._ptr(pts), fmmb._ptr(tau), 5000, 1, fmmb._ptr(u), None) == 0   # still usable
        assert np.all(np.isfinite(u))
        assert L.fmmb_state_destroy(st) == 0
        for name, h in (("fmmb_plan_destroy", plan), ("fmmb_cache_destroy", cache), ("fmmb_ctx_destroy", ctx)):
            if not ((order == "ctx_first" and name == "fmmb_ctx_destroy") or (order == "plan_first" and name == "fmmb_plan_destroy")
                    or (order == "cache_first" and name == "fmmb_cache_destroy")):
                assert getattr(L, name)(h) == 0


def test_dev_entry_points_reject_host_pointers(fmmb):
    """A plain host array handed to a _dev entry point is an ArgumentError raised before any
    launch (the library checks every pointer's attributes), not a device fault."""
    import ctypes as C
    import torch
    from cuda.bindings import runtime as cudart
    rng = np.random.default_rng(61)
    pts = rng.random((4000, 3))
    tau = rng.standard_normal(4000)
    host = np.zeros(3 * 4000)
    err, attr = cudart.cudaPointerGetAttributes(host.ctypes.data)
    if err != cudart.cudaError_t.cudaSuccess or attr.type != cudart.cudaMemoryType.cudaMemoryTypeUnregistered:
        pytest.skip("plain host memory is device-accessible here")
    L = fmmb.lib()
    f = fmmb.FMM(_method(fmmb, 6), pts, ppl=40, bbox=BOX)
    st = fmmb.FMMState(f)
    x_d = torch.from_numpy(pts).cuda()
    t_d = torch.from_numpy(tau).cuda()
    u_d = torch.zeros(4000, dtype=torch.float64, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    H = C.c_void_p(host.ctypes.data)
    assert L.fmmb_build_expansions_dev(st._h, H, P(t_d), 4000) == 1
    assert L.fmmb_build_expansions_dev(st._h, P(x_d), H, 4000) == 1
    assert b"device pointers" in L.fmmb_last_error()
    assert L.fmmb_matvec_dev(st._h, P(x_d), P(t_d), 4000, 1, H, None) == 1
    assert L.fmmb_evaluate_dev(st._h, H, 10, 1, P(u_d), None) == 1
    assert L.fmmb_direct_dev(fmmb.default_context()._h, H, P(t_d), 4000, P(x_d), None, 10, P(u_d), None) == 1
    # the state is still usable and correct afterwards
    assert L.fmmb_matvec_dev(st._h, P(x_d), P(t_d), 4000, 1, P(u_d), None) == 0
    ref = fmmb.evaluate_at_sources(f, fmmb.build_expansions(f, pts, tau))
    assert np.array_equal(u_d.cpu().numpy(), ref)
