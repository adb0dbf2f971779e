"""The mixed path (FP32 P2M, tensor-core FP16x3 M2L with power-of-two scaling, FP32 compensated
near field and L2P) against the FP64 path and FP64 direct sums. Tolerances: the multipoles within
1e-6 and the locals within 2e-6 (max-norm relative) of the FP64 path's; potentials within 1e-6
relative L2 of the FP64 path and of FP64 direct sums beyond the truncation error (the metric's
target), gradients within 1e-5."""
import numpy as np
import pytest

from helpers import DISTRIBUTIONS3, mrd, rel_l2

pytestmark = pytest.mark.gpu
BOX = ((0.0, 0.0, 0.0), 1.0)


@pytest.mark.parametrize("name,n,ppl,seed,p", [("uniform", 60000, 64, 1, 10), ("mixed", 20000, 40, 2, 10),
                                               ("sphere", 20000, 40, 3, 10), ("clustered", 15000, 30, 4, 10),
                                               ("uniform", 60000, 64, 5, 11), ("mixed", 20000, 40, 6, 11),
                                               ("helix", 20000, 40, 7, 9), ("one_octant", 20000, 40, 8, 7)])
def test_mixed_locals_match_fp64(fmmb, name, n, ppl, seed, p):
    rng = np.random.default_rng(seed)
    pts = DISTRIBUTIONS3[name](rng, n)
    tau = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=p), pts, ppl=ppl, bbox=BOX)
    s64 = fmmb.build_expansions(f, pts, tau, precision="fp64")
    s32 = fmmb.build_expansions(f, pts, tau, precision="mixed")
    M64, L64 = s64.expansions()
    M32, L32 = s32.expansions()
    # P2M in FP32 (box-centred coordinates) on the mixed path, M2M in FP64 on both
    assert np.max(np.abs(M32 - M64)) < 1e-6 * np.max(np.abs(M64))
    assert np.max(np.abs(L32 - L64)) < 2e-6 * np.max(np.abs(L64))
    u64, g64 = fmmb.evaluate_at_sources_both(f, s64)
    u32, g32 = fmmb.evaluate_at_sources_both(f, s32)
    assert rel_l2(u32, u64) < 1e-6
    assert rel_l2(g32, g64) < 1e-5


def test_mixed_accuracy_vs_direct(oracle, fmmb):
    rng = np.random.default_rng(9)
    n = 100000
    pts = rng.random((n, 3))
    tau = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=10), pts, ppl=64, bbox=BOX)
    st = fmmb.build_expansions(f, pts, tau, precision="mixed")
    s64 = fmmb.build_expansions(f, pts, tau, precision="fp64")
    u, g = fmmb.evaluate_at_sources_both(f, st)
    u64, g64 = fmmb.evaluate_at_sources_both(f, s64)
    sel = np.sort(rng.choice(n, 512, replace=False))
    du, dg = oracle.direct_sample(pts, tau, sel)
    # the p = 10 truncation error dominates: the mixed path adds at most 1e-6 relative L2
    e64, e32 = rel_l2(u64[sel], du), rel_l2(u[sel], du)
    assert e64 < 1e-5 and e32 < e64 + 1e-6
    assert rel_l2(g[sel], dg) < rel_l2(g64[sel], dg) + 1e-5
    tg = rng.random((300, 3))
    tu, tgr = oracle.direct(pts, tau, tg)
    assert rel_l2(fmmb.evaluate(f, st, tg), tu) < rel_l2(fmmb.evaluate(f, s64, tg), tu) + 1e-6
    assert rel_l2(fmmb.evaluate(f, st, tg, output=fmmb.Gradient()), tgr) < 1e-4


def test_mixed_deterministic_and_recovers(fmmb):
    rng = np.random.default_rng(10)
    pts = DISTRIBUTIONS3["mixed"](rng, 20000)
    tau = rng.standard_normal(20000)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=8), pts, ppl=40, bbox=BOX)
    st = fmmb.FMMState(f, "mixed")
    u0 = fmmb.device_matvec(f, st, pts, tau)
    bad = tau.copy()
    bad[3] = np.inf
    assert not np.all(np.isfinite(fmmb.device_matvec(f, st, pts, bad)))
    assert np.array_equal(fmmb.device_matvec(f, st, pts, tau), u0)
    assert np.array_equal(fmmb.device_matvec(f, fmmb.FMMState(f, "mixed"), pts, tau), u0)


def test_mixed_supported_orders(fmmb):
    rng = np.random.default_rng(12)
    pts = rng.random((5000, 3))
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=12), pts, ppl=40, bbox=BOX)
    with pytest.raises(fmmb.Unsupported):
        fmmb.FMMState(f, "mixed")
    for p in (1, 2, 3, 4, 5, 6, 8, 11):
        tau = rng.standard_normal(5000)
        g = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=p), pts, ppl=40, bbox=BOX)
        u32 = fmmb.evaluate_at_sources(g, fmmb.build_expansions(g, pts, tau, precision="mixed"))
        u64 = fmmb.evaluate_at_sources(g, fmmb.build_expansions(g, pts, tau, precision="fp64"))
        assert rel_l2(u32, u64) < 1e-6


@pytest.mark.parametrize("kernel,precision", [("laplace", "mixed"), ("laplace", "fp64"), ("yukawa", "fp64")])
def test_matvec_equals_build_then_evaluate(fmmb, kernel, precision):
    """fmmb_matvec runs the near field on a side stream beside the upward and downward passes and
    adds the far field after both; its outputs equal build_expansions + evaluate_at_sources bit
    for bit (one addition, in either order), for one and both outputs, and over repeated calls."""
    rng = np.random.default_rng(21)
    n = 60000
    pts = DISTRIBUTIONS3["mixed"](rng, n)
    tau = rng.standard_normal(n)
    k = fmmb.Laplace3D() if kernel == "laplace" else fmmb.Yukawa3D(3.0)
    f = fmmb.FMM(fmmb.SphericalHarmonics(k, p=8), pts, ppl=40, bbox=BOX)
    st = fmmb.build_expansions(f, pts, tau, precision=precision)
    u_ref, g_ref = fmmb.evaluate_at_sources_both(f, st)
    L = fmmb.lib()
    for _ in range(2):
        pot, grad = np.zeros(n), np.zeros((n, 3))
        fmmb._check(L.fmmb_matvec(st._h, fmmb._ptr(pts), fmmb._ptr(tau), n, 3, fmmb._ptr(pot), fmmb._ptr(grad)))
        assert np.array_equal(pot, u_ref)
        assert np.array_equal(fmmb._grad_out(f, grad), g_ref)
    pot = np.zeros(n)
    fmmb._check(L.fmmb_matvec(st._h, fmmb._ptr(pts), fmmb._ptr(tau), n, 1, fmmb._ptr(pot), None))
    assert np.array_equal(pot, u_ref)


def test_bounded_wait_gives_up_and_recovers(fmmb):
    """The tensor-core M2L's waits are bounded: with the test hook one K-step slab of every block
    is never reported gathered, so the MMA issuer's wait runs out (20 ms here), every role gives
    up, the kernel frees its tensor memory and returns, and the call reports a timeout; the same
    state then recomputes the same result. No fault, trap or endless wait is involved."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(31)
    n = 30000
    pts = rng.random((n, 3))
    tau = rng.standard_normal(n)
    f = fmmb.FMM(fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=10), pts, ppl=64, bbox=BOX)
    st = fmmb.FMMState(f, "mixed")
    u0 = fmmb.device_matvec(f, st, pts, tau)
    L = fmmb.lib()
    try:
        fmmb._test_m2l_stall(3, 0.02)
        with pytest.raises(fmmb.FMMBError) as e:                       # host-pointer call: reported at once
            fmmb.device_matvec(f, st, pts, tau)
        assert e.value.code == 5
        # device-pointer call: enqueued without error, reported at the state's synchronisation
        P = lambda t: C.c_void_p(t.data_ptr())
        xd, td = torch.from_numpy(pts).cuda(), torch.from_numpy(tau).cuda()
        pd, gd = torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        fmmb._check(L.fmmb_matvec_dev(st._h, P(xd), P(td), n, 3, P(pd), P(gd)))
        with pytest.raises(fmmb.FMMBError) as e:
            st.synchronize()
        assert e.value.code == 5
        st.synchronize()                                               # reported once
    finally:
        fmmb._test_m2l_stall(-1)
    assert np.array_equal(fmmb.device_matvec(f, st, pts, tau), u0)
    fmmb._check(L.fmmb_matvec_dev(st._h, P(xd), P(td), n, 1, P(pd), None))
    st.synchronize()
    assert np.array_equal(pd.cpu().numpy(), u0)
