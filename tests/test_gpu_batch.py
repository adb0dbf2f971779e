"""Batch plans (fmmb_batch_plan_create): several independent FMMs in one forest. Each instance's
tree, far pairs and outputs must be bitwise those of its own plan, built with the same operator
cache after the plans of the instances before it (the batch fits its boxes in that order). The
single-instance plans are themselves pinned to the oracle by the other device tests."""
import numpy as np
import pytest

from helpers import clustered3, mixed3, sphere3, stokes_direct, uniform3

pytestmark = pytest.mark.gpu

TREE_KEYS = ("cell", "parent", "child_first", "plo", "phi", "leaf", "ghost", "xlist", "has_source", "colleagues")


def instance_sets(rng):
    """Uneven point sets in boxes of different sizes and places: the batch's roots then sit on
    different global levels."""
    return [
        uniform3(rng, 9000),
        0.25 + 0.5 * clustered3(rng, 4000),            # a smaller box: its root one level down
        sphere3(rng, 12000),
        3.0 + 2.0 * uniform3(rng, 2500),               # a larger box elsewhere: the widest root
        mixed3(rng, 7000),
        0.5 + 0.01 * uniform3(rng, 25),                # one leaf: a root with no children
    ]


def instance_tree(bt, i, rl):
    """Instance i's nodes of the batch tree, renumbered in batch order (level by level), with
    levels relative to its root and point ranges relative to its first point."""
    t = bt["tree"]
    nodes = np.nonzero(bt["node_instance"] == i)[0]
    loc = -np.ones(len(bt["node_instance"]), np.int64)
    loc[nodes] = np.arange(len(nodes))
    off = bt["offsets"][i]
    out = {"level": t["level"][nodes] - rl}
    for k in ("cell", "leaf", "ghost", "xlist", "has_source"):
        out[k] = t[k][nodes]
    for k in ("parent", "child_first"):
        v = t[k][nodes]
        out[k] = np.where(v >= 0, loc[np.maximum(v, 0)], -1)
    col = t["colleagues"][nodes]
    out["colleagues"] = np.where(col >= 0, loc[np.maximum(col, 0)], -1)
    has = out["has_source"].astype(bool)
    out["plo"] = np.where(has, t["plo"][nodes] - off, 0)
    out["phi"] = np.where(has, t["phi"][nodes] - off, -1)
    a, b = bt["offsets"][i], bt["offsets"][i + 1]
    out["perm"] = t["perm"][a:b] - off
    return out, loc


def single_tree(f):
    t = f.tree()
    has = t["has_source"].astype(bool)
    t["plo"] = np.where(has, t["plo"], 0)
    t["phi"] = np.where(has, t["phi"], -1)
    return t


def batch_and_singles(fmmb, method, sets, ppl, bbox=None):
    bf = fmmb.BatchFMM(method, sets, ppl=ppl, bbox=bbox)
    cache = fmmb.OperatorCache(method)
    singles = [fmmb.FMM(method, x, ppl=ppl, cache=cache, bbox=None if bbox is None else bbox) for x in sets]
    return bf, singles


def test_batch_trees_and_pairs_equal_single_plans(fmmb):
    rng = np.random.default_rng(70)
    sets = instance_sets(rng)
    m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=6)
    bf, singles = batch_and_singles(fmmb, m, sets, 32)
    assert len(set(bf.root_level.tolist())) >= 3              # roots on different global levels
    bt = {"tree": bf.tree(), "node_instance": bf.node_instance, "offsets": bf.offsets}
    for i, f in enumerate(singles):
        np.testing.assert_array_equal(bf.boxes[i], [*f.origin, f.width])
        rl = bf.root_level[i]
        got, loc = instance_tree(bt, i, rl)
        ref = single_tree(f)
        assert len(got["level"]) == f.nnodes
        np.testing.assert_array_equal(got["level"], ref["level"])
        for k in TREE_KEYS:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"instance {i}: {k}")
        np.testing.assert_array_equal(got["perm"], ref["perm"])
        # far pairs: the batch's of this instance's nodes, per relative level, equal the plan's
        for l in range(2, f.nlevels):
            t, s, fa = bf.pairs(l + rl)
            sel = bf.node_instance[t] == i
            a = np.stack([loc[t[sel]], loc[s[sel]], fa[sel]], 1)
            b = np.stack(f.pairs(l), 1)
            a = a[np.lexsort(a.T[::-1])]
            b = b[np.lexsort(b.T[::-1])]
            np.testing.assert_array_equal(a, b, err_msg=f"instance {i} level {l}")
    assert bf.N == sum(len(x) for x in sets) and bf.ninst == len(sets)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_laplace_outputs_bitwise_equal(fmmb, precision):
    rng = np.random.default_rng(71)
    sets = instance_sets(rng)
    taus = [rng.standard_normal(len(x)) for x in sets]
    m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=8)
    bf, singles = batch_and_singles(fmmb, m, sets, 40)
    st = fmmb.build_expansions(bf, bf.sources, bf.concat(taus), precision=precision)
    u, g = fmmb.evaluate_at_sources_both(bf, st)
    for i, (f, x, t) in enumerate(zip(singles, sets, taus)):
        s1 = fmmb.build_expansions(f, x, t, precision=precision)
        u1, g1 = fmmb.evaluate_at_sources_both(f, s1)
        np.testing.assert_array_equal(bf.split(u)[i], u1, err_msg=f"instance {i}")
        np.testing.assert_array_equal(bf.split(g)[i], g1, err_msg=f"instance {i}")
    # the same through the one-call matvec
    u2 = fmmb.device_matvec(bf, fmmb.FMMState(bf, precision), bf.sources, bf.concat(taus))
    np.testing.assert_array_equal(u2, u)


def test_batch_yukawa_outputs_bitwise_equal(fmmb):
    rng = np.random.default_rng(72)
    sets = instance_sets(rng)[:4]
    taus = [rng.standard_normal(len(x)) for x in sets]
    m = fmmb.SphericalHarmonics(fmmb.Yukawa3D(5.0), p=8)
    bf, singles = batch_and_singles(fmmb, m, sets, 40)
    st = fmmb.build_expansions(bf, bf.sources, bf.concat(taus))
    u, g = fmmb.evaluate_at_sources_both(bf, st)
    for i, (f, x, t) in enumerate(zip(singles, sets, taus)):
        u1, g1 = fmmb.evaluate_at_sources_both(f, fmmb.build_expansions(f, x, t))
        np.testing.assert_array_equal(bf.split(u)[i], u1, err_msg=f"instance {i}")
        np.testing.assert_array_equal(bf.split(g)[i], g1, err_msg=f"instance {i}")


def test_batch_stokes_velocities_bitwise_equal_and_accurate(fmmb):
    """The batched Stokes form: jittered unit-sphere point sets of uneven sizes in one common box,
    Stokeslets N(0,1); each instance's velocities bitwise those of its own StokesFMMPlan, and within
    1e-4 relative L2 of FP64 direct sums (p = 10 with ppl = 100 gives about 1e-5)."""
    rng = np.random.default_rng(73)
    sizes = [3000, 11000, 6000, 20000, 4500]
    sets, forces = [], []
    for n in sizes:
        v = rng.standard_normal((n, 3))
        sets.append(v / np.linalg.norm(v, axis=1)[:, None] + rng.uniform(-0.01, 0.01, (n, 3)))
        forces.append(rng.standard_normal((n, 3)))
    box = ((-1.02, -1.02, -1.02), 2.04)
    bp = fmmb.BatchStokesFMMPlan(sets, p=10, ppl=100, bbox=box)
    vel = fmmb.stokes_fmm_eval(bp, stokeslets=bp.fmm.concat(forces))
    for i, (x, f) in enumerate(zip(sets, forces)):
        sp = fmmb.StokesFMMPlan(x, p=10, ppl=100, bbox=box)
        v1 = fmmb.stokes_fmm_eval(sp, stokeslets=f)
        vi = bp.fmm.split(vel)[i]
        np.testing.assert_array_equal(vi, v1, err_msg=f"instance {i}")
        sel = np.sort(rng.choice(len(x), 40, replace=False))
        ud = stokes_direct(x, f, sel)
        assert np.linalg.norm(vi[sel] - ud) / np.linalg.norm(ud) < 1e-4


def test_batch_of_one_equals_plain_plan(fmmb):
    rng = np.random.default_rng(74)
    x = clustered3(rng, 20000)
    tau = rng.standard_normal(len(x))
    m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=8)
    bf = fmmb.BatchFMM(m, [x], ppl=50)
    f = fmmb.FMM(m, x, ppl=50)
    assert bf.nnodes == f.nnodes and bf.ninst == 1
    for prec in ("fp64", "mixed"):
        u = fmmb.evaluate_at_sources(bf, fmmb.build_expansions(bf, x, tau, precision=prec))
        u1 = fmmb.evaluate_at_sources(f, fmmb.build_expansions(f, x, tau, precision=prec))
        np.testing.assert_array_equal(u, u1)


def test_batch_errors(fmmb):
    rng = np.random.default_rng(75)
    m = fmmb.SphericalHarmonics(fmmb.Laplace3D(), p=6)
    with pytest.raises(fmmb.ArgumentError):
        fmmb.BatchFMM(m, [uniform3(rng, 100), np.zeros((0, 3))])
    with pytest.raises(fmmb.ArgumentError):
        fmmb.BatchFMM(m, [uniform3(rng, 100), np.full((5, 3), np.nan)])
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.BatchFMM(m, [uniform3(rng, 100), uniform3(rng, 100)], bbox=[((0, 0, 0), 1.0)])
    with pytest.raises(fmmb.ArgumentError):                   # points outside the given box
        fmmb.BatchFMM(m, [uniform3(rng, 100), 2 + uniform3(rng, 100)], bbox=((0, 0, 0), 1.0))
    with pytest.raises(fmmb.Unsupported):
        fmmb.BatchFMM(fmmb.CubeKernelIndependent(fmmb.Laplace3D(), p=4), [uniform3(rng, 500)])
    bf = fmmb.BatchFMM(m, [uniform3(rng, 3000), uniform3(rng, 2000)], ppl=32)
    st = fmmb.build_expansions(bf, bf.sources, rng.standard_normal(bf.N))
    with pytest.raises(fmmb.Unsupported):
        fmmb.evaluate(bf, st, uniform3(rng, 10))
    with pytest.raises(fmmb.DimensionMismatch):
        bf.concat([np.zeros(3000)])
