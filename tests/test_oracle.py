"""Pins the CPU oracle to the reference's own known-answer tests and tolerances (CPU only).

The reference (Julia) cannot run here, so the oracle is pinned by restating its tests:
  test/test_harmonics.jl:17-67    Hobson values at x = (0.3, -0.5, 0.4) and the identities
  test/test_harmonics.jl:69-92    the Schmidt recurrences against the Hobson values
  test/test_harmonics.jl:109-115  convergence in p
  test/test_harmonics.jl:129-152  FMM end to end vs direct sums (p = 16, 6000 points)
  test/test_harmonics.jl:235-293  34 classes, orbit sizes, classes reproduce every offset
  test/test_tree.jl:7-131         the tree invariants, edge cases and guards
and against analytic golden values committed in tests/golden/.
"""
import json
import math
import os

import numpy as np
import pytest

from helpers import DISTRIBUTIONS3, check_tree_invariants, mrd, oracle_tree_dict

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def cidx(n, m):
    return n * n + n + m


def test_hobson_values(oracle):
    x = np.array([0.3, -0.5, 0.4])
    r = np.linalg.norm(x)
    p = 7
    Y = oracle.regular_hobson(x, p)
    T = oracle.irregular_hobson(x, p)
    xy = complex(x[0], x[1])
    assert Y[cidx(0, 0)] == 1
    assert np.isclose(Y[cidx(1, 0)], x[2]) and np.isclose(Y[cidx(1, 1)], -xy / 2)
    assert np.isclose(Y[cidx(2, 2)], xy ** 2 / 8)
    assert np.isclose(Y[cidx(2, 0)], (3 * x[2] ** 2 - r ** 2) / 4) and np.isclose(Y[cidx(2, 1)], -x[2] * xy / 2)
    assert np.isclose(T[cidx(0, 0)], 1 / r) and np.isclose(T[cidx(1, 0)], x[2] / r ** 3)
    assert np.isclose(T[cidx(1, 1)], -xy / r ** 3)
    for n in range(p + 1):
        for m in range(-n, n + 1):
            f = math.factorial(n - abs(m)) * math.factorial(n + abs(m))
            assert np.isclose(T[cidx(n, m)], f * Y[cidx(n, m)] / r ** (2 * n + 1), rtol=1e-12, atol=0)
            if m > 0:
                assert Y[cidx(n, -m)] == (-1) ** m * np.conj(Y[cidx(n, m)])
                assert T[cidx(n, -m)] == (-1) ** m * np.conj(T[cidx(n, m)])


def test_hobson_identities(oracle):
    x = np.array([0.3, -0.5, 0.4])
    # harmonic: the Laplacian vanishes (finite differences in place of automatic differentiation)
    h = 1e-3
    for n in range(6):
        for m in range(n + 1):
            for f in (oracle.regular_hobson, oracle.irregular_hobson):
                lap = -6 * f(x, 6)[cidx(n, m)]
                for d in range(3):
                    e = np.zeros(3)
                    e[d] = h
                    lap += f(x + e, 6)[cidx(n, m)] + f(x - e, 6)[cidx(n, m)]
                assert abs(lap / h ** 2) < 1e-4 * (1 + abs(f(x, 6)[cidx(n, m)]) * 1e3)
    # 1/|x − y| = Σ conj Υ(y) Θ(x), |y| < |x|
    y = np.array([0.1, 0.05, -0.08])
    s = np.sum(np.conj(oracle.regular_hobson(y, 30)) * oracle.irregular_hobson(x, 30))
    assert abs(s - 1 / np.linalg.norm(x - y)) < 1e-13 / np.linalg.norm(x - y)
    # the regular addition theorem
    p = 7
    a, b = np.array([0.2, 0.1, -0.3]), np.array([-0.1, 0.4, 0.2])
    Ya, Yb, Yab = oracle.regular_hobson(a, p), oracle.regular_hobson(b, p), oracle.regular_hobson(a + b, p)
    for n in range(p + 1):
        for m in range(-n, n + 1):
            acc = 0j
            for k in range(n + 1):
                for l in range(-k, k + 1):
                    if abs(m - l) <= n - k:
                        acc += Ya[cidx(k, l)] * Yb[cidx(n - k, m - l)]
            assert abs(acc - Yab[cidx(n, m)]) < 1e-15
    # Θ_n^m(a + b) = Σ (−1)^k conj Υ_k^l(b) Θ_{n+k}^{m+l}(a), |b| < |a|
    a, b, q = np.array([1.5, -0.8, 1.1]), np.array([0.1, 0.2, -0.15]), 40
    Ta, Yb, Tab = oracle.irregular_hobson(a, q), oracle.regular_hobson(b, q), oracle.irregular_hobson(a + b, 3)
    for n in range(4):
        for m in range(-n, n + 1):
            acc = 0j
            for k in range(q - n + 1):
                for l in range(-k, k + 1):
                    acc += (-1) ** k * np.conj(Yb[cidx(k, l)]) * Ta[cidx(n + k, m + l)]
            assert abs(acc - Tab[cidx(n, m)]) <= 1e-12 * abs(Tab[cidx(n, m)])
    # the derivative identities, by central differences
    Y = oracle.regular_hobson(x, p)
    at = lambda k, m: Y[cidx(k, m)] if abs(m) <= k else 0j
    h = 1e-6
    for n in range(1, p + 1):
        for m in range(-n, n + 1):
            g = []
            for d in range(3):
                e = np.zeros(3)
                e[d] = h
                g.append((oracle.regular_hobson(x + e, p)[cidx(n, m)] - oracle.regular_hobson(x - e, p)[cidx(n, m)]) / (2 * h))
            assert abs(g[2] - at(n - 1, m)) < 1e-8
            assert abs(g[0] - 1j * g[1] + at(n - 1, m - 1)) < 1e-8
            assert abs(g[0] + 1j * g[1] - at(n - 1, m + 1)) < 1e-8


def test_schmidt_recurrences(oracle):
    p = 9
    x = np.array([0.25, -0.4, 0.35])
    s = oracle.scaling_factors(p)
    Y = oracle.regular_hobson(x, p)
    v = oracle.fold_regular(x, p)
    for n in range(p + 1):
        for m in range(n + 1):
            assert np.isclose(v[cidx(n, m)], s[cidx(n, m)] * Y[cidx(n, m)], rtol=1e-13, atol=0)
            assert abs(v[cidx(n, m)]) <= np.linalg.norm(x) ** n * (1 + 1e-12)


def test_symmetry_classes(oracle):
    sc = oracle.harmonic_classes(6)
    assert len(sc["reps"]) == 34
    sizes = sorted(np.bincount(sc["cls"], minlength=34).tolist())
    assert sizes == sorted([16] * 9 + [8] * 19 + [4] * 4 + [2] * 2)
    for f in (0, 49, 199, 315):
        assert sorted(sc["idx"][f]) == list(range(49)) and sorted(sc["idx_t"][f]) == list(range(49))


@pytest.mark.parametrize("p", [6, 16])
def test_classes_reproduce_every_offset(oracle, p):
    """check_harmonic_classes (src/operators/harmonics.jl:653-671): < 1e-13."""
    sc = oracle.harmonic_classes(p)
    offs = oracle.far_offsets()
    reps = [oracle.harmonic_m2l(r, p, 1.0) for r in sc["reps"]]
    worst = 0.0
    for f in range(316):
        M = oracle.harmonic_m2l(offs[f], p, 1.0)
        R = reps[sc["cls"][f]]
        B = np.zeros_like(M)
        it, st, is_, ss = sc["idx_t"][f], sc["sgn_t"][f], sc["idx"][f], sc["sgn"][f]
        B[np.ix_(it, is_)] = st[:, None] * ss[None, :] * R
        worst = max(worst, np.max(np.abs(M - B)) / np.max(np.abs(M)))
    assert worst < 1e-13


def test_convergence_in_p(oracle):
    """test/test_harmonics.jl:109-115 in the form of the FMM error vs direct sums."""
    rng = np.random.default_rng(3)
    pts = rng.random((4000, 3))
    tau = rng.standard_normal(4000)
    du, _ = oracle.direct(pts, tau)
    errs = []
    for p in (4, 8, 12, 16):
        f = oracle.FMM(p, pts, 40)
        f.build_expansions(pts, tau)
        errs.append(mrd(f.evaluate_at_sources()[0], du))
    assert errs[0] > 5 * errs[1] > 25 * errs[2] and errs[3] < 1e-5


@pytest.mark.parametrize("name", list(DISTRIBUTIONS3))
def test_fmm_end_to_end(oracle, name):
    rng = np.random.default_rng(hash(name) % 1000)
    pts = DISTRIBUTIONS3[name](rng, 6000)
    tau = rng.standard_normal(6000)
    tg = rng.random((500, 3))
    f = oracle.FMM(16, pts, 40)
    f.build_expansions(pts, tau)
    u, g = f.evaluate_at_sources()
    du, dg = oracle.direct(pts, tau)
    tu, tgr = f.evaluate(tg)
    dtu, dtg = oracle.direct(pts, tau, tg)
    assert mrd(u, du) < 1e-5
    assert mrd(tu, dtu) < 1e-5
    assert mrd(tgr, dtg) < 1e-4
    assert mrd(g, dg) < 1e-4


@pytest.mark.parametrize("name,n,ppl", [("uniform", 1500, 10), ("mixed", 2000, 8), ("sphere", 2000, 20), ("helix", 1500, 12),
                                        ("one_octant", 800, 5), ("clustered", 1500, 10)])
def test_tree_invariants(oracle, name, n, ppl):
    rng = np.random.default_rng(n + ppl)
    pts = DISTRIBUTIONS3[name](rng, n)
    T = oracle.Tree.build(pts, ppl)
    check_tree_invariants(oracle_tree_dict(T), pts)


def test_tree_edge_cases(oracle):
    rng = np.random.default_rng(5)
    pts = rng.random((10, 3))
    T = oracle.Tree.build(pts, 10)
    assert T.L == 1 and T.n == 1 and np.all(T.point_node == 0)
    # two levels: eight octant clusters of ppl points each
    ppl = 6
    c = np.array([[0.25 + 0.5 * ((k >> d) & 1) for d in range(3)] for k in range(8)])
    pts = np.repeat(c, ppl, axis=0) + 0.01 * rng.standard_normal((8 * ppl, 3))
    T = oracle.Tree.build(pts, ppl)
    assert T.L == 2 and T.n == 9 and T.ghost.sum() == 0
    # one octant: sparse levels, restriction refines the empty octants
    pts = 0.5 * rng.random((500, 3))
    T = oracle.Tree.build(pts, 5)
    check_tree_invariants(oracle_tree_dict(T), pts)
    lv1 = np.nonzero(T.level == 1)[0]
    assert len(lv1) == 8 and T.has_source[lv1].sum() == 1
    with pytest.raises(oracle.OracleError, match="max_levels"):
        oracle.Tree.build(np.full((20, 3), 0.3), 5, max_levels=10)
    with pytest.raises(oracle.OracleError):
        oracle.Tree.build(pts, 0)
    with pytest.raises(oracle.OracleError, match="outside"):
        oracle.Tree.build(pts, 5, origin=(0.3, 0.3, 0.3))
    # points on the box faces and corners are accepted and located
    pts = np.vstack([rng.random((200, 3)), [[0, 0, 0], [1, 1, 1], [1, 0, 0.5], [0.5, 0.5, 0.0]]])
    T = oracle.Tree.build(pts, 5)
    check_tree_invariants(oracle_tree_dict(T), pts)


def test_golden_analytic_values(oracle):
    """tests/golden/hobson.json: closed forms of Υ and Θ (make_golden.py) against the oracle."""
    g = json.load(open(os.path.join(GOLDEN, "hobson.json")))
    for case in g["cases"]:
        x = np.array(case["x"])
        Y = oracle.regular_hobson(x, 2)
        T = oracle.irregular_hobson(x, 2)
        for key, val in case["regular"].items():
            n, m = map(int, key.split(","))
            assert abs(Y[cidx(n, m)] - complex(*val)) < 1e-14
        for key, val in case["irregular"].items():
            n, m = map(int, key.split(","))
            assert abs(T[cidx(n, m)] - complex(*val)) < 1e-13 * abs(complex(*val))


def test_golden_direct_sums(oracle):
    """tests/golden/direct_small.npz: numpy FP64 direct sums against the oracle's."""
    d = np.load(os.path.join(GOLDEN, "direct_small.npz"))
    u, g = oracle.direct(d["points"], d["tau"])
    assert mrd(u, d["pot"]) < 1e-14 and mrd(g, d["grad"]) < 1e-13
    f = oracle.FMM(16, d["points"], 20)
    f.build_expansions(d["points"], d["tau"])
    fu, fg = f.evaluate_at_sources()
    assert mrd(fu, d["pot"]) < 1e-5 and mrd(fg, d["grad"]) < 1e-4
