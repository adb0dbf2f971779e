"""The kernel-free coverage invariant on the oracle's tree (CPU), restating
test/test_coverage.jl:86-96: every (source terminal, target leaf) pair covered exactly once,
the far pairs exactly the V lists, offsets and levels consistent."""
import numpy as np
import pytest

from helpers import DISTRIBUTIONS3, check_coverage, oracle_tree_dict


def _pairs(T):
    return [T.pairs(l) for l in range(T.L)]


@pytest.mark.parametrize("name", sorted(DISTRIBUTIONS3))
def test_coverage_oracle_tree(oracle, name):
    rng = np.random.default_rng(4)
    pts = DISTRIBUTIONS3[name](rng, 400)
    T = oracle.Tree.build(pts, 4)
    check_coverage(oracle_tree_dict(T), _pairs(T), oracle.far_offsets())


def test_coverage_small_ppl_many_ghosts(oracle):
    rng = np.random.default_rng(5)
    T = oracle.Tree.build(DISTRIBUTIONS3["mixed"](rng, 800), 3)
    assert T.ghost.sum() > 0
    check_coverage(oracle_tree_dict(T), _pairs(T), oracle.far_offsets())
    T = oracle.Tree.build(DISTRIBUTIONS3["uniform"](rng, 12), 12)
    check_coverage(oracle_tree_dict(T), _pairs(T), oracle.far_offsets())


def test_coverage_detects_a_missing_pair(oracle):
    """The check itself: drop one far pair (a planted mistake in the oracle's lists) and it fails."""
    rng = np.random.default_rng(6)
    T = oracle.Tree.build(DISTRIBUTIONS3["uniform"](rng, 2000), 8)
    pairs = _pairs(T)
    l = max(range(T.L), key=lambda k: len(pairs[k][0]))
    pairs[l] = tuple(x[1:] for x in pairs[l])
    with pytest.raises(AssertionError):
        check_coverage(oracle_tree_dict(T), pairs, oracle.far_offsets())
