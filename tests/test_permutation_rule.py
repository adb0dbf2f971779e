"""The tensor-core M2L computes the D4h signed permutations of each far offset from the
offset's group element (rotation k, εy, εz) instead of reading tables. This restates that
rule (m2l_tc.cu: coef_nmp, perm_sign) and checks it against the oracle's tables for every
far offset and entry (src/operators/symmetry.jl:252-319)."""
import numpy as np
import pytest


def coef_nmp(k):
    n = int(np.floor(np.sqrt(k + 0.5)))
    while n * n > k:
        n -= 1
    while (n + 1) ** 2 <= k:
        n += 1
    r = k - n * n
    return n, (r + 1) >> 1, 0 if r == 0 else (1 if r & 1 else 2)


def perm_sign(part, q, npm, fac):
    s = -1 if (fac & 8) and (npm & 1) else 1
    if part == 0:
        return s
    if part == 1:
        return s if q < 2 else -s
    sig = -1 if fac & 4 else 1
    return s * sig if q in (0, 3) else -s * sig


def d4h_factors(offs):
    """k | εy << 2 | εz << 3 of the first D4h element mapping the class representative to each offset."""
    G = []
    for perm in ((0, 1, 2), (1, 0, 2)):
        for sb in range(8):
            G.append((perm, tuple(-1 if (sb >> d) & 1 else 1 for d in range(3))))
    rots = ([[1, 0], [0, 1]], [[0, -1], [1, 0]], [[-1, 0], [0, -1]], [[0, 1], [-1, 0]])
    out = []
    for o in offs:
        a, b = abs(o[0]), abs(o[1])
        r = (max(a, b), min(a, b), abs(o[2]))
        perm, sign = next(g for g in G if all(g[1][k] * r[g[0][k]] == o[k] for k in range(3)))
        ez = sign[2] == -1
        A = [[0, 0], [0, 0]]
        A[0][perm[0]] = sign[0]
        A[1][perm[1]] = sign[1]
        ey = A[0][0] * A[1][1] - A[0][1] * A[1][0] == -1
        if ey:
            A[0][1], A[1][1] = -A[0][1], -A[1][1]
        k = rots.index(A)
        out.append(k | (4 if ey else 0) | (8 if ez else 0))
    return out


@pytest.mark.parametrize("p", [4, 10])
def test_rule_reproduces_the_tables(oracle, p):
    sc = oracle.harmonic_classes(p)
    fac = d4h_factors(oracle.far_offsets())
    N = (p + 1) ** 2
    for f in range(316):
        for i in range(N):
            n, m, part = coef_nmp(i)
            partner = i if part == 0 else (i + 1 if part == 1 else i - 1)
            # source side: G[i] = sgn[i] M[idx[i]]
            q = (-m * (fac[f] & 3)) & 3
            sw = part != 0 and (q & 1)
            assert sc["idx"][f][i] == (partner if sw else i)
            assert sc["sgn"][f][i] == perm_sign(part, q, n + m, fac[f])
            # target side: L[j] += sgn_t[i] Y[i] with idx_t[i] = j
            q = (m * (fac[f] & 3)) & 3
            sw = part != 0 and (q & 1)
            src = partner if sw else i
            ipart = (3 - part) if sw else part
            assert sc["idx_t"][f][src] == i
            assert sc["sgn_t"][f][src] == perm_sign(ipart, q, n + m, fac[f])
