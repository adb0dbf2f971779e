"""Point distributions and structural checks for the tests, restating the reference's
test utilities (test/testutils.jl:1-76) and tree invariants (test/test_tree.jl:7-131)."""
import numpy as np

# ---------------------------------------------------------------- distributions (test/testutils.jl:50-76)
def uniform3(rng, n):
    return rng.random((n, 3))


def clustered3(rng, n, nclusters=10, spread=0.01):
    c = 0.1 + 0.8 * rng.random((nclusters, 3))
    x = c[np.arange(n) % nclusters] + spread * rng.standard_normal((n, 3))
    return np.clip(x, 0.0, 1.0)


def sphere3(rng, n, center=(0.5, 0.5, 0.5), radius=0.4):
    v = rng.standard_normal((n, 3))
    return np.asarray(center) + radius * v / np.linalg.norm(v, axis=1)[:, None]


def helix3(rng, n):
    th = 6 * np.pi * rng.random(n)
    x = np.stack([0.5 + 0.3 * np.cos(th), 0.5 + 0.3 * np.sin(th), 0.05 + 0.9 * th / (6 * np.pi)], axis=1)
    return np.clip(x + 1e-3 * rng.standard_normal((n, 3)), 0.0, 1.0)


def one_octant3(rng, n):
    return 0.3 * rng.random((n, 3))


def mixed3(rng, n):
    ns, nk = n // 2, n // 4
    s = sphere3(rng, ns, radius=0.3)
    k = np.clip(0.9 + 0.002 * rng.standard_normal((nk, 3)), 0.0, 1.0)
    return np.vstack([s, k, uniform3(rng, n - ns - nk)])


DISTRIBUTIONS3 = dict(uniform=uniform3, clustered=clustered3, sphere=sphere3, helix=helix3, one_octant=one_octant3,
                      mixed=mixed3)


def mrd(a, b):
    """max-norm relative difference (test/testutils.jl:9)"""
    a, b = np.asarray(a), np.asarray(b)
    if a.ndim == 2:
        return np.max(np.linalg.norm(a - b, axis=1)) / np.max(np.linalg.norm(b, axis=1))
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# ---------------------------------------------------------------- tree invariants (test/test_tree.jl:7-131)
def child_slot(x, c):
    return (x[..., 0] > c[..., 0]).astype(int) | ((x[..., 1] > c[..., 1]).astype(int) << 1) | \
           ((x[..., 2] > c[..., 2]).astype(int) << 2)


def centers(t, origin, W0):
    w = np.ldexp(W0, -t["level"].astype(int))
    return np.asarray(origin) + (t["cell"] + 0.5) * w[:, None]


def check_tree_invariants(t, pts, origin=(0.0, 0.0, 0.0), W0=1.0):
    """Every structural invariant of the ghost-cell tree, brute force. `t` is a dict of
    arrays with 0-based indices (-1 for none)."""
    N = pts.shape[0]
    n = len(t["level"])
    perm = t["perm"]
    assert sorted(perm) == list(range(N))
    sp = pts[perm]
    lev = t["level"]
    assert lev[0] == 0 and t["parent"][0] == -1 and tuple(t["cell"][0]) == (0, 0, 0)
    assert np.all(np.diff(lev) >= 0)
    assert t["plo"][0] == 0 and t["phi"][0] == N - 1
    leaf, ghost, xlist, hs = (t[k].astype(bool) for k in ("leaf", "ghost", "xlist", "has_source"))
    cf = t["child_first"]
    w = np.ldexp(W0, -lev.astype(int))
    assert np.all((t["cell"] >= 0) & (t["cell"] < (1 << lev)[:, None]))
    assert np.all(hs == (t["phi"] >= t["plo"]))
    assert not np.any(ghost & leaf)
    cen = centers(t, origin, W0)
    for i in range(n):
        lo, hi = t["plo"][i], t["phi"][i]
        if hi >= lo:
            blo = np.asarray(origin) + t["cell"][i] * w[i]
            bhi = np.asarray(origin) + (t["cell"][i] + 1) * w[i]
            assert np.all((sp[lo:hi + 1] >= blo) & (sp[lo:hi + 1] <= bhi))
        if cf[i] >= 0:
            ch = np.arange(cf[i], cf[i] + 8)
            assert np.all(t["parent"][ch] == i) and np.all(lev[ch] == lev[i] + 1)
            offs = np.array([[(k >> d) & 1 for d in range(3)] for k in range(8)])
            assert np.array_equal(t["cell"][ch], 2 * t["cell"][i] + offs)
            assert t["plo"][ch[0]] == lo and t["phi"][ch[-1]] == hi
            assert np.all(t["phi"][ch[:-1]] + 1 == t["plo"][ch[1:]])
            for k in range(8):
                a, b = t["plo"][ch[k]], t["phi"][ch[k]]
                if b >= a:
                    assert np.all(child_slot(sp[a:b + 1], cen[i]) == k)
            assert not ghost[i]
            if leaf[i]:
                assert xlist[i] and np.all(ghost[ch])
            else:
                assert not np.any(ghost[ch])
        else:
            assert not xlist[i]
            assert leaf[i] or ghost[i]
    # unique cells and brute-force colleagues
    col = t["colleagues"]
    L = lev.max() + 1
    coffs = np.array([[k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1] for k in range(27)])
    for l in range(L):
        idx = np.nonzero(lev == l)[0]
        lookup = {tuple(t["cell"][i]): i for i in idx}
        assert len(lookup) == len(idx)
        for i in idx:
            assert col[i, 13] == i
            for k in range(27):
                assert col[i, k] == lookup.get(tuple(t["cell"][i] + coffs[k]), -1)
    # 2:1 balance of real depths between colleagues
    rdepth = np.zeros(n, int)
    for i in range(n - 1, -1, -1):
        if cf[i] >= 0 and not leaf[i]:
            rdepth[i] = 1 + rdepth[cf[i]:cf[i] + 8].max()
    for i in np.nonzero(leaf)[0]:
        for j in col[i]:
            if j < 0 or ghost[j]:
                continue
            assert abs(rdepth[i] - rdepth[j]) <= 1
    # ghosts and xlist flags
    for i in range(n):
        if not leaf[i] and not ghost[i]:
            for j in col[i]:
                if j >= 0:
                    assert not ghost[j] and cf[j] >= 0
        if leaf[i]:
            nonleaf = any(j >= 0 and not leaf[j] and not ghost[j] for j in col[i])
            assert xlist[i] == nonleaf
    # point_node
    pn = t["point_node"]
    for j in range(N):
        p = pn[j]
        assert leaf[p] and t["plo"][p] <= j <= t["phi"][p]


def vlists(t):
    """V(y) of every node (test/test_coverage.jl:16-29): the children of the colleagues of
    parent(y) that are not colleagues of y (0-based, -1 for none)."""
    cf, par, col = t["child_first"], t["parent"], t["colleagues"]
    out = []
    for y in range(len(cf)):
        p = par[y]
        if p < 0:
            out.append(np.zeros(0, np.int64))
            continue
        c = col[p][col[p] >= 0]
        c = c[cf[c] >= 0]
        ch = (cf[c][:, None] + np.arange(8)[None, :]).ravel()
        out.append(np.setdiff1d(ch, col[y][col[y] >= 0]))
    return out


def check_coverage(t, pairs, far):
    """The kernel-free invariant of the FMM structure (test/test_coverage.jl:31-84), on a tree
    `t` (dict of arrays, 0-based) and its far pairs `pairs[l] = (target, source, far index)`:
    every (source terminal, target leaf) pair is covered exactly once, by the near field or by
    exactly one V-list interaction between an ancestor-or-self of each; the pairs are exactly
    the V lists restricted to sourced sources and non-ghost targets; offsets and levels agree
    with `far`; a target appears at most once per offset; levels 0 and 1 have no pairs.
    Terminals are childless, so "X is an ancestor-or-self of terminal T" is "T's points lie in
    X's point range": the count runs over points, one difference array per leaf."""
    n = len(t["level"])
    N = len(t["perm"])
    cf, par, col = t["child_first"], t["parent"], t["colleagues"]
    plo, phi = t["plo"].astype(np.int64), t["phi"].astype(np.int64)
    hs, leaf, ghost = (t[k].astype(bool) for k in ("has_source", "leaf", "ghost"))
    V = vlists(t)
    anc = []
    for i in range(n):
        a, j = [], i
        while j >= 0:
            a.append(j)
            j = par[j]
        anc.append(a)
    term = np.nonzero((cf < 0) & hs)[0]
    bad = 0
    for B in np.nonzero(leaf)[0]:
        near = np.zeros(N + 1, np.int64)
        c = col[B][col[B] >= 0]
        c = c[hs[c]]
        np.add.at(near, plo[c], 1)
        np.add.at(near, phi[c] + 1, -1)
        X = np.concatenate([V[Y] for Y in anc[B]]) if anc[B] else np.zeros(0, np.int64)
        X = X[hs[X]]
        cnt = np.zeros(N + 1, np.int64)
        np.add.at(cnt, plo[X], 1)
        np.add.at(cnt, phi[X] + 1, -1)
        nr, ct = np.cumsum(near)[plo[term]], np.cumsum(cnt)[plo[term]]
        ok = ((nr > 0) & (ct == 0)) | ((nr == 0) & (ct == 1))
        bad += int(np.count_nonzero(~ok))
    assert bad == 0, f"{bad} (terminal, leaf) pairs not covered exactly once"
    # the pairs are exactly V restricted to sourced sources and non-ghost targets
    got = np.concatenate([np.stack([pt[0], pt[1]]).astype(np.int64) for pt in pairs], axis=1) if pairs else np.zeros((2, 0), np.int64)
    key = got[0] * n + got[1]
    assert len(np.unique(key)) == len(key), "a pair listed twice"
    exp = [y * n + x for y in range(n) if not ghost[y] for x in V[y] if hs[x]]
    assert np.array_equal(np.sort(key), np.sort(np.asarray(exp, np.int64))), "pairs differ from the V lists"
    # offsets and levels; each target at most once per offset; nothing at levels 0 and 1
    for l, (tg, sc, f) in enumerate(pairs):
        if l < 2:
            assert len(tg) == 0
        if len(tg) == 0:
            continue
        assert np.all(t["level"][tg] == l) and np.all(t["level"][sc] == l)
        assert np.array_equal(t["cell"][sc] - t["cell"][tg], far[f])
        k = f.astype(np.int64) * n + tg
        assert len(np.unique(k)) == len(k), "a target twice for one offset"


def same_structure(a, b, keys=("cell", "level", "parent", "child_first", "plo", "phi", "leaf", "ghost", "xlist",
                                "has_source", "colleagues", "point_node")):
    """test/test_device_tree.jl:110-112: every structural field equal."""
    for k in keys:
        if not np.array_equal(np.asarray(a[k]), np.asarray(b[k])):
            return k
    return None


def oracle_tree_dict(T):
    return {k: getattr(T, k) for k in ("cell", "level", "parent", "child_first", "plo", "phi", "leaf", "ghost", "xlist",
                                       "has_source", "colleagues", "perm", "point_node")}


# ---------------------------------------------------------------- Stokes (src/kernels.jl:253-272)
def sphere_points(rng, n):
    """Points on the unit sphere jittered by U(−0.01, 0.01)³ (the batched Stokes workload)."""
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None] + rng.uniform(-0.01, 0.01, (n, 3))


def stokes_direct(src, f, sel):
    """FP64 Stokeslet velocities (1/8π)Σ_{j≠i}[f_j/r + d(d·f_j)/r³] at the sources `sel`."""
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


def stokes_direct_all(src, sel, f=None, fs=None, nu=None, g=None, w=None, output="velocity", tgt=None):
    """FP64 direct sums at the sources `sel` (i = j skipped), or at the points `tgt` (sel None),
    of weighted Stokeslets f, stresslets
    (fs, ν) and doublets g (src/sources.jl:203-251, c = 1/8π, d = t − s): velocities
    c[f/r + d(d·f)/r³] − 6c d(d·f_s)(d·ν)/r⁵ + c(g/r³ − 3d(d·g)/r⁵), or pressures
    2c(d·f)/r³ + 4c[(f_s·ν)/r³ − 3(d·f_s)(d·ν)/r⁵]."""
    n = src.shape[0]
    wt = np.ones(n) if w is None else w
    z = np.zeros((n, 3))
    f = z if f is None else f * wt[:, None]
    fs = z if fs is None else fs * wt[:, None]
    nu = z if nu is None else nu
    g = z if g is None else g * wt[:, None]
    c = 1 / (8 * np.pi)
    m = len(sel) if tgt is None else len(tgt)
    out = np.zeros({"velocity": (m, 3), "pressure": (m,), "gradient": (m, 3, 3)}[output])
    for a in range(0, m, 64):
        if tgt is None:
            idx = sel[a:a + 64]
            d = src[idx, None, :] - src[None, :, :]
            r2 = np.einsum("tsk,tsk->ts", d, d)
            r2[np.arange(len(idx)), idx] = np.inf
        else:
            d = tgt[a:a + 64, None, :] - src[None, :, :]
            r2 = np.einsum("tsk,tsk->ts", d, d)
        ir = 1.0 / np.sqrt(r2)
        ir3, ir5 = ir ** 3, ir ** 5
        df = np.einsum("tsk,sk->ts", d, f)
        ds = np.einsum("tsk,sk->ts", d, fs)
        dn = np.einsum("tsk,sk->ts", d, nu)
        if output == "velocity":
            dg = np.einsum("tsk,sk->ts", d, g)
            coef = df * ir3 - (3 * dg + 6 * ds * dn) * ir5
            out[a:a + 64] = c * (ir @ f + ir3 @ g + np.einsum("ts,tsk->tk", coef, d))
        elif output == "gradient":
            # ∂u_i/∂t_j of each kind in closed form (src/sources.jl:242-276), summed
            dg = np.einsum("tsk,sk->ts", d, g)
            ir7 = ir5 * ir * ir
            eye = np.eye(3)
            ddt = np.einsum("tsi,tsj->tsij", d, d)
            gr = np.einsum("ts,tsij->tij", ir3 * df, eye[None, None] * np.ones_like(ir)[..., None, None])
            gr += np.einsum("ts,tsi,sj->tij", ir3, d, f) - np.einsum("ts,si,tsj->tij", ir3, f, d)
            gr -= np.einsum("ts,tsij->tij", 3 * ir5 * df, ddt)
            gr -= np.einsum("ts,ij->tij", 6 * ir5 * ds * dn, eye)
            gr -= np.einsum("ts,tsi,sj->tij", 6 * ir5 * dn, d, fs) + np.einsum("ts,tsi,sj->tij", 6 * ir5 * ds, d, nu)
            gr += np.einsum("ts,tsij->tij", 30 * ir7 * ds * dn, ddt)
            gr -= np.einsum("ts,si,tsj->tij", 3 * ir5, g, d) + np.einsum("ts,ij->tij", 3 * ir5 * dg, eye)
            gr -= np.einsum("ts,tsi,sj->tij", 3 * ir5, d, g)
            gr += np.einsum("ts,tsij->tij", 15 * ir7 * dg, ddt)
            out[a:a + 64] = c * gr
        else:
            sn = np.einsum("sk,sk->s", fs, nu)
            out[a:a + 64] = c * np.sum(2 * df * ir3 + 4 * sn[None, :] * ir3 - 12 * ds * dn * ir5, axis=1)
    return out


# ---------------------------------------------------------------- Yukawa (src/kernels.jl:224-242)
def yukawa_direct(src, tau, tgt, kappa, self_excluded=False, gradient=False):
    """FP64 Σ_j τ_j e^{−κr}/(4πr) (and its gradient in the target) at tgt, in chunks."""
    pot = np.zeros(len(tgt))
    grad = np.zeros((len(tgt), 3))
    for a in range(0, len(tgt), 256):
        d = tgt[a:a + 256, None, :] - src[None, :, :]
        r = np.sqrt(np.einsum("tsk,tsk->ts", d, d))
        if self_excluded:
            r[np.arange(len(r)), np.arange(a, a + len(r))] = np.inf
        e = np.exp(-kappa * r) / r
        pot[a:a + 256] = e @ tau / (4 * np.pi)
        if gradient:
            g = -(e * (1 + kappa * r) / r ** 2) * tau[None, :]
            grad[a:a + 256] = np.einsum("ts,tsk->tk", g, d) / (4 * np.pi)
    return (pot, grad) if gradient else pot


# ---------------------------------------------------------------- the adaptive cloud (16 Gaussians, sigma 0.01)
def gaussian_cloud(n, seed=4, ncentres=16, sigma=0.01):
    """n points from `ncentres` isotropic Gaussians with centres uniform in [0.1, 0.9]^3, points
    outside the unit box redrawn (the adaptive cube-KI configuration's point cloud)."""
    rng = np.random.default_rng(seed)
    c = 0.1 + 0.8 * rng.random((ncentres, 3))
    pts = c[rng.integers(0, ncentres, n)] + sigma * rng.standard_normal((n, 3))
    bad = np.any((pts < 0) | (pts >= 1), axis=1)
    while bad.any():
        pts[bad] = c[rng.integers(0, ncentres, int(bad.sum()))] + sigma * rng.standard_normal((int(bad.sum()), 3))
        bad = np.any((pts < 0) | (pts >= 1), axis=1)
    return pts


def pairs_equal_as_sets(a, b):
    """(target, source, far index) arrays of one level equal as sets of triples."""
    a, b = np.stack(a), np.stack(b)
    return a.shape == b.shape and np.array_equal(a[:, np.lexsort(a)], b[:, np.lexsort(b)])
