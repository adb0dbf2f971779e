"""CPU restatement of the reference's kernel-independent method on circles, KernelIndependent(
Laplace2D(); nequiv), for the tests (test infrastructure, never the product path). It follows
the reference's own generic passes on a quadtree, here the plane z = 0 of the octree that the
oracle's tree builder (oracle.Tree) builds on the embedded points — the same embedding the device
path uses, and a tree whose in-plane nodes are the quadtree's (an octree node's refinement,
balance and ghost decisions depend on its points only, all of which lie in one z-slab).

  kernel           Laplace2D: c·log r², c = −1/(4π)                      src/kernels.jl:54-67
  surfaces         circles of nequiv points, radii √2/2·w (small) and
                   (4 − √2)/2·w (large), θ_k = 2πk/n                   src/operators/kifmm.jl:36-37,63-65
  kernel matrix    A[j, i] = K(s_i, t_j) (rows: targets)                 src/kernels.jl:404-416
  pseudo-inverse   truncated SVD, σ ≥ rtol·σ₁, kept as factors          src/operators/ki_common.jl:38-44
  operators        P_up = pinv(K(small → large)), P_down = pinv(K(large → small)); M2M and
                   L2L with the pseudo-inverse folded in, children at (δ − ½)·w/2, δ in slot
                   order (coordinate 1 least significant); M2L = K(small + o·w → small)
                                                                         src/operators/ki_common.jl:185-207,
                                                                         src/operators/kifmm.jl:67-80,
                                                                         src/util.jl:25-28
  passes           P2M: check potentials of a childless sourced node's sources on its large
                   circle, then P_up; M2M into parents, levels L−1 … 2 (0-based); M2L over the
                   far pairs; L2L on the check data, levels ≥ 3; leaves: P_down   src/fmm.jl:170-269,
                                                                         src/operators/ki_common.jl:240-285
  evaluation       L2T over the leaf's large circle plus the direct sum over its colleagues'
                   sources, self excluded                                src/evaluate.jl:27-50,
                                                                         src/operators/ki_common.jl:303-322
"""
import numpy as np

import oracle as O

C2 = -1.0 / (4.0 * np.pi)
SMALL = np.sqrt(2.0) / 2.0
LARGE = (4.0 - np.sqrt(2.0)) / 2.0


def circle_points(n, r):
    """circle_points (src/operators/kifmm.jl:63-65)."""
    th = (2.0 * np.pi / n) * np.arange(n)
    return np.stack([r * np.cos(th), r * np.sin(th)], axis=1)


def kernel_matrix(sources, targets):
    """kernel_matrix (src/kernels.jl:404-416) of Laplace2D: rows targets, columns sources."""
    d = targets[:, None, :] - sources[None, :, :]
    return C2 * np.log(np.einsum("tsk,tsk->ts", d, d))


class Pinv:
    """FactoredPinv (src/operators/ki_common.jl:21-44): V·diag(1/σ)·Uᴴ, σ ≥ rtol·σ₁ kept."""

    def __init__(self, A, rtol):
        U, s, Vh = np.linalg.svd(A)
        r = int(np.count_nonzero(s >= rtol * s[0]))
        self.Uh, self.invS, self.V = U[:, :r].T, 1.0 / s[:r], Vh[:r].T

    def apply(self, x):
        return self.V @ (self.invS[:, None] * (self.Uh @ x)) if x.ndim == 2 else self.V @ (self.invS * (self.Uh @ x))


class CircleLevel:
    """level_operators(m::KernelIndependent, w) (src/operators/kifmm.jl:67-80) with the dense
    parts of _ki_dense_operators (src/operators/ki_common.jl:185-207)."""

    def __init__(self, n, w, rtol):
        self.w = w
        self.small = circle_points(n, SMALL * w)
        self.large = circle_points(n, LARGE * w)
        child_small = circle_points(n, SMALL * w / 2)
        self.up = Pinv(kernel_matrix(self.small, self.large), rtol)
        self.down = Pinv(kernel_matrix(self.large, self.small), rtol)
        centers = [(np.array([k & 1, (k >> 1) & 1], float) - 0.5) * (w / 2) for k in range(4)]
        m2mc = np.hstack([kernel_matrix(child_small + c, self.large) for c in centers])
        l2lc = np.vstack([kernel_matrix(self.large, child_small + c) for c in centers])
        # the pseudo-inverses folded in the order that keeps the 1/σ inside its own mode
        self.m2m = self.up.V @ (self.up.invS[:, None] * (self.up.Uh @ m2mc))
        self.l2l = ((l2lc @ self.down.V) * self.down.invS[None, :]) @ self.down.Uh
        self.n = n
        self._m2l = {}

    def m2l(self, off):
        """The M2L of far offset `off` (in widths): K(small + off·w → small)."""
        key = (int(off[0]), int(off[1]))
        if key not in self._m2l:
            o = np.array(key, float) * self.w
            self._m2l[key] = kernel_matrix(self.small + o, self.small)
        return self._m2l[key]


def circle_fmm(pts2, tau, nequiv, ppl, origin2, width, rtol=50 * np.finfo(float).eps, max_levels=30):
    """evaluate_at_sources (potential and gradient, self excluded) of the circle KI FMM of the
    2D points `pts2` (N, 2) with charges `tau`, in the square box (origin2, width); returns
    (potential, gradient (N, 2), the tree)."""
    N = len(pts2)
    xyz = np.concatenate([pts2, np.zeros((N, 1))], axis=1)
    T = O.Tree.build(xyz, ppl, origin=(origin2[0], origin2[1], -width / 2), width=width, max_levels=max_levels)
    L = T.L
    perm = T.perm
    xs = pts2[perm]                          # sources in tree order
    ts = tau[perm]
    ops = [CircleLevel(nequiv, width / 2.0 ** l, rtol) if l >= 2 else None for l in range(L)]
    org = np.asarray(origin2, float)

    def center(i):
        l = T.level[i]
        return org + (T.cell[i, :2] + 0.5) * (width / 2.0 ** l)

    nn = T.n
    M = np.zeros((nn, nequiv))
    for l in range(L - 1, 1, -1):
        op = ops[l]
        for i in range(T.level_start[l], T.level_start[l + 1]):
            if T.child_first[i] < 0 and T.has_source[i]:
                x = xs[T.plo[i]:T.phi[i] + 1] - center(i)
                pm = kernel_matrix(x, op.large) @ ts[T.plo[i]:T.phi[i] + 1]
                M[i] = op.up.apply(pm)
            elif T.child_first[i] >= 0:
                # the sourced children of the plane, each in its quadtree slot
                acc = np.zeros(4 * nequiv)
                for c in range(T.child_first[i], T.child_first[i] + 8):
                    if T.has_source[c]:
                        slot = (T.cell[c, 0] & 1) | ((T.cell[c, 1] & 1) << 1)
                        acc[slot * nequiv:(slot + 1) * nequiv] += M[c]
                M[i] = op.m2m @ acc
    Pl = np.zeros((nn, nequiv))
    Lc = np.zeros((nn, nequiv))
    for l in range(2, L):
        op = ops[l]
        if l > 2:
            pop = ops[l - 1]
            for i in range(T.level_start[l], T.level_start[l + 1]):
                p = T.parent[i]
                slot = (T.cell[i, 0] & 1) | ((T.cell[i, 1] & 1) << 1)
                Pl[i] += pop.l2l[slot * nequiv:(slot + 1) * nequiv] @ Pl[p]
        t, s, _ = T.pairs(l)
        for a, b in zip(t, s):
            if T.cell[b, 2] != T.cell[a, 2]:
                continue                     # an empty target outside the plane: nothing to evaluate there
            off = T.cell[b, :2] - T.cell[a, :2]
            Pl[a] += op.m2l(off) @ M[b]
        for i in range(T.level_start[l], T.level_start[l + 1]):
            if T.leaf[i]:
                Lc[i] = op.down.apply(Pl[i])
    pot = np.zeros(N)
    grad = np.zeros((N, 2))
    for i in range(nn):
        if not (T.leaf[i] and T.has_source[i]):
            continue
        l = T.level[i]
        lo, hi = T.plo[i], T.phi[i] + 1
        x = xs[lo:hi]
        c = center(i)
        if l >= 2:
            large = ops[l].large
            d = (x - c)[:, None, :] - large[None, :, :]
            r2 = np.einsum("tsk,tsk->ts", d, d)
            pot[lo:hi] += (C2 * np.log(r2)) @ Lc[i]
            grad[lo:hi] += np.einsum("ts,tsk->tk", (2 * C2 / r2) * Lc[i][None, :], d)
        for cc in T.colleagues[i]:
            if cc < 0 or not T.has_source[cc]:
                continue
            y = xs[T.plo[cc]:T.phi[cc] + 1]
            q = ts[T.plo[cc]:T.phi[cc] + 1]
            d = x[:, None, :] - y[None, :, :]
            r2 = np.einsum("tsk,tsk->ts", d, d)
            self_ = np.eye(len(x), dtype=bool) if cc == i else np.zeros(r2.shape, bool)   # by index
            r2 = np.where(self_, 1.0, r2)
            g = np.where(self_, 0.0, C2 * np.log(r2))
            pot[lo:hi] += g @ q
            gg = np.where(self_, 0.0, 2 * C2 / r2) * q[None, :]
            grad[lo:hi] += np.einsum("ts,tsk->tk", gg, d)
    out_p = np.empty(N)
    out_g = np.empty((N, 2))
    out_p[perm] = pot
    out_g[perm] = grad
    return out_p, out_g, T


# ---------------------------------------------------------------- CubeKernelIndependent{3}(Laplace3D)
# The cube surfaces (src/operators/cubeki.jl:55-79, src/operators/spectral_m2l.jl:103-115): the
# boundary points of p-per-edge lattices on cubes of half-width (1 + d)·w/2 (small: upward
# equivalent, downward check) and (3 − 2d)·w/2 (large, pc per edge: upward check, downward
# equivalent), coordinate 1 fastest. The M2L here is the dense kernel-matrix product
# K(small + o·w → small) per far pair — what the spectral translation computes exactly
# (src/operators/spectral_m2l.jl:1-14; the reference's own check, test/test_cubeki.jl:43-69).
C3 = 1.0 / (4.0 * np.pi)


def cube_boundary_points(p, a):
    """cube_boundary_points(Val(3), p, a) (src/operators/spectral_m2l.jl:103-115)."""
    coords = -a + 2 * a * np.arange(p) / (p - 1)
    out = []
    for k in range(p):
        for j in range(p):
            for i in range(p):          # coordinate 1 fastest
                if i in (0, p - 1) or j in (0, p - 1) or k in (0, p - 1):
                    out.append((coords[i], coords[j], coords[k]))
    return np.array(out)


def kernel_matrix3(sources, targets):
    """kernel_matrix (src/kernels.jl:404-416) of Laplace3D, 1/(4πr)."""
    d = targets[:, None, :] - sources[None, :, :]
    return C3 / np.sqrt(np.einsum("tsk,tsk->ts", d, d))


def cube_boundary_lattice(p):
    """The lattice indices (i1, i2, i3) in [0, p)³ of the boundary points, in the order of
    cube_boundary_points (coordinate 1 fastest): the embedding of the spectral translation
    (src/operators/spectral_m2l.jl:103-115)."""
    out = []
    for k in range(p):
        for j in range(p):
            for i in range(p):
                if i in (0, p - 1) or j in (0, p - 1) or k in (0, p - 1):
                    out.append((i, j, k))
    return np.array(out)


def spectral_m2l(p, a, off, w, sigma):
    """The spectral M2L of one far pair (src/operators/spectral_m2l.jl: `_kernel_tables` :117-135
    and the single-vector `apply!` :144-173), FP64 with numpy's FFT: the source box's density σ on
    its p-per-edge boundary lattice of half-width a (spacing h = 2a/(p − 1)) embedded in the
    zero-padded (2p)³ lattice, transformed, multiplied by the transform of the circulant kernel
    table κ(m) = G(h·m − off·w), m ∈ [−(p − 1), p − 1]³ at the wrapped index m mod 2p, transformed
    back, and read at the target box's boundary lattice points: the check potentials
    Σ_j G(y_i − x_j) σ_j with y on the target's surface and x = y' + off·w on the source's."""
    n = 2 * p
    h = 2.0 * a / (p - 1)
    m = np.arange(-(p - 1), p)
    M1, M2, M3 = np.meshgrid(m, m, m, indexing="ij")
    o = np.asarray(off, float) * w
    r = np.sqrt((h * M1 - o[0]) ** 2 + (h * M2 - o[1]) ** 2 + (h * M3 - o[2]) ** 2)
    tab = np.zeros((n, n, n))
    tab[M1 % n, M2 % n, M3 % n] = C3 / r
    lat = cube_boundary_lattice(p)
    sg = np.zeros((n, n, n))
    sg[lat[:, 0], lat[:, 1], lat[:, 2]] = sigma
    u = np.fft.ifftn(np.fft.fftn(tab) * np.fft.fftn(sg)).real
    return u[lat[:, 0], lat[:, 1], lat[:, 2]]


class CubeLevel:
    """level_operators(m::CubeKernelIndependent{3}, w) (src/operators/cubeki.jl:55-79) with
    _ki_dense_operators (src/operators/ki_common.jl:185-207), the M2L dense."""

    def __init__(self, p, pc, d, w, rtol):
        self.w = w
        a_small, a_large = (1 + d) * w / 2, (3 - 2 * d) * w / 2
        self.small = cube_boundary_points(p, a_small)
        self.large = cube_boundary_points(pc, a_large)
        child_small = cube_boundary_points(p, a_small / 2)
        self.up = Pinv(kernel_matrix3(self.small, self.large), rtol)
        self.down = Pinv(kernel_matrix3(self.large, self.small), rtol)
        centers = [(np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1], float) - 0.5) * (w / 2) for k in range(8)]
        m2mc = np.hstack([kernel_matrix3(child_small + c, self.large) for c in centers])
        l2lc = np.vstack([kernel_matrix3(self.large, child_small + c) for c in centers])
        self.m2m = self.up.V @ (self.up.invS[:, None] * (self.up.Uh @ m2mc))
        self.l2l = ((l2lc @ self.down.V) * self.down.invS[None, :]) @ self.down.Uh
        self.ns = len(self.small)
        self._m2l = {}

    def m2l(self, off):
        key = tuple(int(v) for v in off)
        if key not in self._m2l:
            self._m2l[key] = kernel_matrix3(self.small + np.array(key, float) * self.w, self.small)
        return self._m2l[key]


def cube_fmm(pts, tau, p, ppl, origin, width, pc=None, d=0.1, rtol=50 * np.finfo(np.float32).eps, max_levels=30):
    """evaluate_at_sources (potential and gradient, self excluded) of the cube KI FMM of Laplace3D
    on the 3D points `pts` with charges `tau`, in the box (origin, width), FP64 throughout, with
    the reference's default truncation for Laplace3D(Float32) (50·eps(Float32)); returns
    (potential, gradient, multipoles (nnodes × small points), leaf densities (nnodes × large
    points), the tree)."""
    pc = 2 * p if pc is None else pc
    N = len(pts)
    T = O.Tree.build(pts, ppl, origin=origin, width=width, max_levels=max_levels)
    L = T.L
    perm = T.perm
    xs = pts[perm]
    ts = tau[perm]
    ops = [CubeLevel(p, pc, d, width / 2.0 ** l, rtol) if l >= 2 else None for l in range(L)]
    org = np.asarray(origin, float)
    ns = ops[2].ns if L > 2 else 0
    nl = len(ops[2].large) if L > 2 else 0

    def center(i):
        return org + (T.cell[i] + 0.5) * (width / 2.0 ** T.level[i])

    nn = T.n
    M = np.zeros((nn, ns))
    for l in range(L - 1, 1, -1):
        op = ops[l]
        for i in range(T.level_start[l], T.level_start[l + 1]):
            if T.child_first[i] < 0 and T.has_source[i]:
                x = xs[T.plo[i]:T.phi[i] + 1] - center(i)
                M[i] = op.up.apply(kernel_matrix3(x, op.large) @ ts[T.plo[i]:T.phi[i] + 1])
            elif T.child_first[i] >= 0:
                M[i] = op.m2m @ M[T.child_first[i]:T.child_first[i] + 8].reshape(-1)
    Pl = np.zeros((nn, ns))                  # check data on the small surfaces
    Lc = np.zeros((nn, nl))                  # the leaves' densities on the large surfaces
    for l in range(2, L):
        op = ops[l]
        if l > 2:
            pop = ops[l - 1]
            for i in range(T.level_start[l], T.level_start[l + 1]):
                k = (T.cell[i, 0] & 1) | ((T.cell[i, 1] & 1) << 1) | ((T.cell[i, 2] & 1) << 2)
                Pl[i] += pop.l2l[k * ns:(k + 1) * ns] @ Pl[T.parent[i]]
        t, s, _ = T.pairs(l)
        for a, b in zip(t, s):
            Pl[a] += op.m2l(T.cell[b] - T.cell[a]) @ M[b]
        for i in range(T.level_start[l], T.level_start[l + 1]):
            if T.leaf[i]:
                Lc[i] = op.down.apply(Pl[i])
    pot = np.zeros(N)
    grad = np.zeros((N, 3))
    for i in range(nn):
        if not (T.leaf[i] and T.has_source[i]):
            continue
        lo, hi = T.plo[i], T.phi[i] + 1
        x = xs[lo:hi]
        if T.level[i] >= 2:
            dd = (x - center(i))[:, None, :] - ops[T.level[i]].large[None, :, :]
            ir = 1.0 / np.sqrt(np.einsum("tsk,tsk->ts", dd, dd))
            pot[lo:hi] += (C3 * ir) @ Lc[i]
            grad[lo:hi] -= np.einsum("ts,tsk->tk", C3 * ir ** 3 * Lc[i][None, :], dd)
        for cc in T.colleagues[i]:
            if cc < 0 or not T.has_source[cc]:
                continue
            y = xs[T.plo[cc]:T.phi[cc] + 1]
            q = ts[T.plo[cc]:T.phi[cc] + 1]
            dd = x[:, None, :] - y[None, :, :]
            r2 = np.einsum("tsk,tsk->ts", dd, dd)
            self_ = np.eye(len(x), dtype=bool) if cc == i else np.zeros(r2.shape, bool)
            ir = np.where(self_, 0.0, 1.0 / np.sqrt(np.where(self_, 1.0, r2)))
            pot[lo:hi] += (C3 * ir) @ q
            grad[lo:hi] -= np.einsum("ts,tsk->tk", C3 * ir ** 3 * q[None, :], dd)
    out_p = np.empty(N)
    out_g = np.empty((N, 3))
    out_p[perm] = pot
    out_g[perm] = grad
    return out_p, out_g, M, Lc, T
