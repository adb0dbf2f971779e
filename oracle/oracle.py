"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the reference CPU path of FlexibleFMM.jl for the harmonic methods:
`SphericalHarmonics` of Laplace3D (src/tree/*.jl, src/operators/harmonics.jl, symmetry.jl,
src/fmm.jl, src/evaluate.jl, src/kernels.jl) and of Yukawa3D (harmonics_yukawa.jl), and
`StokesHarmonics` of Stokeslet3D (harmonics_stokes.jl). Only the tests, the smoke check and
the CPU baseline of the benchmark import this module; the product never does.
Node and point indices here are 0-based (-1 for "none"), levels 0-based (root 0).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")


def build():
    """Compile the oracle library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def numpy_blas_path():
    """The OpenBLAS bundled with numpy (ILP64, scipy_ prefixed symbols), or ''."""
    d = os.path.join(os.path.dirname(np.__file__), "..", "numpy.libs")
    if os.path.isdir(d):
        for f in sorted(os.listdir(d)):
            if f.startswith("libscipy_openblas64_"):
                return os.path.abspath(os.path.join(d, f))
    return ""


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    L.orc_last_error.restype = C.c_char_p
    L.orc_set_blas.argtypes = [C.c_char_p, C.c_int]
    L.orc_num_threads.restype = C.c_int
    L.orc_tree_build.argtypes = [f64p, C.c_int64, C.c_int, f64p, C.c_double, C.c_int, C.POINTER(C.c_void_p)]
    L.orc_tree_free.argtypes = [C.c_void_p]
    L.orc_tree_info.argtypes = [C.c_void_p, i64p]
    L.orc_tree_get.argtypes = [C.c_void_p, i32p, i32p, i32p, i32p, i32p, i32p, u8p, u8p, u8p, u8p, i32p, i32p, i32p]
    L.orc_tree_npairs.argtypes = [C.c_void_p, C.c_int]
    L.orc_tree_npairs.restype = C.c_int64
    L.orc_tree_pairs.argtypes = [C.c_void_p, C.c_int, i32p, i32p, i32p]
    L.orc_fmm_create.argtypes = [C.c_int, f64p, C.c_int64, C.c_int, f64p, C.c_double, C.c_int, C.c_double, C.POINTER(C.c_void_p)]
    L.orc_fmm_create_kind.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, f64p, C.c_int64, C.c_int,
                                      f64p, C.c_double, C.c_int, C.c_double, C.POINTER(C.c_void_p)]
    L.orc_fmm_eval_sources_stokes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_fmm_eval_targets_stokes.argtypes = [C.c_void_p, f64p, C.c_int64, C.c_void_p, C.c_void_p]
    L.orc_fmm_nblocks.argtypes = [C.c_void_p]
    L.orc_fmm_free.argtypes = [C.c_void_p]
    L.orc_fmm_tree.argtypes = [C.c_void_p]
    L.orc_fmm_tree.restype = C.c_void_p
    L.orc_fmm_build.argtypes = [C.c_void_p, f64p, f64p]
    L.orc_fmm_eval_sources.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_fmm_eval_targets.argtypes = [C.c_void_p, f64p, C.c_int64, C.c_void_p, C.c_void_p]
    L.orc_fmm_locate.argtypes = [C.c_void_p, f64p, C.c_int64, i32p]
    L.orc_fmm_np.argtypes = [C.c_void_p]
    L.orc_fmm_expansions.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_fmm_operators.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_regular_hobson.argtypes = [f64p, C.c_int, f64p]
    L.orc_irregular_hobson.argtypes = [f64p, C.c_int, f64p]
    L.orc_scaling_factors.argtypes = [C.c_int, f64p]
    L.orc_fold_regular.argtypes = [f64p, C.c_int, f64p]
    L.orc_harmonic_m2l.argtypes = [i32p, C.c_int, C.c_double, f64p]
    L.orc_harmonic_classes.argtypes = [C.c_int, i32p, i32p, i32p, i8p, i32p, i8p]
    L.orc_far_offsets.argtypes = [i32p]
    L.orc_yukawa_uv.argtypes = [C.c_double, C.c_int, f64p, f64p]
    L.orc_yukawa_bases.argtypes = [f64p, f64p, C.c_double, C.c_int, f64p, f64p]
    L.orc_direct.argtypes = [f64p, f64p, C.c_int64, f64p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_direct_sample.argtypes = [f64p, f64p, C.c_int64, i64p, C.c_int64, C.c_void_p, C.c_void_p]
    _lib = L
    return L


def set_threads(threads=0, blas=True):
    """Use numpy's OpenBLAS for the products (one BLAS thread per task) and `threads` OpenMP threads."""
    path = numpy_blas_path() if blas else ""
    rc = lib().orc_set_blas(path.encode(), int(threads))
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return lib().orc_num_threads()


class OracleError(Exception):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(lib().orc_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _pts(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    assert x.ndim == 2 and x.shape[1] == 3
    return x


# ---------------------------------------------------------------- tree
class Tree:
    """The host tree (src/tree/builder.jl:482-496) flattened to arrays."""

    FIELDS = ("cell", "level", "parent", "child_first", "plo", "phi", "leaf", "ghost", "xlist",
              "has_source", "colleagues", "perm", "point_node")

    def __init__(self, handle, owner=True):
        self._h = handle
        self._owner = owner
        info = np.zeros(3 + 64, np.int64)
        lib().orc_tree_info(self._h, info)
        self.L, self.n, self.N = int(info[0]), int(info[1]), int(info[2])
        self.level_start = info[3:3 + self.L + 1].astype(np.int64)
        n, N = self.n, self.N
        self.cell = np.zeros((n, 3), np.int32)
        self.level = np.zeros(n, np.int32)
        self.parent = np.zeros(n, np.int32)
        self.child_first = np.zeros(n, np.int32)
        self.plo = np.zeros(n, np.int32)
        self.phi = np.zeros(n, np.int32)
        self.leaf = np.zeros(n, np.uint8)
        self.ghost = np.zeros(n, np.uint8)
        self.xlist = np.zeros(n, np.uint8)
        self.has_source = np.zeros(n, np.uint8)
        self.colleagues = np.zeros((n, 27), np.int32)
        self.perm = np.zeros(N, np.int32)
        self.point_node = np.zeros(N, np.int32)
        lib().orc_tree_get(self._h, self.cell, self.level, self.parent, self.child_first, self.plo, self.phi,
                           self.leaf, self.ghost, self.xlist, self.has_source, self.colleagues, self.perm,
                           self.point_node)

    @classmethod
    def build(cls, xyz, ppl, origin=(0.0, 0.0, 0.0), width=1.0, max_levels=30):
        x = _pts(xyz)
        h = C.c_void_p()
        _check(lib().orc_tree_build(x, x.shape[0], int(ppl), np.asarray(origin, np.float64), float(width),
                                    int(max_levels), C.byref(h)))
        return cls(h)

    def pairs(self, level):
        """Far pairs of a level as (target, source, far index) arrays, in the fill order of src/tree/lists.jl."""
        n = lib().orc_tree_npairs(self._h, level)
        t = np.zeros(n, np.int32)
        s = np.zeros(n, np.int32)
        f = np.zeros(n, np.int32)
        if n:
            lib().orc_tree_pairs(self._h, level, t, s, f)
        return t, s, f

    def __del__(self):
        if getattr(self, "_owner", False) and self._h:
            lib().orc_tree_free(self._h)
            self._h = None


# ---------------------------------------------------------------- FMM
def gauss_legendre(n):
    """The Gauss–Legendre rule on [−1, 1] by the Golub–Welsch eigenvalues of the Jacobi matrix,
    as src/operators/harmonics_yukawa.jl:89-93 computes it (LAPACK through numpy): nodes
    ascending, weights 2 v₁²."""
    k = np.arange(1, n)
    beta = k / np.sqrt(4.0 * k * k - 1)
    J = np.diag(beta, 1) + np.diag(beta, -1)
    t, V = np.linalg.eigh(J)
    return np.ascontiguousarray(t), np.ascontiguousarray(2 * V[0, :] ** 2)


KINDS = {"laplace": 0, "yukawa": 1, "stokes": 2}


class FMM:
    """FMM(method, sources; ppl, bbox) with build_expansions and evaluation, for the harmonic
    methods: kernel "laplace" (SphericalHarmonics(Laplace3D())), "yukawa" (SphericalHarmonics(
    Yukawa3D(kappa))) or "stokes" (StokesHarmonics(Stokeslet3D()): forces (N, 3), velocity and
    pressure outputs)."""

    def __init__(self, p, xyz, ppl, origin=(0.0, 0.0, 0.0), width=1.0, max_levels=30, ref_width=0.0, kernel="laplace",
                 kappa=0.0):
        x = _pts(xyz)
        h = C.c_void_p()
        self.kernel = kernel
        if kernel == "laplace":
            _check(lib().orc_fmm_create(int(p), x, x.shape[0], int(ppl), np.asarray(origin, np.float64), float(width),
                                        int(max_levels), float(ref_width), C.byref(h)))
        else:
            gt, gw = gauss_legendre(2 * p + 10)
            _check(lib().orc_fmm_create_kind(KINDS[kernel], int(p), float(kappa), _ptr(gt), _ptr(gw), len(gt), x,
                                             x.shape[0], int(ppl), np.asarray(origin, np.float64), float(width),
                                             int(max_levels), float(ref_width), C.byref(h)))
        self._h = h
        self.p = p
        self.np_ = lib().orc_fmm_np(self._h)
        self.nb = lib().orc_fmm_nblocks(self._h)
        self.tree = Tree(C.c_void_p(lib().orc_fmm_tree(self._h)), owner=False)
        self.N = x.shape[0]

    def build_expansions(self, xyz, tau):
        x = _pts(xyz)
        t = np.ascontiguousarray(tau, dtype=np.float64)
        assert t.shape == ((self.N, 3) if self.kernel == "stokes" else (self.N,))
        _check(lib().orc_fmm_build(self._h, x, t))

    def evaluate_at_sources_stokes(self):
        """(velocity (N, 3), pressure (N,)) at the sources, each source's own term excluded."""
        vel, pres = np.zeros((self.N, 3)), np.zeros(self.N)
        _check(lib().orc_fmm_eval_sources_stokes(self._h, _ptr(vel), _ptr(pres)))
        return vel, pres

    def evaluate_stokes(self, targets):
        tg = _pts(targets)
        vel, pres = np.zeros((tg.shape[0], 3)), np.zeros(tg.shape[0])
        _check(lib().orc_fmm_eval_targets_stokes(self._h, tg, tg.shape[0], _ptr(vel), _ptr(pres)))
        return vel, pres

    def evaluate_at_sources(self, potential=True, gradient=True):
        pot = np.zeros(self.N) if potential else None
        grad = np.zeros((self.N, 3)) if gradient else None
        _check(lib().orc_fmm_eval_sources(self._h, _ptr(pot), _ptr(grad)))
        return pot, grad

    def evaluate(self, targets, potential=True, gradient=True):
        tg = _pts(targets)
        nt = tg.shape[0]
        pot = np.zeros(nt) if potential else None
        grad = np.zeros((nt, 3)) if gradient else None
        _check(lib().orc_fmm_eval_targets(self._h, tg, nt, _ptr(pot), _ptr(grad)))
        return pot, grad

    def locate(self, targets):
        tg = _pts(targets)
        out = np.zeros(tg.shape[0], np.int32)
        _check(lib().orc_fmm_locate(self._h, tg, tg.shape[0], out))
        return out

    def expansions(self):
        """(multipoles, locals) as (nnodes, nblocks·(p+1)^2) arrays in node order (Stokes: the blocks
        Φ₁, Φ₂, Φ₃, Ψ̂ one after the other)."""
        n = self.tree.n
        M = np.zeros((n, self.nb * self.np_))
        Lc = np.zeros((n, self.nb * self.np_))
        lib().orc_fmm_expansions(self._h, _ptr(M), _ptr(Lc))
        return M, Lc

    def operators(self):
        N = self.np_
        M2M = np.zeros(N * 8 * N)
        L2L = np.zeros(8 * N * N)
        reps = np.zeros(34 * N * N)
        lib().orc_fmm_operators(self._h, _ptr(M2M), _ptr(L2L), _ptr(reps))
        return (M2M.reshape(8 * N, N).T, L2L.reshape(N, 8 * N).T, reps.reshape(34, N, N).transpose(0, 2, 1))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_fmm_free(self._h)
            self._h = None


# ---------------------------------------------------------------- pieces
def regular_hobson(x, p):
    out = np.zeros(2 * (p + 1) ** 2)
    lib().orc_regular_hobson(np.asarray(x, np.float64), p, out)
    return out[0::2] + 1j * out[1::2]


def irregular_hobson(x, p):
    out = np.zeros(2 * (p + 1) ** 2)
    lib().orc_irregular_hobson(np.asarray(x, np.float64), p, out)
    return out[0::2] + 1j * out[1::2]


def scaling_factors(p):
    out = np.zeros((p + 1) ** 2)
    lib().orc_scaling_factors(p, out)
    return out


def fold_regular(x, p):
    out = np.zeros(2 * (p + 1) ** 2)
    lib().orc_fold_regular(np.asarray(x, np.float64), p, out)
    return out[0::2] + 1j * out[1::2]


def harmonic_m2l(o, p, c):
    N = (p + 1) ** 2
    out = np.zeros(N * N)
    lib().orc_harmonic_m2l(np.asarray(o, np.int32), p, float(c), out)
    return out.reshape(N, N).T


def harmonic_classes(p):
    N = (p + 1) ** 2
    cls = np.zeros(316, np.int32)
    reps = np.zeros(34 * 3, np.int32)
    idx = np.zeros(316 * N, np.int32)
    sgn = np.zeros(316 * N, np.int8)
    idx_t = np.zeros(316 * N, np.int32)
    sgn_t = np.zeros(316 * N, np.int8)
    nrep = lib().orc_harmonic_classes(p, cls, reps, idx, sgn, idx_t, sgn_t)
    return dict(cls=cls, reps=reps.reshape(34, 3)[:nrep], idx=idx.reshape(316, N), sgn=sgn.reshape(316, N),
                idx_t=idx_t.reshape(316, N), sgn_t=sgn_t.reshape(316, N))


def far_offsets():
    out = np.zeros(316 * 3, np.int32)
    lib().orc_far_offsets(out)
    return out.reshape(316, 3)


def direct(src, tau, targets=None, potential=True, gradient=True):
    """FP64 direct sums (src/kernels.jl:463-487); targets=None: at the sources, self excluded."""
    s = _pts(src)
    t = np.ascontiguousarray(tau, np.float64)
    self_ = targets is None
    tg = s if self_ else _pts(targets)
    nt = tg.shape[0]
    pot = np.zeros(nt) if potential else None
    grad = np.zeros((nt, 3)) if gradient else None
    lib().orc_direct(s, t, s.shape[0], tg, nt, int(self_), _ptr(pot), _ptr(grad))
    return pot, grad


def direct_sample(src, tau, sel, potential=True, gradient=True):
    """FP64 direct sums at the sources `sel` (indices), each excluding itself."""
    s = _pts(src)
    t = np.ascontiguousarray(tau, np.float64)
    sel = np.ascontiguousarray(sel, np.int64)
    pot = np.zeros(len(sel)) if potential else None
    grad = np.zeros((len(sel), 3)) if gradient else None
    lib().orc_direct_sample(s, t, s.shape[0], sel, len(sel), _ptr(pot), _ptr(grad))
    return pot, grad


def yukawa_radial(z, nmax):
    """(u_n(z), v_n(z)) for n = 0..nmax (src/operators/harmonics_yukawa.jl:44-73)."""
    u, v = np.zeros(nmax + 1), np.zeros(nmax + 1)
    lib().orc_yukawa_uv(float(z), int(nmax), u, v)
    return u, v


def yukawa_bases(y, x, kappa, p):
    """The real regular basis at y and the real irregular basis at x (harmonics_yukawa.jl:111-142)."""
    N = (p + 1) ** 2
    br, bi = np.zeros(N), np.zeros(N)
    lib().orc_yukawa_bases(np.asarray(y, np.float64), np.asarray(x, np.float64), float(kappa), int(p), br, bi)
    return br, bi
