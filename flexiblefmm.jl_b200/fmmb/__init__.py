"""fmmb: the host-side mirror of FlexibleFMM.jl's API over the sm_100a C ABI (include/fmmb.h).

The names, argument meanings and errors follow the reference (src/FlexibleFMM.jl:37-47):

    m = SphericalHarmonics(Laplace3D(), p=10)
    cache = OperatorCache(m)
    f = FMM(m, points, ppl=64, bbox=((0, 0, 0), 1.0), cache=cache)   # src/fmm.jl:31-49
    st = build_expansions(f, points, tau)                             # src/fmm.jl:306-314
    u = evaluate_at_sources(f, st)                                    # src/evaluate.jl:111-132
    g = evaluate(f, st, targets, output=Gradient())                   # src/evaluate.jl:81-102

Points are (N, 3) float64 arrays (the memory of Vector{SVector{3,Float64}}); gradients come
back as (N, 3). ArgumentError and DimensionMismatch mirror the reference's exceptions.
Everything runs on the GPU through libfmmb.so; there is no CPU path, and importing this
module fails when the library is missing.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_HERE), "libfmmb.so")

FMMB_OK = 0
_CODES = {1: "ArgumentError", 2: "DimensionMismatch", 3: "OutOfMemory", 4: "DeviceError", 5: "Timeout",
          6: "Unsupported"}
PRECISION_FP64 = 0
PRECISION_MIXED = 1
OUTPUT_POTENTIAL = 1
OUTPUT_GRADIENT = 2
KERNEL_LAPLACE3D = 1
KERNEL_YUKAWA3D = 2
KERNEL_STOKESLET3D = 3
KERNEL_LAPLACE2D = 4


class FMMBError(RuntimeError):
    """A device, memory or timeout failure reported by libfmmb."""

    def __init__(self, code, msg):
        super().__init__(f"{_CODES.get(code, code)}: {msg}")
        self.code = code


class ArgumentError(FMMBError, ValueError):
    pass


class DimensionMismatch(FMMBError, ValueError):
    pass


class Unsupported(FMMBError, NotImplementedError):
    pass


class _MethodDesc(C.Structure):
    _fields_ = [("method", C.c_int32), ("kernel", C.c_int32), ("p", C.c_int32), ("reserved", C.c_int32),
                ("tol", C.c_double), ("kappa", C.c_double), ("pc", C.c_int32), ("reserved2", C.c_int32),
                ("d", C.c_double), ("pinv_rtol", C.c_double)]


class _TreeOpts(C.Structure):
    _fields_ = [("ppl", C.c_int32), ("max_levels", C.c_int32), ("has_bbox", C.c_int32), ("reserved", C.c_int32),
                ("origin", C.c_double * 3), ("width", C.c_double)]


class _ServerOpts(C.Structure):
    _fields_ = [("slots", C.c_int32), ("ppl", C.c_int32), ("hbm_budget", C.c_int64), ("group_max", C.c_int32),
                ("reserved", C.c_int32), ("group_points", C.c_int64)]


class _Request(C.Structure):
    _fields_ = [("xyz", C.c_void_p), ("tau", C.c_void_p), ("n", C.c_int64), ("tol", C.c_double), ("kernel", C.c_int32),
                ("p", C.c_int32), ("outputs", C.c_int32), ("precision", C.c_int32), ("ppl", C.c_int32),
                ("pot", C.c_void_p), ("grad", C.c_void_p), ("kappa", C.c_double)]


class _StokesDensities(C.Structure):
    _fields_ = [("stokeslets", C.c_void_p), ("stresslets", C.c_void_p), ("stressvecs", C.c_void_p),
                ("doublets", C.c_void_p), ("weights", C.c_void_p)]


class _RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("p", C.c_int32), ("precision", C.c_int32), ("slot", C.c_int32),
                ("queued_s", C.c_double), ("run_s", C.c_double), ("latency_s", C.c_double),
                ("bytes_estimate", C.c_int64), ("plan_s", C.c_double), ("matvec_s", C.c_double),
                ("device_s", C.c_double), ("group", C.c_int32), ("reserved", C.c_int32)]


_lib = None
EXPORTS = (
    "fmmb_last_error", "fmmb_version", "fmmb_ctx_create", "fmmb_ctx_destroy", "fmmb_ctx_stream", "fmmb_ctx_synchronize",
    "fmmb_cache_create", "fmmb_cache_destroy", "fmmb_cache_base_width", "fmmb_plan_create", "fmmb_plan_create_dev",
    "fmmb_plan_destroy", "fmmb_plan_info", "fmmb_plan_box", "fmmb_plan_tree", "fmmb_plan_pairs", "fmmb_state_create",
    "fmmb_state_destroy", "fmmb_build_expansions", "fmmb_build_expansions_dev", "fmmb_evaluate_at_sources",
    "fmmb_evaluate_at_sources_dev", "fmmb_matvec", "fmmb_matvec_dev", "fmmb_evaluate", "fmmb_evaluate_dev",
    "fmmb_state_expansions", "fmmb_direct_dev", "fmmb_profile_matvec", "fmmb_direct_noalloc_dev",
    "fmmb_server_create", "fmmb_server_submit", "fmmb_server_wait", "fmmb_server_destroy", "fmmb_stokes_eval",
    "fmmb_stokes_eval_dev", "fmmb_build_expansions_dipoles", "fmmb_build_expansions_dipoles_dev",
    "fmmb_stokes_eval_densities", "fmmb_stokes_eval_densities_dev", "fmmb_stokes_eval_src_trg",
    "fmmb_stokes_eval_src_trg_dev", "fmmb_state_synchronize", "fmmb_test_m2l_stall",
    "fmmb_batch_plan_create", "fmmb_batch_plan_create_dev", "fmmb_batch_plan_instances", "fmmb_autotune",
    "fmmb_autotune_dev",
)


def library_path():
    return _LIB_PATH


def lib():
    """The loaded libfmmb.so; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"libfmmb.so is missing at {_LIB_PATH}: build it (python flexiblefmm.jl_b200/build.py)")
    L = C.CDLL(_LIB_PATH)
    vp, i64, i32, dp = C.c_void_p, C.c_int64, C.c_int, C.c_void_p
    L.fmmb_last_error.restype = C.c_char_p
    L.fmmb_version.restype = C.c_char_p
    sig = {
        "fmmb_ctx_create": [i32, C.POINTER(vp)],
        "fmmb_ctx_destroy": [vp],
        "fmmb_ctx_stream": [vp, C.POINTER(vp)],
        "fmmb_ctx_synchronize": [vp],
        "fmmb_cache_create": [vp, C.POINTER(_MethodDesc), C.POINTER(vp)],
        "fmmb_cache_destroy": [vp],
        "fmmb_cache_base_width": [vp, C.POINTER(C.c_double)],
        "fmmb_plan_create": [vp, dp, i64, C.POINTER(_TreeOpts), C.POINTER(vp)],
        "fmmb_plan_create_dev": [vp, dp, i64, C.POINTER(_TreeOpts), C.POINTER(vp)],
        "fmmb_plan_destroy": [vp],
        "fmmb_batch_plan_create": [vp, dp, dp, i64, C.POINTER(_TreeOpts), dp, C.POINTER(vp)],
        "fmmb_batch_plan_create_dev": [vp, dp, dp, i64, C.POINTER(_TreeOpts), dp, C.POINTER(vp)],
        "fmmb_batch_plan_instances": [vp, C.POINTER(i64), dp, dp, dp, dp],
        "fmmb_autotune": [vp, dp, dp, i64, i32, dp],
        "fmmb_autotune_dev": [vp, dp, dp, i64, i32, dp],
        "fmmb_plan_info": [vp, dp, i32],
        "fmmb_plan_box": [vp, dp, dp],
        "fmmb_plan_tree": [vp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp],
        "fmmb_plan_pairs": [vp, i32, dp, dp, dp, i64, C.POINTER(i64)],
        "fmmb_state_create": [vp, i32, C.POINTER(vp)],
        "fmmb_state_destroy": [vp],
        "fmmb_state_synchronize": [vp],
        "fmmb_test_m2l_stall": [i64, C.c_double],
        "fmmb_build_expansions": [vp, dp, dp, i64],
        "fmmb_build_expansions_dev": [vp, dp, dp, i64],
        "fmmb_evaluate_at_sources": [vp, i32, dp, dp],
        "fmmb_evaluate_at_sources_dev": [vp, i32, dp, dp],
        "fmmb_matvec": [vp, dp, dp, i64, i32, dp, dp],
        "fmmb_matvec_dev": [vp, dp, dp, i64, i32, dp, dp],
        "fmmb_evaluate": [vp, dp, i64, i32, dp, dp],
        "fmmb_evaluate_dev": [vp, dp, i64, i32, dp, dp],
        "fmmb_state_expansions": [vp, dp, dp],
        "fmmb_direct_dev": [vp, dp, dp, i64, dp, dp, i64, dp, dp],
        "fmmb_profile_matvec": [vp, dp, dp, i64, i32, dp, dp, dp, i32, C.POINTER(C.c_int)],
        "fmmb_direct_noalloc_dev": [vp, dp, dp, i64, dp, dp, i64, dp, dp],
        "fmmb_server_create": [i32, C.POINTER(_ServerOpts), C.POINTER(vp)],
        "fmmb_server_submit": [vp, C.POINTER(_Request), C.POINTER(i64)],
        "fmmb_server_wait": [vp, i64, C.c_double, C.POINTER(_RequestInfo)],
        "fmmb_server_destroy": [vp],
        "fmmb_stokes_eval": [vp, dp, dp, i64, dp],
        "fmmb_build_expansions_dipoles": [vp, dp, dp, dp, i64],
        "fmmb_build_expansions_dipoles_dev": [vp, dp, dp, dp, i64],
        "fmmb_stokes_eval_dev": [vp, dp, dp, i64, dp],
        "fmmb_stokes_eval_densities": [vp, dp, C.POINTER(_StokesDensities), i64, i32, dp],
        "fmmb_stokes_eval_densities_dev": [vp, dp, C.POINTER(_StokesDensities), i64, i32, dp],
        "fmmb_stokes_eval_src_trg": [vp, dp, C.POINTER(_StokesDensities), i64, dp, i64, i32, dp, dp],
        "fmmb_stokes_eval_src_trg_dev": [vp, dp, C.POINTER(_StokesDensities), i64, dp, i64, i32, dp, dp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = L
    return L


def _check(rc):
    if rc == FMMB_OK:
        return
    msg = lib().fmmb_last_error().decode()
    cls = {1: ArgumentError, 2: DimensionMismatch, 6: Unsupported}.get(rc, FMMBError)
    raise cls(rc, msg)


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _points(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 3:
        raise DimensionMismatch(2, f"expected an (N, 3) array of points, got {x.shape}")
    return x


def _points2(x):
    """(N, 2) points of a 2D method, embedded as (N, 3) in the plane z = 0."""
    x = np.asarray(x, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 2:
        raise DimensionMismatch(2, f"expected an (N, 2) array of points, got {x.shape}")
    return np.ascontiguousarray(np.concatenate([x, np.zeros((x.shape[0], 1))], axis=1))


def _pts(fmm_or_method, x):
    m = getattr(fmm_or_method, "method", fmm_or_method)
    return _points2(x) if getattr(m, "dimension", 3) == 2 else _points(x)


def _grad_out(fmm, g):
    return g[:, :2].copy() if getattr(fmm.method, "dimension", 3) == 2 else g


# ---------------------------------------------------------------- kernels, methods, outputs
class Laplace3D:
    """Free-space Laplace Green's function 1/(4π|t − s|) (src/kernels.jl:179-200)."""
    c = 1.0 / (4.0 * np.pi)


class Yukawa3D:
    """Modified Helmholtz (Yukawa) Green's function e^{−k|t − s|}/(4π|t − s|) (src/kernels.jl:224-242)."""
    c = 1.0 / (4.0 * np.pi)

    def __init__(self, k):
        self.k = float(k)


class Stokeslet3D:
    """The 3D Stokeslet (1/8π)(f/r + d(d·f)/r³) (src/kernels.jl:253-272)."""
    c = 1.0 / (8.0 * np.pi)


class StokesHarmonics:
    """StokesHarmonics(Stokeslet3D(); p=16) (src/operators/harmonics_stokes.jl:34-45): four
    solid-harmonic expansions per box; Stokeslet, stresslet and doublet densities, velocity,
    pressure and velocity-gradient outputs, FP64 path."""

    def __init__(self, kernel, p=16, tol=0.0):
        if not isinstance(kernel, Stokeslet3D):
            raise ArgumentError(1, "StokesHarmonics takes Stokeslet3D")
        if p < 1:
            raise ArgumentError(1, "p must be at least 1")
        if tol != 0:
            raise Unsupported(6, "low-rank translations (tol > 0) are not provided")
        self.kernel, self.p, self.tol = kernel, int(p), 0.0


class Laplace2D:
    """Free-space Laplace Green's function −log|t − s|/2π = c·log r², c = −1/(4π)
    (src/kernels.jl:53-66)."""
    c = -1.0 / (4.0 * np.pi)


class KernelIndependent:
    """KernelIndependent(kernel; nequiv=50, pinv_rtol=50·eps(Float64)) (src/operators/kifmm.jl:17-33):
    the 2D kernel-independent method on circles of nequiv equispaced points. Laplace2D; points
    (N, 2), gradients (N, 2); FP64."""
    dimension = 2

    def __init__(self, kernel, nequiv=50, pinv_rtol=None):
        if not isinstance(kernel, Laplace2D):
            raise ArgumentError(1, "the device circle KI method is written for Laplace2D")
        if nequiv < 4:
            raise ArgumentError(1, "nequiv must be at least 4")
        self.kernel, self.nequiv, self.p = kernel, int(nequiv), int(nequiv)
        self.pinv_rtol = 50 * float(np.finfo(np.float64).eps) if pinv_rtol is None else float(pinv_rtol)
        self.tol = 0.0

    @property
    def nsurface(self):
        return self.nequiv


class CubeKernelIndependent:
    """CubeKernelIndependent{3}(kernel; p=8, pc=2p, d=0.1, pinv_rtol=50·eps(Float32))
    (src/operators/cubeki.jl:35-42): the kernel-independent method on cube surfaces with p
    points per edge on the small surface (p³ − (p−2)³ points), pc on the large one, margin d;
    the M2L by FFT. Laplace3D only; the far field and the near field in FP32 on the "mixed"
    precision path, in FP64 on the "fp64" path (the spectra are FP32 on both)."""

    def __init__(self, kernel, p=8, pc=None, d=0.1, pinv_rtol=None):
        if not isinstance(kernel, Laplace3D):
            raise ArgumentError(1, "the device cube KI method is written for Laplace3D")
        pc = 2 * p if pc is None else pc
        if p < 2:
            raise ArgumentError(1, "p must be at least 2")
        if pc < p:
            raise ArgumentError(1, "pc must be at least p")
        if not (0 < d < 2 / 3):
            raise ArgumentError(1, "d must lie in (0, 2/3)")
        self.kernel, self.p, self.pc, self.d = kernel, int(p), int(pc), float(d)
        self.pinv_rtol = 50 * float(np.finfo(np.float32).eps) if pinv_rtol is None else float(pinv_rtol)
        self.tol = 0.0

    @property
    def nsurface(self):
        return self.p ** 3 - (self.p - 2) ** 3


class SphericalHarmonics:
    """SphericalHarmonics(kernel; p=16, tol=0) (src/operators/harmonics.jl:303-308)."""

    def __init__(self, kernel, p=16, tol=0.0):
        if not isinstance(kernel, (Laplace3D, Yukawa3D)):
            raise ArgumentError(1, "the device method is written for Laplace3D and Yukawa3D")
        if p < 1:
            raise ArgumentError(1, "p must be at least 1")
        if not (0 <= tol < 1):
            raise ArgumentError(1, "tol must lie in [0, 1)")
        self.kernel, self.p, self.tol = kernel, int(p), float(tol)


class Potential:
    pass


class Gradient:
    pass


def _output_flag(output):
    if isinstance(output, Potential) or output is Potential:
        return OUTPUT_POTENTIAL
    if isinstance(output, Gradient) or output is Gradient:
        return OUTPUT_GRADIENT
    raise ArgumentError(1, f"output {output!r} is not available with SphericalHarmonics")


# ---------------------------------------------------------------- device context
class Context:
    """One GPU and its stream (fmmb_ctx)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _check(lib().fmmb_ctx_create(int(device), C.byref(h)))
        self._h = h
        self.device = device

    @property
    def stream(self):
        s = C.c_void_p()
        _check(lib().fmmb_ctx_stream(self._h, C.byref(s)))
        return s.value

    def synchronize(self):
        _check(lib().fmmb_ctx_synchronize(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.fmmb_ctx_destroy(self._h)
            self._h = None


_default_ctx = {}


def default_context(device=0):
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]


class OperatorCache:
    """OperatorCache(method) (src/operators/cache.jl:19-22): shared by the plans built with it."""

    def __init__(self, method, ctx=None):
        self.method = method
        self.ctx = ctx or default_context()
        if isinstance(method, CubeKernelIndependent):
            d = _MethodDesc(2, KERNEL_LAPLACE3D, method.p, 0, 0.0, 0.0, method.pc, 0, method.d, method.pinv_rtol)
        elif isinstance(method, KernelIndependent):
            d = _MethodDesc(3, KERNEL_LAPLACE2D, method.nequiv, 0, 0.0, 0.0, 0, 0, 0.0, method.pinv_rtol)
        else:
            if isinstance(method, StokesHarmonics):
                kernel, kappa = KERNEL_STOKESLET3D, 0.0
            elif isinstance(method.kernel, Yukawa3D):
                kernel, kappa = KERNEL_YUKAWA3D, method.kernel.k
            else:
                kernel, kappa = KERNEL_LAPLACE3D, 0.0
            d = _MethodDesc(1, kernel, method.p, 0, method.tol, kappa)
        h = C.c_void_p()
        _check(lib().fmmb_cache_create(self.ctx._h, C.byref(d), C.byref(h)))
        self._h = h

    @property
    def W0(self):
        w = C.c_double()
        _check(lib().fmmb_cache_base_width(self._h, C.byref(w)))
        return w.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.fmmb_cache_destroy(self._h)
            self._h = None


class FMM:
    """FMM(method, sources; ppl=50, bbox=None, cache=OperatorCache(method), max_levels=30)
    (src/fmm.jl:31-49): the tree built on the device, the lists and the operators."""

    def __init__(self, method, sources, ppl=50, bbox=None, cache=None, max_levels=30, device_points=None):
        cache = cache if cache is not None else OperatorCache(method)
        if cache.method is not method:
            raise ArgumentError(1, "the cache was built for a different method")
        self.method, self.cache = method, cache
        opts = _TreeOpts()
        opts.ppl, opts.max_levels = int(ppl), int(max_levels)
        two_d = getattr(method, "dimension", 3) == 2
        if two_d and bbox is None:
            bbox = square_bbox2(sources)
        if bbox is not None:
            opts.has_bbox = 1
            if two_d:                            # the square as the cube's mid-plane z = 0
                opts.origin[0], opts.origin[1] = float(bbox[0][0]), float(bbox[0][1])
                opts.origin[2] = -float(bbox[1]) / 2
            else:
                for d in range(3):
                    opts.origin[d] = float(bbox[0][d])
            opts.width = float(bbox[1])
        h = C.c_void_p()
        if device_points is not None:           # (pointer, n) of a 3×n device array
            ptr, n = device_points
            _check(lib().fmmb_plan_create_dev(cache._h, C.c_void_p(ptr), int(n), C.byref(opts), C.byref(h)))
            self.N = int(n)
        else:
            x = _pts(method, sources)
            if x.shape[0] == 0:
                raise ArgumentError(1, "no points")
            _check(lib().fmmb_plan_create(cache._h, _ptr(x), x.shape[0], C.byref(opts), C.byref(h)))
            self.N = x.shape[0]
        self._h = h
        info = np.zeros(4 + 64, np.int64)
        _check(lib().fmmb_plan_info(self._h, _ptr(info), len(info)))
        self.nlevels, self.nnodes, self.npairs = int(info[0]), int(info[1]), int(info[3])
        self.level_start = info[4:4 + self.nlevels + 1].copy()
        self.block_targets = int(info[5 + self.nlevels])
        o = np.zeros(3)
        w = C.c_double()
        _check(lib().fmmb_plan_box(self._h, _ptr(o), C.byref(w)))
        self.origin, self.width = o, w.value

    def tree(self):
        """The flat tree as numpy arrays (node indices 0-based, -1 for none)."""
        n, N = self.nnodes, self.N
        t = dict(cell=np.zeros((n, 3), np.int32), level=np.zeros(n, np.int32), parent=np.zeros(n, np.int32),
                 child_first=np.zeros(n, np.int32), plo=np.zeros(n, np.int32), phi=np.zeros(n, np.int32),
                 flags=np.zeros(n, np.uint8), colleagues=np.zeros((n, 27), np.int32), perm=np.zeros(N, np.int32),
                 point_node=np.zeros(N, np.int32))
        _check(lib().fmmb_plan_tree(self._h, *[_ptr(t[k]) for k in ("cell", "level", "parent", "child_first", "plo", "phi",
                                                                       "flags", "colleagues", "perm", "point_node")]))
        fl = t.pop("flags")
        t["leaf"], t["ghost"] = (fl & 1).astype(np.uint8), ((fl >> 1) & 1).astype(np.uint8)
        t["xlist"], t["has_source"] = ((fl >> 2) & 1).astype(np.uint8), ((fl >> 3) & 1).astype(np.uint8)
        return t

    def pairs(self, level):
        n = C.c_int64()
        _check(lib().fmmb_plan_pairs(self._h, int(level), None, None, None, 0, C.byref(n)))
        t, s, f = (np.zeros(n.value, np.int32) for _ in range(3))
        if n.value:
            _check(lib().fmmb_plan_pairs(self._h, int(level), _ptr(t), _ptr(s), _ptr(f), n.value, C.byref(n)))
        return t, s, f

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.fmmb_plan_destroy(self._h)
            self._h = None


class BatchFMM(FMM):
    """Several independent FMMs of one method in one plan (fmmb_batch_plan_create): each point set
    of `sources` (a list of (N_i, 3) arrays) gets its own tree in its own box (`bbox`: None for each
    set's square_bbox, one (origin, width) for all, or a list of them), fitted in order as FMM(...)
    calls with the same cache would fit them. One tree build, one list build and one launch per
    pass and level serve every instance, and each instance's results are bitwise those of its own
    FMM. States, build_expansions and evaluate_at_sources take the plan like any other FMM, with
    the instances' points, densities and outputs concatenated in order (`concat`, `split`)."""

    def __init__(self, method, sources, ppl=50, bbox=None, cache=None, max_levels=30):
        cache = cache if cache is not None else OperatorCache(method)
        if cache.method is not method:
            raise ArgumentError(1, "the cache was built for a different method")
        if getattr(method, "dimension", 3) != 3:
            raise Unsupported(6, "batch plans take the 3D harmonic methods")
        self.method, self.cache = method, cache
        xs = [_pts(method, x) for x in sources]
        if not xs:
            raise ArgumentError(1, "no instances")
        self.counts = np.array([x.shape[0] for x in xs], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.sources = np.ascontiguousarray(np.concatenate(xs))
        self.ninst, self.N = len(xs), int(self.offsets[-1])
        opts = _TreeOpts()
        opts.ppl, opts.max_levels = int(ppl), int(max_levels)
        boxes = None
        if bbox is not None:
            bl = [bbox] * self.ninst if (len(bbox) == 2 and np.ndim(bbox[1]) == 0) else list(bbox)
            if len(bl) != self.ninst:
                raise DimensionMismatch(2, f"{len(bl)} boxes for {self.ninst} instances")
            boxes = np.array([[*map(float, b[0]), float(b[1])] for b in bl], np.float64)
        h = C.c_void_p()
        _check(lib().fmmb_batch_plan_create(cache._h, _ptr(self.sources), _ptr(self.counts), self.ninst,
                                            C.byref(opts), _ptr(boxes), C.byref(h)))
        self._h = h
        info = np.zeros(4 + 512, np.int64)
        _check(lib().fmmb_plan_info(self._h, _ptr(info), len(info)))
        self.nlevels, self.nnodes, self.npairs = int(info[0]), int(info[1]), int(info[3])
        self.level_start = info[4:4 + self.nlevels + 1].copy()
        self.block_targets = int(info[5 + self.nlevels])
        n = C.c_int64()
        self.boxes = np.zeros((self.ninst, 4))
        self.root_level = np.zeros(self.ninst, np.int32)
        self.node_instance = np.zeros(self.nnodes, np.int32)
        _check(lib().fmmb_batch_plan_instances(self._h, C.byref(n), None, _ptr(self.boxes), _ptr(self.root_level),
                                               _ptr(self.node_instance)))
        o = np.zeros(3)
        w = C.c_double()
        _check(lib().fmmb_plan_box(self._h, _ptr(o), C.byref(w)))
        self.origin, self.width = o, w.value

    def split(self, a):
        """The per-instance pieces of an array in the concatenated (instance) order."""
        return [a[self.offsets[i]:self.offsets[i + 1]] for i in range(self.ninst)]

    def concat(self, arrays):
        """The per-instance arrays (densities), concatenated in instance order."""
        if len(arrays) != self.ninst:
            raise DimensionMismatch(2, f"{len(arrays)} arrays for {self.ninst} instances")
        for i, a in enumerate(arrays):
            if len(a) != self.counts[i]:
                raise DimensionMismatch(2, f"instance {i}: {len(a)} values for {self.counts[i]} points")
        return np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in arrays]))


class FMMState:
    """FMMState (src/fmm.jl:64-94): the expansions of one right-hand side on the device.
    precision: "fp64" (the plain drop-in path) or "mixed"."""

    def __init__(self, fmm, precision="fp64"):
        self.fmm = fmm
        self.precision = precision
        prec = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}.get(precision)
        if prec is None:
            raise ArgumentError(1, f"unknown precision {precision!r}")
        h = C.c_void_p()
        _check(lib().fmmb_state_create(fmm._h, prec, C.byref(h)))
        self._h = h

    def expansions(self):
        """(multipoles, locals): nnodes × (p+1)² for Laplace3D, nnodes × 4 × (p+1)² for the
        Stokeslet (blocks Φ₁, Φ₂, Φ₃, Ψ̂)."""
        m = self.fmm.method
        n, np_ = self.fmm.nnodes, (m.nsurface if isinstance(m, CubeKernelIndependent) else (m.p + 1) ** 2)
        shape = (n, 4, np_) if isinstance(m, StokesHarmonics) else (n, np_)
        M = np.zeros(shape)
        Lc = np.zeros(shape)
        _check(lib().fmmb_state_expansions(self._h, _ptr(M), _ptr(Lc)))
        return M, Lc

    def synchronize(self):
        """Wait for the state's device work; raises FMMBError (Timeout) when a bounded wait of
        the tensor-core M2L gave up since the last report (fmmb_state_synchronize)."""
        _check(lib().fmmb_state_synchronize(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.fmmb_state_destroy(self._h)
            self._h = None


def _densities(tau, n):
    t = np.asarray(tau)
    if np.iscomplexobj(t) or t.dtype == object or t.ndim != 1:
        raise ArgumentError(1, f"densities of type {t.dtype} are not supported by SphericalHarmonics")
    t = np.ascontiguousarray(t, dtype=np.float64)
    if t.shape[0] != n:
        raise DimensionMismatch(2, f"expected {n} densities in group 1")
    return t


class Dipoles:
    """Dipole densities Dipole(d) per source (src/sources.jl:16-31): moments d (N, 3), field
    d·∇ₛG. As build_expansions' τ alone, or with charges as the tuple (charges, Dipoles(d))."""

    def __init__(self, d):
        self.d = np.ascontiguousarray(d, dtype=np.float64)


def autotune(state, sources, densities, tune_blocks=True):
    """The autotuner (fmmb_autotune): times the launch shapes of the state's matvec on these
    inputs (the plan's sources; charges, or (N, 3) Stokeslets), applies the fastest and records
    them for later plans and states of the same kind; returns the choices. The state's
    expansions must be built again afterwards."""
    x = _pts(state.fmm, sources)
    t = np.ascontiguousarray(densities, dtype=np.float64)
    out = np.zeros(5)
    _check(lib().fmmb_autotune(state._h, _ptr(x), _ptr(t), x.shape[0], 1 if tune_blocks else 0, _ptr(out)))
    return {"block_targets": int(out[0]), "f64_chunk_variant": int(out[1]), "near_warps": int(out[2]),
            "m2l_ms": float(out[3]), "near_ms": float(out[4])}


def build_expansions_(state, fmm, sources, tau):
    """build_expansions!(state, fmm, sources, τ) (src/fmm.jl:270-298); τ: charges (N,),
    Dipoles(d), or the tuple (charges, Dipoles(d))."""
    x = _pts(fmm, sources)
    if x.shape[0] != fmm.N:
        raise DimensionMismatch(2, f"expected {fmm.N} sources in group 1")
    charges, dip = tau, None
    if isinstance(tau, Dipoles):
        charges, dip = None, tau
    elif isinstance(tau, tuple):
        if len(tau) != 2 or not isinstance(tau[1], Dipoles):
            raise ArgumentError(1, "densities as a tuple: (charges, Dipoles(d))")
        charges, dip = tau
    if dip is None:
        t = _densities(charges, fmm.N)
        _check(lib().fmmb_build_expansions(state._h, _ptr(x), _ptr(t), fmm.N))
        return state
    if dip.d.shape != (fmm.N, 3):
        raise DimensionMismatch(2, f"expected {fmm.N} dipole moments (N, 3), got {dip.d.shape}")
    t = None if charges is None else _densities(charges, fmm.N)
    _check(lib().fmmb_build_expansions_dipoles(state._h, _ptr(x), _ptr(t), _ptr(dip.d), fmm.N))
    return state


def build_expansions(fmm, sources, tau, precision="fp64"):
    """build_expansions(fmm, sources, τ) -> FMMState (src/fmm.jl:306-314)."""
    return build_expansions_(FMMState(fmm, precision), fmm, sources, tau)


def evaluate_at_sources(fmm, state, g=1, output=Potential()):
    """evaluate_at_sources(fmm, state; output) (src/evaluate.jl:111-132), original order."""
    if g != 1:
        raise ArgumentError(1, f"group {g} of 1")
    flag = _output_flag(output)
    if flag == OUTPUT_POTENTIAL:
        out = np.zeros(fmm.N)
        _check(lib().fmmb_evaluate_at_sources(state._h, flag, _ptr(out), None))
    else:
        out = np.zeros((fmm.N, 3))
        _check(lib().fmmb_evaluate_at_sources(state._h, flag, None, _ptr(out)))
        out = _grad_out(fmm, out)
    return out


def evaluate_at_sources_both(fmm, state):
    """Potential and gradient at the sources in one pass."""
    pot, grad = np.zeros(fmm.N), np.zeros((fmm.N, 3))
    _check(lib().fmmb_evaluate_at_sources(state._h, 3, _ptr(pot), _ptr(grad)))
    return pot, _grad_out(fmm, grad)


def evaluate(fmm, state, targets, output=Potential()):
    """evaluate(fmm, state, targets; output) (src/evaluate.jl:81-102)."""
    flag = _output_flag(output)
    tg = _pts(fmm, targets)
    nt = tg.shape[0]
    if flag == OUTPUT_POTENTIAL:
        out = np.zeros(nt)
        _check(lib().fmmb_evaluate(state._h, _ptr(tg), nt, flag, _ptr(out), None))
    else:
        out = np.zeros((nt, 3))
        _check(lib().fmmb_evaluate(state._h, _ptr(tg), nt, flag, None, _ptr(out)))
        out = _grad_out(fmm, out)
    return out


def device_matvec(fmm, state, sources, tau, output=Potential()):
    """device_matvec!(out, plan, (sources, τ)) (src/device_passes.jl:619-640)."""
    flag = _output_flag(output)
    x = _pts(fmm, sources)
    t = _densities(tau, fmm.N)
    if x.shape[0] != fmm.N:
        raise DimensionMismatch(2, f"expected {fmm.N} sources")
    pot = np.zeros(fmm.N) if flag == OUTPUT_POTENTIAL else None
    grad = np.zeros((fmm.N, 3)) if flag == OUTPUT_GRADIENT else None
    _check(lib().fmmb_matvec(state._h, _ptr(x), _ptr(t), fmm.N, flag, _ptr(pot), _ptr(grad)))
    return pot if flag == OUTPUT_POTENTIAL else _grad_out(fmm, grad)


# ---------------------------------------------------------------- the request server
class Server:
    """A continuous-batching request server on one GPU (fmmb_server): requests of different
    sizes and tolerances are admitted in arrival order onto `slots` concurrent streams as slots
    and device memory (hbm_budget bytes; 0 = 80 % of the free memory) free up; a slot runs the
    front request with later queued ones of the same kind as one batch plan (up to group_max
    requests and group_points points; 0: 64 and 4e6; group_max=1: one at a time); ppl 0: the leaf
    size by each request's order and path. No counterpart in the reference, which runs one FMM
    per call."""

    def __init__(self, device=0, slots=2, ppl=0, hbm_budget=0, group_max=0, group_points=0):
        h = C.c_void_p()
        o = _ServerOpts(int(slots), int(ppl), int(hbm_budget), int(group_max), 0, int(group_points))
        _check(lib().fmmb_server_create(int(device), C.byref(o), C.byref(h)))
        self._h = h
        self._live = {}

    def submit(self, sources, tau, tol=1e-6, p=0, precision=None, gradient=True, ppl=0, kappa=None):
        """Queue one Laplace3D FMM (or Yukawa3D(kappa), FP64) at the sources (potential and,
        optionally, gradient, self excluded); returns a ticket. precision None: chosen from tol
        (FP64 below 1e-8); ppl 0: the server's."""
        x = _points(sources)
        t = np.ascontiguousarray(tau, dtype=np.float64)
        if t.shape != (x.shape[0],):
            raise DimensionMismatch(2, "one charge per source")
        pot = np.zeros(x.shape[0])
        grad = np.zeros((x.shape[0], 3)) if gradient else None
        prec = -1 if precision is None else {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}[precision]
        flags = OUTPUT_POTENTIAL | (OUTPUT_GRADIENT if gradient else 0)
        kernel = KERNEL_LAPLACE3D if kappa is None else KERNEL_YUKAWA3D
        r = _Request(x.ctypes.data, t.ctypes.data, x.shape[0], float(tol), kernel, int(p), flags, prec,
                     int(ppl), pot.ctypes.data, None if grad is None else grad.ctypes.data,
                     0.0 if kappa is None else float(kappa))
        return self._submit(r, (x, t, pot, grad))

    def submit_stokes(self, sources, stokeslets, tol=1e-6, p=0, ppl=0):
        """Queue one StokesHarmonics(Stokeslet3D()) FMM (velocities at the sources, self
        excluded, FP64); p 0: chosen from tol. wait() returns (velocities, None, info)."""
        x = _points(sources)
        f = np.ascontiguousarray(stokeslets, dtype=np.float64)
        if f.shape != x.shape:
            raise DimensionMismatch(2, f"stokeslets has shape {f.shape}, expected {x.shape}")
        vel = np.zeros_like(f)
        r = _Request(x.ctypes.data, f.ctypes.data, x.shape[0], float(tol), KERNEL_STOKESLET3D, int(p), 0, -1,
                     int(ppl), vel.ctypes.data, None)
        return self._submit(r, (x, f, vel, None))

    def _submit(self, r, bufs):
        ticket = C.c_int64()
        _check(lib().fmmb_server_submit(self._h, C.byref(r), C.byref(ticket)))
        self._live[ticket.value] = bufs     # the buffers stay alive until the request is waited for
        return ticket.value

    def wait(self, ticket, timeout=-1.0):
        """(pot, grad, info) of a request; info: p, precision, slot, queued_s, run_s, latency_s, plan_s
        (host time of its plan and state), matvec_s (host time of its matvec) and device_s (the
        matvec's time on the slot's stream)."""
        info = _RequestInfo()
        rc = lib().fmmb_server_wait(self._h, int(ticket), float(timeout), C.byref(info))
        if rc == 5 and info.latency_s == 0 and ticket in self._live:
            raise TimeoutError("the request is not done yet")
        bufs = self._live.pop(ticket)
        _check(rc)
        d = {k: getattr(info, k) for k, _ in _RequestInfo._fields_}
        d["precision"] = "fp64" if info.precision == PRECISION_FP64 else "mixed"
        return bufs[2], bufs[3], d

    def close(self):
        if self._h:
            _check(lib().fmmb_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- the Stokes plan API
def square_bbox2(points):
    """square_bbox of 2D points (src/tree/tree.jl:97-113): the square of their largest extent."""
    x = np.asarray(points, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 2:
        raise DimensionMismatch(2, f"expected an (N, 2) array of points, got {x.shape}")
    o, w = square_bbox(np.concatenate([x, np.zeros((x.shape[0], 1))], axis=1))
    return (o[0], o[1]), w


def square_bbox(points):
    """square_bbox(points) (src/tree/tree.jl:97-113): the cube of the points' largest extent
    about their midpoint, widened by 4 ulps at a time until every point is inside."""
    x = _points(points)
    if x.shape[0] == 0:
        raise ArgumentError(1, "no points")
    if not np.all(np.isfinite(x)):
        raise ArgumentError(1, "the points must be finite")
    lo, hi = x.min(axis=0), x.max(axis=0)
    w0 = float(np.max(hi - lo))
    if not np.isfinite(w0):
        raise ArgumentError(1, "the points' extent overflows")
    if not w0 > 0:
        w0 = 1.0
    c = lo + (hi - lo) / 2
    origin = c - w0 / 2
    for _ in range(64):
        if np.all(origin <= lo) and np.all(origin + w0 >= hi):
            return tuple(float(v) for v in origin), w0
        w0 *= 1 + 4 * np.finfo(np.float64).eps
        origin = c - w0 / 2
    raise ArgumentError(1, "could not fit a box around the points")


class StokesFMMPlan:
    """StokesFMMPlan(sources; targets, method=:harmonics, p=16, ppl, bbox) (src/stokes_api.jl:20-62):
    the tree and operators of StokesHarmonics(Stokeslet3D(); p) for a fixed geometry, reused by
    every stokes_fmm_eval; with targets, the box covers the sources and the targets (square_bbox of
    both, as the reference plan fits it) and stokes_fmm_eval evaluates there. The device path
    provides the :harmonics method with Stokeslet, stresslet and doublet densities and velocity and
    pressure outputs."""

    def __init__(self, sources, method="harmonics", p=16, ppl=200, bbox=None, targets=None, cache=None):
        if method != "harmonics":
            raise Unsupported(6, "the device path provides method=:harmonics")
        self.sources = _points(sources)
        self.targets = None if targets is None else _points(targets)
        if bbox is None:
            bbox = square_bbox(self.sources if self.targets is None
                               else np.concatenate([self.sources, self.targets]))
        # cache: an OperatorCache of a StokesHarmonics(Stokeslet3D(), p) method shared by plans
        self.method = cache.method if cache is not None else StokesHarmonics(Stokeslet3D(), p=p)
        self.fmm = FMM(self.method, self.sources, ppl=ppl, bbox=bbox, cache=cache)
        self.state = FMMState(self.fmm, "fp64")


class BatchStokesFMMPlan(StokesFMMPlan):
    """Many StokesFMMPlans in one batch plan (fmmb_batch_plan_create): StokesHarmonics(Stokeslet3D();
    p) self plans of the point sets in `sources` (a list of (N_i, 3) arrays), each in its own box
    (`bbox` as BatchFMM takes it; None: each set's square_bbox), computed together; stokes_fmm_eval
    takes the densities concatenated in instance order (plan.fmm.concat) and returns the outputs so
    (plan.fmm.split)."""

    def __init__(self, sources, method="harmonics", p=16, ppl=200, bbox=None, cache=None):
        if method != "harmonics":
            raise Unsupported(6, "the device path provides method=:harmonics")
        self.method = cache.method if cache is not None else StokesHarmonics(Stokeslet3D(), p=p)
        self.fmm = BatchFMM(self.method, sources, ppl=ppl, bbox=bbox, cache=cache)
        self.sources = self.fmm.sources
        self.targets = None
        self.state = FMMState(self.fmm, "fp64")


STOKES_VELOCITY = 0
STOKES_PRESSURE = 1
STOKES_GRADIENT = 2


def stokes_densities(n, weights=None, stokeslets=None, stresslets=None, stressvecs=None, doublets=None):
    """stokes_densities (src/stokes_api.jl:72-83): the checks of the density arrays, as float64
    arrays in C order ((n, 3) each, weights (n,)); returns them in the order of the C struct."""
    if (stresslets is None) != (stressvecs is None):
        raise ArgumentError(1, "stresslets and stressvecs must be given together")
    out = []
    for name, a in (("stokeslets", stokeslets), ("stresslets", stresslets), ("stressvecs", stressvecs),
                    ("doublets", doublets), ("weights", weights)):
        if a is None:
            out.append(None)
            continue
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape[0] != n:
            raise DimensionMismatch(2, f"{name} has length {a.shape[0]}, expected {n}")
        if name != "weights" and a.shape != (n, 3):
            raise DimensionMismatch(2, f"{name} has shape {a.shape}, expected ({n}, 3)")
        if name == "weights" and a.shape != (n,):
            raise DimensionMismatch(2, f"weights has shape {a.shape}, expected ({n},)")
        out.append(a)
    if out[0] is None and out[1] is None and out[3] is None:
        raise ArgumentError(1, "provide at least one of stokeslets, stresslets, doublets")
    return out


def _stokes_call(plan, sources, targets, at_sources, output, dens):
    x = plan.sources if sources is None else _points(sources)
    n = x.shape[0]
    outs = {"velocity": STOKES_VELOCITY, "pressure": STOKES_PRESSURE, "gradient": STOKES_GRADIENT}
    if output not in outs:
        raise Unsupported(6, "Stokes outputs are 'velocity', 'pressure' and 'gradient'")
    arrs = stokes_densities(n, **dens)
    tg = plan.targets if targets is None else _points(targets)
    shape = {"velocity": lambda m: (m, 3), "pressure": lambda m: (m,), "gradient": lambda m: (m, 3, 3)}[output]
    src = np.zeros(shape(n)) if at_sources else None
    trg = None if tg is None else np.zeros(shape(tg.shape[0]))
    if src is not None and trg is None and arrs[1] is None and arrs[3] is None and arrs[4] is None \
            and output == "velocity":
        _check(lib().fmmb_stokes_eval(plan.state._h, _ptr(x), _ptr(arrs[0]), n, _ptr(src)))
        return src, None
    d = _StokesDensities(*[None if a is None else a.ctypes.data for a in arrs])
    _check(lib().fmmb_stokes_eval_src_trg(plan.state._h, _ptr(x), C.byref(d), n, _ptr(tg),
                                          0 if tg is None else tg.shape[0], outs[output], _ptr(src), _ptr(trg)))
    return src, trg


def stokes_fmm_eval(plan, stokeslets=None, sources=None, stresslets=None, stressvecs=None, doublets=None,
                    weights=None, targets=None, output="velocity"):
    """stokes_fmm_eval!(out, plan; stokeslets, stresslets, stressvecs, doublets, weights, sources,
    targets, output) (src/stokes_api.jl:107-123): the velocities ((M, 3), output="velocity"),
    pressures ((M,), output="pressure") or velocity gradients ((M, 3, 3), [k, i, j] = ∂u_i/∂t_j,
    output="gradient") at the plan's targets (or `targets`, inside the plan's box), or at the
    sources of a self plan with the i = j term skipped. Stokeslets, stresslet
    strengths with their stressvecs, and doublets are (N, 3); weights (N,) multiply the
    stokeslets, stresslet strengths and doublets."""
    dens = dict(weights=weights, stokeslets=stokeslets, stresslets=stresslets, stressvecs=stressvecs,
                doublets=doublets)
    self_plan = plan.targets is None and targets is None
    src, trg = _stokes_call(plan, sources, targets, self_plan, output, dens)
    return src if self_plan else trg


def stokes_fmm_eval_src_trg(plan, stokeslets=None, sources=None, stresslets=None, stressvecs=None, doublets=None,
                            weights=None, targets=None, output="velocity"):
    """stokes_fmm_eval_src_trg!(vel_src, vel_trg, plan; ...) (src/stokes_api.jl:125-146): one
    expansion build, the outputs at the sources (i = j skipped) and at the plan's targets (or
    `targets`); returns (at the sources, at the targets)."""
    if plan.targets is None and targets is None:
        raise ArgumentError(1, "the plan has no targets")
    dens = dict(weights=weights, stokeslets=stokeslets, stresslets=stresslets, stressvecs=stressvecs,
                doublets=doublets)
    return _stokes_call(plan, sources, targets, True, output, dens)

def _test_m2l_stall(slab, wait_seconds=0.0):
    """Test hook of the bounded waits (fmmb_test_m2l_stall): the tensor-core M2L launches stop
    reporting K-step slab `slab` of every block as gathered (-1: back to normal) and wait at most
    `wait_seconds` (≤ 0: one second) on each barrier."""
    _check(lib().fmmb_test_m2l_stall(int(slab), float(wait_seconds)))
