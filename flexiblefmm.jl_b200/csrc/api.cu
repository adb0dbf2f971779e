// The C ABI of fmmb (include/fmmb.h): handles, validation with the reference's error
// semantics, host↔device staging, and the order of the passes.
#include <algorithm>
#include <cstring>

#include "passes.cuh"

using namespace fmmb;

// Handles may be destroyed in any order (a garbage collector finalises in any order): each
// handle counts the handles built on it (a context its caches, a cache its plans, a plan its
// states) and is freed once it was destroyed and nothing depends on it any more.
struct fmmb_ctx { Ctx c; int deps = 0; bool released = false; };
struct fmmb_cache { Cache c; fmmb_ctx* parent = nullptr; int deps = 0; bool released = false; };
struct fmmb_plan { Plan p; fmmb_cache* parent = nullptr; int deps = 0; bool released = false; };
struct fmmb_state { State s; fmmb_plan* parent = nullptr; };

namespace {

std::mutex g_handles;   // guards the dependency counts

void free_ctx_locked(fmmb_ctx* x) {
  if (!x->released || x->deps > 0) return;
  cudaSetDevice(x->c.device);
  if (x->c.own_stream) { cudaStreamSynchronize(x->c.stream); cudaStreamDestroy(x->c.stream); }
  delete x;
}
void free_cache_locked(fmmb_cache* x) {
  if (!x->released || x->deps > 0) return;
  fmmb_ctx* parent = x->parent;
  cudaSetDevice(parent->c.device);
  delete x;
  --parent->deps;
  free_ctx_locked(parent);
}
void free_plan_locked(fmmb_plan* x) {
  if (!x->released || x->deps > 0) return;
  fmmb_cache* parent = x->parent;
  cudaSetDevice(x->p.ctx->device);
  cudaStreamSynchronize(x->p.ctx->stream);
  delete x;
  --parent->deps;
  free_cache_locked(parent);
}

thread_local std::string g_last_error;

}  // namespace

namespace fmmb {
// the calling thread's message (the server hands a request's error to the thread that waits)
void set_last_error(const std::string& m) { g_last_error = m; }
// fixes a fresh cache's base width, so that every plan's box is snapped from its own points
// (ldexp(w, e) ⊇ the points) and not from the first box the cache saw
void fix_cache_base_width(fmmb_cache* c, double w) {
  std::lock_guard<std::mutex> lk(c->c.mu);
  if (std::isnan(c->c.W0)) c->c.W0 = w;
}
}  // namespace fmmb

namespace {

template <class F>
int guard(F&& f) {
  try {
    f();
    g_last_error.clear();
    return FMMB_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return FMMB_ERR_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return FMMB_ERR_DEVICE;
  }
}

// every entry point: the context's device, and its stream for the thread's device allocations
void set_device(const Ctx& c) {
  FMMB_CUDA(cudaSetDevice(c.device));
  g_alloc_stream = c.stream;
}

// A device-pointer argument must be memory the context's device can read and write: its own
// device memory, managed memory, or host memory allocated or registered by CUDA. A plain host
// pointer (or another device's memory) would fault in the first kernel that touches it; this
// turns that mistake into FMMB_ERR_ARGUMENT before anything is enqueued.
void require_device_ptr(const Ctx& c, const void* p, const char* what) {
  if (!p) return;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    throw Error(FMMB_ERR_ARGUMENT, std::string(what) + ": not a CUDA pointer");
  }
  const bool ok = (a.type == cudaMemoryTypeDevice && a.device == c.device) || a.type == cudaMemoryTypeManaged ||
                  (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr);
  require(ok, FMMB_ERR_ARGUMENT,
          std::string(what) + ": not memory the context's device can access (the _dev entry points take device pointers)");
}

// square_bbox (src/tree/tree.jl:97-114) from the points' bounds
void square_bbox(const double lo[3], const double hi[3], double origin[3], double& W0) {
  W0 = 0;
  for (int d = 0; d < 3; ++d) W0 = std::max(W0, hi[d] - lo[d]);
  require(std::isfinite(W0), FMMB_ERR_ARGUMENT, "the points' extent overflows");
  if (!(W0 > 0)) W0 = 1.0;
  double c[3];
  for (int d = 0; d < 3; ++d) c[d] = lo[d] + (hi[d] - lo[d]) / 2;
  for (int it = 0; it < 64; ++it) {
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      origin[d] = c[d] - W0 / 2;
      ok = ok && origin[d] <= lo[d] && origin[d] + W0 >= hi[d];
    }
    if (ok) return;
    W0 *= 1 + 4 * 2.220446049250313e-16;
  }
  throw Error(FMMB_ERR_ARGUMENT, "could not fit a box around the points");
}

// fit_box! (src/operators/cache.jl:293-313): a box of width ldexp(cache W0, e) containing the bounds
void fit_box(Cache& C, const double lo[3], const double hi[3], const double bo[3], double bw, double origin[3], double& W,
             int& e) {
  require(bw > 0, FMMB_ERR_ARGUMENT, "box width must be positive");
  for (int d = 0; d < 3; ++d)
    require(bo[d] <= lo[d] && bo[d] + bw >= hi[d], FMMB_ERR_ARGUMENT, "points lie outside the requested box");
  std::lock_guard<std::mutex> lk(C.mu);
  if (std::isnan(C.W0)) {
    C.W0 = bw;
    for (int d = 0; d < 3; ++d) origin[d] = bo[d];
    W = bw;
    e = 0;
    return;
  }
  int ex;
  double f = std::frexp(bw / C.W0, &ex);
  e = f == 0.5 ? ex - 1 : ex;
  double cen[3];
  for (int d = 0; d < 3; ++d) cen[d] = bo[d] + bw / 2;
  for (int it = 0; it < 2; ++it) {
    double Wn = std::ldexp(C.W0, e);
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      origin[d] = std::min(cen[d] - Wn / 2, lo[d]);
      ok = ok && origin[d] + Wn >= hi[d];
    }
    if (ok) { W = Wn; return; }
    ++e;
  }
  throw Error(FMMB_ERR_ARGUMENT, "could not fit a box");
}

void finish_plan(fmmb_cache* cache, std::unique_ptr<fmmb_plan>& h, const double* xyz, const fmmb_tree_opts* opts,
                 fmmb_plan** out);

void plan_from_device_points(fmmb_cache* cache, const double* xyz, int64_t n, const fmmb_tree_opts* opts, fmmb_plan** out) {
  require(cache && opts && out, FMMB_ERR_ARGUMENT, "null argument");
  Cache& C = cache->c;
  Ctx& ctx = *C.ctx;
  set_device(ctx);
  require(n > 0, FMMB_ERR_ARGUMENT, "no points");
  require(opts->ppl >= 1, FMMB_ERR_ARGUMENT, "ppl must be positive");
  require(opts->max_levels >= 1, FMMB_ERR_ARGUMENT, "max_levels must be positive");
  double lo[3], hi[3];
  int64_t bad = 0;
  bounds(ctx, xyz, n, lo, hi, &bad);
  require(bad == 0, FMMB_ERR_ARGUMENT, "the points must be finite");
  double bo[3], bw;
  if (opts->has_bbox) {
    for (int d = 0; d < 3; ++d) bo[d] = opts->origin[d];
    bw = opts->width;
  } else {
    square_bbox(lo, hi, bo, bw);
  }
  std::unique_ptr<fmmb_plan> h(new fmmb_plan());
  Plan& P = h->p;
  P.cache = &C;
  P.ctx = &ctx;
  P.N = n;
  fit_box(C, lo, hi, bo, bw, P.origin, P.W0, P.e0);
  finish_plan(cache, h, xyz, opts, out);
}

// the tree, scales, operators and lists of a plan whose box (or a batch's boxes) is fitted
void finish_plan(fmmb_cache* cache, std::unique_ptr<fmmb_plan>& h, const double* xyz, const fmmb_tree_opts* opts,
                 fmmb_plan** out) {
  Cache& C = cache->c;
  Ctx& ctx = *C.ctx;
  Plan& P = h->p;
  {
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.uploaded) {
      // the harmonic tables and the symmetry classes the lists use (the KI methods take order 2)
      C.host = build_operators(C.method == FMMB_METHOD_SPHERICAL_HARMONICS ? C.p : 2, C.W0);
      upload_operators(C);
    }
  }
  build_tree(P, xyz, opts->ppl, opts->max_levels);
  P.scale.resize(P.L);
  P.m2l_scale.resize(P.L);
  for (int l = 0; l < P.L; ++l) {
    int e = P.e0 - l;                       // the level's width is ldexp(cache W0, e)
    double lam = std::ldexp(1.0, e);        // w / W_ref (src/operators/harmonics.jl:414-418)
    P.scale[l] = e == 0 ? 1.0 / C.W0 : (1.0 / C.W0) / lam;
    // Yukawa3D is not homogeneous: its operators carry their width's c_K / w themselves
    P.m2l_scale[l] = C.kernel == FMMB_KERNEL_YUKAWA3D ? 1.0 : (e == 0 ? 1.0 : 1.0 / lam);
  }
  // the translation operators of every level: the cache's (homogeneous kernels), or the
  // level width's own (Yukawa3D, built on first use)
  P.lv_reps.assign(P.L, C.reps.p);
  P.lv_m2m.assign(P.L, C.m2m.p);
  P.lv_l2l.assign(P.L, C.l2l.p);
  if (C.kernel == FMMB_KERNEL_YUKAWA3D) yukawa_prepare(P);
  {
    std::vector<uint64_t> t(P.L);
    for (int l = 0; l < P.L; ++l) t[l] = (uint64_t)(uintptr_t)P.lv_reps[l];
    to_device(P.d_lv_reps, t, ctx.stream);
  }
  build_lists(P);
  if (C.method == FMMB_METHOD_CUBE_KI) ki_prepare(P);   // its operators, its target-major pairs
  if (C.method == FMMB_METHOD_KI_CIRCLE) kic_prepare(P);
  h->parent = cache;
  std::lock_guard<std::mutex> lk(g_handles);
  ++cache->deps;
  *out = h.release();
}

// a batch: ninst point sets (counts[i] points each, consecutive in xyz), each with its own box
// (boxes: 4 per instance, origin and width, or null for each set's square_bbox) fitted by
// fit_box! in instance order, as plans built one after another with the same cache would be
void batch_plan_from_device_points(fmmb_cache* cache, const double* xyz, const int64_t* counts, int64_t ninst,
                                   const fmmb_tree_opts* opts, const double* boxes, fmmb_plan** out) {
  require(cache && counts && opts && out, FMMB_ERR_ARGUMENT, "null argument");
  Cache& C = cache->c;
  Ctx& ctx = *C.ctx;
  set_device(ctx);
  require(ninst >= 1 && ninst < (1 << 24), FMMB_ERR_ARGUMENT, "the instance count must be in 1 .. 2^24 - 1");
  require(C.method == FMMB_METHOD_SPHERICAL_HARMONICS, FMMB_ERR_UNSUPPORTED,
          "batch plans take the harmonic methods (Laplace3D, Yukawa3D, Stokeslet3D)");
  require(opts->ppl >= 1, FMMB_ERR_ARGUMENT, "ppl must be positive");
  require(opts->max_levels >= 1, FMMB_ERR_ARGUMENT, "max_levels must be positive");
  std::vector<int64_t> off(ninst + 1, 0);
  for (int64_t i = 0; i < ninst; ++i) {
    require(counts[i] > 0, FMMB_ERR_ARGUMENT, "instance " + std::to_string(i) + " has no points");
    off[i + 1] = off[i] + counts[i];
    require(off[i + 1] < (1ll << 31) - 1, FMMB_ERR_ARGUMENT, "too many points for 32-bit indices");
  }
  std::vector<double> lo, hi;
  int64_t bad = 0;
  bounds_batch(ctx, xyz, off, lo, hi, &bad);
  require(bad == 0, FMMB_ERR_ARGUMENT, "the points must be finite");
  std::unique_ptr<fmmb_plan> h(new fmmb_plan());
  Plan& P = h->p;
  P.cache = &C;
  P.ctx = &ctx;
  P.N = off[ninst];
  P.ninst = (int)ninst;
  P.inst_off = off;
  P.inst_box.resize(4 * ninst);
  P.inst_e.resize(ninst);
  for (int64_t i = 0; i < ninst; ++i) {
    double bo[3], bw;
    if (boxes) {
      for (int d = 0; d < 3; ++d) bo[d] = boxes[4 * i + d];
      bw = boxes[4 * i + 3];
    } else {
      square_bbox(&lo[3 * i], &hi[3 * i], bo, bw);
    }
    double o[3], W;
    fit_box(C, &lo[3 * i], &hi[3 * i], bo, bw, o, W, P.inst_e[i]);
    for (int d = 0; d < 3; ++d) P.inst_box[4 * i + d] = o[d];
    P.inst_box[4 * i + 3] = W;
  }
  // the global levels: the widest root on level 0, every root on the level of its width
  const int64_t iw = std::max_element(P.inst_e.begin(), P.inst_e.end()) - P.inst_e.begin();
  P.e0 = P.inst_e[iw];
  P.W0 = P.inst_box[4 * iw + 3];
  for (int d = 0; d < 3; ++d) P.origin[d] = P.inst_box[4 * iw + d];
  P.inst_root.resize(ninst);
  for (int64_t i = 0; i < ninst; ++i) P.inst_root[i] = P.e0 - P.inst_e[i];
  finish_plan(cache, h, xyz, opts, out);
}

void check_outputs(int outputs) {
  require(outputs >= 1 && outputs <= 3, FMMB_ERR_ARGUMENT, "outputs must be POTENTIAL, GRADIENT or both");
}

// after a synchronisation: a bounded device wait that gave up is reported (once) as a timeout
void check_state_errors(State& S) {
  if (S.precision == FMMB_PRECISION_MIXED && mixed_error_flag(S))
    throw Error(FMMB_ERR_TIMEOUT, "a bounded wait of the tensor-core M2L gave up; the expansions are incomplete");
}

void state_build(State& S, const double* xyz, const double* tau) {
  gather_inputs(S, xyz, tau);
  upward_pass(S);
  downward_pass(S);
  S.built = true;
}

// build_expansions! + evaluate_at_sources! in one call: the near field (it needs the sources and
// charges only) runs on the state's side stream beside the upward and downward passes, and the
// far field adds to it after both; the outputs equal those of the two calls bit for bit
void matvec_sources(State& S, const double* xyz, const double* tau, int outputs, double* pot, double* grad) {
  Plan& P = *S.plan;
  gather_inputs(S, xyz, tau);
  if (!split_evaluation(S)) {
    upward_pass(S);
    downward_pass(S);
    S.built = true;
    evaluate_sources(S, outputs, pot, grad);
    return;
  }
  cudaStream_t s = P.ctx->stream;
  S.side.ensure();
  FMMB_CUDA(cudaEventRecord(S.side.fork, s));
  FMMB_CUDA(cudaStreamWaitEvent(S.side.s, S.side.fork, 0));
  near_sources(S, outputs, pot, grad, S.side.s);
  FMMB_CUDA(cudaEventRecord(S.side.join, S.side.s));
  try {
    upward_pass(S);
    downward_pass(S);
  } catch (...) {
    cudaStreamWaitEvent(s, S.side.join, 0);   // later work on the stream stays ordered after the near field
    throw;
  }
  S.built = true;
  FMMB_CUDA(cudaStreamWaitEvent(s, S.side.join, 0));
  far_sources(S, outputs, pot, grad);
}

}  // namespace

extern "C" {

const char* fmmb_last_error(void) { return g_last_error.c_str(); }
const char* fmmb_version(void) { return "fmmb 0.1 (sm_100a)"; }

int fmmb_ctx_create(int device, fmmb_ctx** out) {
  return guard([&] {
    require(out != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    int nd = 0;
    FMMB_CUDA(cudaGetDeviceCount(&nd));
    require(device >= 0 && device < nd, FMMB_ERR_ARGUMENT, "no such device");
    std::unique_ptr<fmmb_ctx> h(new fmmb_ctx());
    h->c.device = device;
    FMMB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FMMB_CUDA(cudaGetDeviceProperties(&prop, device));
    require(prop.major == 10, FMMB_ERR_UNSUPPORTED, "the library targets sm_100a (B200)");
    h->c.num_sms = prop.multiProcessorCount;
    // the highest priority: the split matvec's near field (on a lowest-priority side stream)
    // fills what the passes leave of the SMs
    int lo = 0, hi = 0;
    FMMB_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    FMMB_CUDA(cudaStreamCreateWithPriority(&h->c.stream, cudaStreamNonBlocking, hi));
    h->c.own_stream = true;
    init_device_constants(h->c.stream);
    // the device's stream-ordered pool keeps up to 16 GiB of freed memory mapped instead of
    // returning it at every synchronisation, so that the buffers of one plan after another (a
    // server's requests, a time-stepping loop) reuse memory instead of mapping it again
    {
      cudaMemPool_t pool;
      FMMB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
      uint64_t keep = 0;
      FMMB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
      if (keep < (16ull << 30)) {
        keep = 16ull << 30;
        FMMB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
      }
    }
    direct_noalloc_prepare();                       // the no-allocation scratch's address, at set-up
    *out = h.release();
  });
}

int fmmb_ctx_destroy(fmmb_ctx* ctx) {
  return guard([&] {
    if (!ctx) return;
    std::lock_guard<std::mutex> lk(g_handles);
    ctx->released = true;
    free_ctx_locked(ctx);
  });
}

int fmmb_ctx_stream(fmmb_ctx* ctx, void** stream) {
  return guard([&] {
    require(ctx && stream, FMMB_ERR_ARGUMENT, "null argument");
    *stream = (void*)ctx->c.stream;
  });
}

int fmmb_ctx_synchronize(fmmb_ctx* ctx) {  // state errors surface at the next host-pointer call on the state
  return guard([&] {
    require(ctx != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    set_device(ctx->c);
    FMMB_CUDA(cudaStreamSynchronize(ctx->c.stream));
  });
}

int fmmb_cache_create(fmmb_ctx* ctx, const fmmb_method_desc* m, fmmb_cache** out) {
  return guard([&] {
    require(ctx && m && out, FMMB_ERR_ARGUMENT, "null argument");
    require(m->method == FMMB_METHOD_SPHERICAL_HARMONICS || m->method == FMMB_METHOD_CUBE_KI ||
                m->method == FMMB_METHOD_KI_CIRCLE,
            FMMB_ERR_UNSUPPORTED,
            "the methods provided are SphericalHarmonics, StokesHarmonics, CubeKernelIndependent{3} and KernelIndependent");
    if (m->method == FMMB_METHOD_KI_CIRCLE) {
      // KernelIndependent(Laplace2D(); nequiv = p, pinv_rtol) (src/operators/kifmm.jl:17-33), FP64
      require(m->kernel == FMMB_KERNEL_LAPLACE2D, FMMB_ERR_UNSUPPORTED, "the circle KI method is provided for Laplace2D");
      require(m->p >= 4, FMMB_ERR_ARGUMENT, "nequiv must be at least 4");
      require(m->p <= 64, FMMB_ERR_UNSUPPORTED, "nequiv above 64 is not provided");
      require(m->pinv_rtol >= 0 && m->pinv_rtol < 1, FMMB_ERR_ARGUMENT, "pinv_rtol must lie in [0, 1)");
      std::unique_ptr<fmmb_cache> h(new fmmb_cache());
      h->c.ctx = &ctx->c;
      h->parent = ctx;
      h->c.method = FMMB_METHOD_KI_CIRCLE;
      h->c.p = m->p;
      h->c.np = m->p;
      h->c.ld = 64;
      h->c.kernel = FMMB_KERNEL_LAPLACE2D;
      h->c.nexp = 1;
      h->c.ki_rtol = m->pinv_rtol > 0 ? m->pinv_rtol : 50 * 2.220446049250313e-16;
      std::lock_guard<std::mutex> lk(g_handles);
      ++ctx->deps;
      *out = h.release();
      return;
    }
    if (m->method == FMMB_METHOD_CUBE_KI) {
      // CubeKernelIndependent{3}(Laplace3D(); p, pc = 2p, d = 0.1, pinv_rtol) (src/operators/cubeki.jl:35-42)
      require(m->kernel == FMMB_KERNEL_LAPLACE3D, FMMB_ERR_UNSUPPORTED, "the cube KI method is provided for Laplace3D");
      require(m->p >= 2, FMMB_ERR_ARGUMENT, "p must be at least 2");
      require(m->p <= KI_PMAX, FMMB_ERR_UNSUPPORTED, "p above 12 is not provided for the cube KI method");
      const int pc = m->pc ? m->pc : 2 * m->p;
      const double d = m->d != 0 ? m->d : 0.1;
      require(pc >= m->p, FMMB_ERR_ARGUMENT, "pc must be at least p");
      require(pc <= 2 * KI_PMAX, FMMB_ERR_UNSUPPORTED, "pc above 24 is not provided");
      require(d > 0 && d < 2.0 / 3.0, FMMB_ERR_ARGUMENT,
              "d must lie in (0, 2/3): the large surface, at (3 − 2d)w/2, must lie outside the small one, at (1 + d)w/2");
      require(m->pinv_rtol >= 0 && m->pinv_rtol < 1, FMMB_ERR_ARGUMENT, "pinv_rtol must lie in [0, 1)");
      std::unique_ptr<fmmb_cache> h(new fmmb_cache());
      h->c.ctx = &ctx->c;
      h->parent = ctx;
      h->c.method = FMMB_METHOD_CUBE_KI;
      h->c.p = m->p;
      h->c.np = 6 * m->p * m->p - 12 * m->p + 8;   // p³ − (p−2)³ small-surface points
      h->c.ld = (h->c.np + 63) / 64 * 64;
      h->c.kernel = FMMB_KERNEL_LAPLACE3D;
      h->c.nexp = 1;
      h->c.ki_pc = pc;
      h->c.ki_d = d;
      h->c.ki_rtol = m->pinv_rtol > 0 ? m->pinv_rtol : 50 * 1.1920928955078125e-7;
      std::lock_guard<std::mutex> lk(g_handles);
      ++ctx->deps;
      *out = h.release();
      return;
    }
    require(m->kernel == FMMB_KERNEL_LAPLACE3D || m->kernel == FMMB_KERNEL_YUKAWA3D || m->kernel == FMMB_KERNEL_STOKESLET3D,
            FMMB_ERR_UNSUPPORTED, "the kernels provided are Laplace3D, Yukawa3D and Stokeslet3D");
    if (m->kernel == FMMB_KERNEL_YUKAWA3D)
      require(std::isfinite(m->kappa) && m->kappa > 0, FMMB_ERR_ARGUMENT, "the Yukawa κ must be positive and finite");
    require(m->p >= 1, FMMB_ERR_ARGUMENT, "p must be at least 1");
    require(m->p <= PMAX, FMMB_ERR_UNSUPPORTED, "p above 20 is not provided");
    require(m->tol >= 0 && m->tol < 1, FMMB_ERR_ARGUMENT, "tol must lie in [0, 1)");
    require(m->tol == 0, FMMB_ERR_UNSUPPORTED, "low-rank class operators (tol > 0) are not provided");
    std::unique_ptr<fmmb_cache> h(new fmmb_cache());
    h->c.ctx = &ctx->c;
    h->parent = ctx;
    h->c.p = m->p;
    h->c.np = (m->p + 1) * (m->p + 1);
    h->c.ld = ld_of(m->p);
    h->c.kernel = m->kernel;
    h->c.nexp = m->kernel == FMMB_KERNEL_STOKESLET3D ? 4 : 1;   // StokesHarmonics: Φ₁..₃, Ψ̂
    h->c.kappa = m->kernel == FMMB_KERNEL_YUKAWA3D ? m->kappa : 0.0;
    std::lock_guard<std::mutex> lk(g_handles);
    ++ctx->deps;
    *out = h.release();
  });
}

int fmmb_cache_destroy(fmmb_cache* cache) {
  return guard([&] {
    if (!cache) return;
    std::lock_guard<std::mutex> lk(g_handles);
    cache->released = true;
    free_cache_locked(cache);
  });
}

int fmmb_cache_base_width(const fmmb_cache* cache, double* w) {
  return guard([&] {
    require(cache && w, FMMB_ERR_ARGUMENT, "null argument");
    *w = cache->c.W0;
  });
}

int fmmb_plan_create(fmmb_cache* cache, const double* xyz, int64_t n, const fmmb_tree_opts* opts, fmmb_plan** out) {
  return guard([&] {
    require(cache && xyz && opts && out, FMMB_ERR_ARGUMENT, "null argument");
    require(n > 0, FMMB_ERR_ARGUMENT, "no points");
    Ctx& ctx = *cache->c.ctx;
    set_device(ctx);
    DBuf<double> d(3 * n);
    FMMB_CUDA(cudaMemcpyAsync(d.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx.stream));
    plan_from_device_points(cache, d.p, n, opts, out);
  });
}

int fmmb_plan_create_dev(fmmb_cache* cache, const double* xyz_dev, int64_t n, const fmmb_tree_opts* opts, fmmb_plan** out) {
  return guard([&] {
    require(cache && xyz_dev != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    set_device(cache->parent->c);
    require_device_ptr(cache->parent->c, xyz_dev, "points");
    plan_from_device_points(cache, xyz_dev, n, opts, out);
  });
}

int fmmb_batch_plan_create(fmmb_cache* cache, const double* xyz, const int64_t* counts, int64_t ninst,
                           const fmmb_tree_opts* opts, const double* boxes, fmmb_plan** out) {
  return guard([&] {
    require(cache && xyz && counts && opts && out, FMMB_ERR_ARGUMENT, "null argument");
    require(ninst >= 1, FMMB_ERR_ARGUMENT, "no instances");
    int64_t n = 0;
    for (int64_t i = 0; i < ninst; ++i) {
      require(counts[i] > 0, FMMB_ERR_ARGUMENT, "instance " + std::to_string(i) + " has no points");
      n += counts[i];
    }
    Ctx& ctx = *cache->c.ctx;
    set_device(ctx);
    DBuf<double> d(3 * n);
    FMMB_CUDA(cudaMemcpyAsync(d.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx.stream));
    batch_plan_from_device_points(cache, d.p, counts, ninst, opts, boxes, out);
  });
}

int fmmb_batch_plan_create_dev(fmmb_cache* cache, const double* xyz_dev, const int64_t* counts, int64_t ninst,
                               const fmmb_tree_opts* opts, const double* boxes, fmmb_plan** out) {
  return guard([&] {
    require(cache && xyz_dev != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    set_device(cache->parent->c);
    require_device_ptr(cache->parent->c, xyz_dev, "points");
    batch_plan_from_device_points(cache, xyz_dev, counts, ninst, opts, boxes, out);
  });
}

int fmmb_batch_plan_instances(const fmmb_plan* plan, int64_t* ninst, int64_t* offsets, double* boxes, int32_t* root_level,
                              int32_t* node_instance) {
  return guard([&] {
    require(plan && ninst, FMMB_ERR_ARGUMENT, "null argument");
    const Plan& P = plan->p;
    *ninst = P.ninst;
    for (int i = 0; i < P.ninst; ++i) {
      if (offsets) offsets[i] = P.inst_off[i];
      if (boxes)
        for (int d = 0; d < 4; ++d) boxes[4 * i + d] = P.inst_box[4 * i + d];
      if (root_level) root_level[i] = P.inst_root[i];
    }
    if (offsets) offsets[P.ninst] = P.inst_off[P.ninst];
    if (node_instance) {
      if (P.ninst > 1) std::copy(P.h_inst.begin(), P.h_inst.end(), node_instance);
      else std::fill(node_instance, node_instance + P.nnodes, 0);
    }
  });
}

int fmmb_plan_destroy(fmmb_plan* plan) {
  return guard([&] {
    if (!plan) return;
    std::lock_guard<std::mutex> lk(g_handles);
    plan->released = true;
    free_plan_locked(plan);
  });
}

int fmmb_plan_info(const fmmb_plan* plan, int64_t* info, int cap) {
  return guard([&] {
    require(plan && info, FMMB_ERR_ARGUMENT, "null argument");
    const Plan& P = plan->p;
    require(cap >= 5 + P.L, FMMB_ERR_DIMENSION, "info needs 5 + levels entries");
    info[0] = P.L;
    info[1] = P.nnodes;
    info[2] = P.N;
    info[3] = P.npairs;
    for (int l = 0; l <= P.L; ++l) info[4 + l] = P.level_start[l];
    if (cap >= 6 + P.L) info[5 + P.L] = P.TB;     // the M2L blocks' targets, where there is room
  });
}

int fmmb_plan_box(const fmmb_plan* plan, double* origin3, double* width) {
  return guard([&] {
    require(plan && origin3 && width, FMMB_ERR_ARGUMENT, "null argument");
    for (int d = 0; d < 3; ++d) origin3[d] = plan->p.origin[d];
    *width = plan->p.W0;
  });
}

int fmmb_plan_tree(const fmmb_plan* plan, int32_t* cell, int32_t* level, int32_t* parent, int32_t* child_first,
                   int32_t* plo, int32_t* phi, uint8_t* flags, int32_t* colleagues, int32_t* perm, int32_t* point_node) {
  return guard([&] {
    require(plan != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    const Plan& P = plan->p;
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    int n = P.nnodes;
    if (cell || level) {
      std::vector<int4> c = to_host(P.cell.p, n, s);
      for (int i = 0; i < n; ++i) {
        if (cell) { cell[3 * i] = c[i].x; cell[3 * i + 1] = c[i].y; cell[3 * i + 2] = c[i].z; }
        if (level) level[i] = c[i].w;
      }
    }
    auto dl = [&](int32_t* dst, const int* src, size_t cnt) {
      if (dst) FMMB_CUDA(cudaMemcpyAsync(dst, src, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    };
    dl(parent, P.parent.p, n);
    dl(child_first, P.cf.p, n);
    dl(plo, P.plo.p, n);
    dl(phi, P.phi.p, n);
    dl(colleagues, P.col.p, (size_t)NCOL * n);
    dl(perm, P.perm.p, P.N);
    dl(point_node, P.point_node.p, P.N);
    if (flags) FMMB_CUDA(cudaMemcpyAsync(flags, P.flags.p, n, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
  });
}

int fmmb_plan_pairs(const fmmb_plan* plan, int level, int32_t* tgt, int32_t* src, int32_t* far, int64_t cap, int64_t* npairs) {
  return guard([&] {
    require(plan && npairs, FMMB_ERR_ARGUMENT, "null argument");
    const Plan& P = plan->p;
    require(level >= 0 && level < P.L, FMMB_ERR_ARGUMENT, "no such level");
    *npairs = P.level_pairs.empty() ? 0 : P.level_pairs[level];
    if (!tgt || !src || !far) return;
    require(cap >= *npairs, FMMB_ERR_DIMENSION, "the pair arrays are too short");
    set_device(*P.ctx);
    std::vector<int2> pr = to_host(P.pairs.p, (size_t)std::max<int64_t>(P.npairs, 0), P.ctx->stream);
    int64_t k = 0;
    for (const M2LBlock& b : P.h_blocks) {
      if (b.level != level) continue;
      int64_t next = P.npairs;
      for (const M2LBlock& b2 : P.h_blocks) if (b2.pair_base > b.pair_base) { next = std::min<int64_t>(next, b2.pair_base); }
      for (int64_t q = b.pair_base; q < next; ++q) {
        tgt[k] = b.first + (pr[q].y & 0xff);
        src[k] = pr[q].x;
        far[k] = pr[q].y >> 8;
        ++k;
      }
    }
  });
}

int fmmb_state_create(fmmb_plan* plan, int precision, fmmb_state** out) {
  return guard([&] {
    require(plan && out, FMMB_ERR_ARGUMENT, "null argument");
    require(precision == FMMB_PRECISION_FP64 || precision == FMMB_PRECISION_MIXED, FMMB_ERR_ARGUMENT, "unknown precision path");
    Plan& P = plan->p;
    require(P.cache->kernel != FMMB_KERNEL_STOKESLET3D || precision == FMMB_PRECISION_FP64, FMMB_ERR_UNSUPPORTED,
            "the Stokeslet method runs on the FP64 path");
    require(P.cache->kernel != FMMB_KERNEL_YUKAWA3D || precision == FMMB_PRECISION_FP64 ||
                P.cache->method == FMMB_METHOD_SPHERICAL_HARMONICS,
            FMMB_ERR_UNSUPPORTED, "the Yukawa method's mixed path is the harmonic one");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    std::unique_ptr<fmmb_state> h(new fmmb_state());
    State& S = h->s;
    S.plan = &P;
    S.precision = precision;
    S.xs.alloc(P.N); S.ys.alloc(P.N); S.zs.alloc(P.N); S.q.alloc(P.N);
    size_t ne = (size_t)P.nnodes * P.cache->ld * P.cache->nexp;
    S.M.alloc(ne);
    S.Pl.alloc(ne);
    FMMB_CUDA(cudaMemsetAsync(S.M.p, 0, S.M.bytes(), s));
    FMMB_CUDA(cudaMemsetAsync(S.Pl.p, 0, S.Pl.bytes(), s));
    if (P.cache->method == FMMB_METHOD_CUBE_KI) {
      ki_state(S);   // its spectra, check and local buffers; the precision selects the far field's and P2P's
    } else if (P.cache->method == FMMB_METHOD_KI_CIRCLE) {
      kic_state(S);
    } else if (precision == FMMB_PRECISION_MIXED) {
      std::lock_guard<std::mutex> lk(P.cache->mu);
      prepare_mixed_operators(*P.cache);
      prepare_mixed_levels(P);
    }
    apply_tuned_state(S);                         // the launch shapes tuned for states of this kind
    FMMB_CUDA(cudaStreamSynchronize(s));
    h->parent = plan;
    std::lock_guard<std::mutex> lk(g_handles);
    ++plan->deps;
    *out = h.release();
  });
}

int fmmb_autotune_dev(fmmb_state* state, const double* xyz_dev, const double* tau_dev, int64_t n, int tune_blocks,
                      double* out) {
  return guard([&] {
    require(state && xyz_dev && tau_dev, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    set_device(*S.plan->ctx);
    require(n == S.plan->N, FMMB_ERR_DIMENSION, "the points must be the plan's");
    require_device_ptr(*S.plan->ctx, xyz_dev, "points");
    require_device_ptr(*S.plan->ctx, tau_dev, "densities");
    autotune(S, xyz_dev, tau_dev, tune_blocks != 0, out);
    check_state_errors(S);
  });
}

int fmmb_autotune(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int tune_blocks, double* out) {
  return guard([&] {
    require(state && xyz && tau, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    Ctx& ctx = *S.plan->ctx;
    set_device(ctx);
    require(n == S.plan->N, FMMB_ERR_DIMENSION, "the points must be the plan's");
    const int dens = S.plan->cache->kernel == FMMB_KERNEL_STOKESLET3D ? 3 : 1;
    DBuf<double> dx(3 * n), dt(dens * n);
    FMMB_CUDA(cudaMemcpyAsync(dx.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx.stream));
    FMMB_CUDA(cudaMemcpyAsync(dt.p, tau, sizeof(double) * dens * n, cudaMemcpyHostToDevice, ctx.stream));
    autotune(S, dx.p, dt.p, tune_blocks != 0, out);
    check_state_errors(S);
  });
}

int fmmb_state_destroy(fmmb_state* state) {
  return guard([&] {
    if (!state) return;
    std::lock_guard<std::mutex> lk(g_handles);
    fmmb_plan* parent = state->parent;
    cudaSetDevice(parent->p.ctx->device);
    cudaStreamSynchronize(parent->p.ctx->stream);
    delete state;
    --parent->deps;
    free_plan_locked(parent);
  });
}

int fmmb_build_expansions_dev(fmmb_state* state, const double* xyz, const double* tau, int64_t n) {
  return guard([&] {
    require(state && xyz && tau, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    require(n == S.plan->N, FMMB_ERR_DIMENSION, "expected " + std::to_string(S.plan->N) + " sources and densities");
    set_device(*S.plan->ctx);
    require_device_ptr(*S.plan->ctx, xyz, "points");
    require_device_ptr(*S.plan->ctx, tau, "densities");
    state_build(S, xyz, tau);
  });
}

int fmmb_build_expansions(fmmb_state* state, const double* xyz, const double* tau, int64_t n) {
  return guard([&] {
    require(state && xyz && tau, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    Plan& P = *S.plan;
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and densities");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    if (S.h_in_xyz.n < (size_t)(3 * n)) { S.h_in_xyz.alloc(3 * n); S.h_in_tau.alloc(n); }
    FMMB_CUDA(cudaMemcpyAsync(S.h_in_xyz.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(S.h_in_tau.p, tau, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    state_build(S, S.h_in_xyz.p, S.h_in_tau.p);
    FMMB_CUDA(cudaStreamSynchronize(s));
    check_state_errors(S);
  });
}

int fmmb_build_expansions_dipoles_dev(fmmb_state* state, const double* xyz, const double* tau, const double* dipoles,
                                      int64_t n) {
  return guard([&] {
    require(state && xyz && (tau || dipoles), FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    require(n == S.plan->N, FMMB_ERR_DIMENSION, "expected " + std::to_string(S.plan->N) + " sources and densities");
    set_device(*S.plan->ctx);
    require_device_ptr(*S.plan->ctx, xyz, "points");
    if (tau) require_device_ptr(*S.plan->ctx, tau, "charges");
    if (dipoles) require_device_ptr(*S.plan->ctx, dipoles, "dipoles");
    gather_inputs_dipoles(S, xyz, tau, dipoles);
    upward_pass(S);
    downward_pass(S);
    S.built = true;
  });
}

int fmmb_build_expansions_dipoles(fmmb_state* state, const double* xyz, const double* tau, const double* dipoles, int64_t n) {
  return guard([&] {
    require(state && xyz && (tau || dipoles), FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    Plan& P = *S.plan;
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and densities");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    DBuf<double> d_xyz(3 * n), d_tau(tau ? n : 0), d_dip(dipoles ? 3 * n : 0);
    FMMB_CUDA(cudaMemcpyAsync(d_xyz.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    if (tau) FMMB_CUDA(cudaMemcpyAsync(d_tau.p, tau, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (dipoles) FMMB_CUDA(cudaMemcpyAsync(d_dip.p, dipoles, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    gather_inputs_dipoles(S, d_xyz.p, tau ? d_tau.p : nullptr, dipoles ? d_dip.p : nullptr);
    upward_pass(S);
    downward_pass(S);
    S.built = true;
    FMMB_CUDA(cudaStreamSynchronize(s));
    check_state_errors(S);
  });
}

int fmmb_evaluate_at_sources_dev(fmmb_state* state, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    State& S = state->s;
    require(S.built, FMMB_ERR_ARGUMENT, "the state has no expansions yet (build_expansions first)");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*S.plan->ctx);
    if (outputs & FMMB_OUTPUT_POTENTIAL) require_device_ptr(*S.plan->ctx, pot, "potential output");
    if (outputs & FMMB_OUTPUT_GRADIENT) require_device_ptr(*S.plan->ctx, grad, "gradient output");
    evaluate_sources(S, outputs, pot, grad);
  });
}

int fmmb_evaluate_at_sources(fmmb_state* state, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    State& S = state->s;
    Plan& P = *S.plan;
    require(S.built, FMMB_ERR_ARGUMENT, "the state has no expansions yet (build_expansions first)");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    if (S.d_pot.n < (size_t)P.N) { S.d_pot.alloc(P.N); S.d_grad.alloc(3 * P.N); }
    evaluate_sources(S, outputs, S.d_pot.p, S.d_grad.p);
    if (outputs & FMMB_OUTPUT_POTENTIAL)
      FMMB_CUDA(cudaMemcpyAsync(pot, S.d_pot.p, sizeof(double) * P.N, cudaMemcpyDeviceToHost, s));
    if (outputs & FMMB_OUTPUT_GRADIENT)
      FMMB_CUDA(cudaMemcpyAsync(grad, S.d_grad.p, sizeof(double) * 3 * P.N, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    check_state_errors(S);
  });
}

int fmmb_matvec_dev(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state && xyz && tau, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    State& S = state->s;
    require(n == S.plan->N, FMMB_ERR_DIMENSION, "expected " + std::to_string(S.plan->N) + " sources and densities");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*S.plan->ctx);
    require_device_ptr(*S.plan->ctx, xyz, "points");
    require_device_ptr(*S.plan->ctx, tau, "densities");
    if (outputs & FMMB_OUTPUT_POTENTIAL) require_device_ptr(*S.plan->ctx, pot, "potential output");
    if (outputs & FMMB_OUTPUT_GRADIENT) require_device_ptr(*S.plan->ctx, grad, "gradient output");
    matvec_sources(S, xyz, tau, outputs, pot, grad);
  });
}

int fmmb_state_synchronize(fmmb_state* state) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    set_device(*S.plan->ctx);
    if (S.side.s) FMMB_CUDA(cudaStreamSynchronize(S.side.s));
    FMMB_CUDA(cudaStreamSynchronize(S.plan->ctx->stream));
    check_state_errors(S);
  });
}

int fmmb_test_m2l_stall(int64_t slab, double wait_seconds) {
  return guard([&] { set_m2l_stall((long long)slab, wait_seconds); });
}

int fmmb_matvec(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state && xyz && tau, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    State& S = state->s;
    Plan& P = *S.plan;
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and densities");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    if (S.h_in_xyz.n < (size_t)(3 * n)) { S.h_in_xyz.alloc(3 * n); S.h_in_tau.alloc(n); }
    if (S.d_pot.n < (size_t)P.N) { S.d_pot.alloc(P.N); S.d_grad.alloc(3 * P.N); }
    FMMB_CUDA(cudaMemcpyAsync(S.h_in_xyz.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(S.h_in_tau.p, tau, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    matvec_sources(S, S.h_in_xyz.p, S.h_in_tau.p, outputs, S.d_pot.p, S.d_grad.p);
    if (outputs & FMMB_OUTPUT_POTENTIAL)
      FMMB_CUDA(cudaMemcpyAsync(pot, S.d_pot.p, sizeof(double) * P.N, cudaMemcpyDeviceToHost, s));
    if (outputs & FMMB_OUTPUT_GRADIENT)
      FMMB_CUDA(cudaMemcpyAsync(grad, S.d_grad.p, sizeof(double) * 3 * P.N, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    check_state_errors(S);
  });
}

int fmmb_evaluate_dev(fmmb_state* state, const double* tg, int64_t nt, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    require(nt >= 0, FMMB_ERR_DIMENSION, "negative target count");
    State& S = state->s;
    require(S.built, FMMB_ERR_ARGUMENT, "the state has no expansions yet (build_expansions first)");
    if (nt == 0) return;
    require(tg != nullptr, FMMB_ERR_ARGUMENT, "null targets");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*S.plan->ctx);
    require_device_ptr(*S.plan->ctx, tg, "targets");
    if (outputs & FMMB_OUTPUT_POTENTIAL) require_device_ptr(*S.plan->ctx, pot, "potential output");
    if (outputs & FMMB_OUTPUT_GRADIENT) require_device_ptr(*S.plan->ctx, grad, "gradient output");
    evaluate_targets(S, tg, nt, outputs, pot, grad);
  });
}

int fmmb_evaluate(fmmb_state* state, const double* tg, int64_t nt, int outputs, double* pot, double* grad) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    check_outputs(outputs);
    require(nt >= 0, FMMB_ERR_DIMENSION, "negative target count");
    State& S = state->s;
    Plan& P = *S.plan;
    require(S.built, FMMB_ERR_ARGUMENT, "the state has no expansions yet (build_expansions first)");
    if (nt == 0) return;
    require(tg != nullptr, FMMB_ERR_ARGUMENT, "null targets");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    DBuf<double> dt(3 * nt), dp(nt), dg(3 * nt);
    FMMB_CUDA(cudaMemcpyAsync(dt.p, tg, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s));
    evaluate_targets(S, dt.p, nt, outputs, dp.p, dg.p);
    if (outputs & FMMB_OUTPUT_POTENTIAL) FMMB_CUDA(cudaMemcpyAsync(pot, dp.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
    if (outputs & FMMB_OUTPUT_GRADIENT) FMMB_CUDA(cudaMemcpyAsync(grad, dg.p, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    check_state_errors(S);
  });
}

int fmmb_profile_matvec(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int outputs, double* pot,
                        double* grad, double* stage_ms, int cap, int* launches) {
  return guard([&] {
    require(state && xyz && tau && stage_ms, FMMB_ERR_ARGUMENT, "null argument");
    require(cap >= 6, FMMB_ERR_DIMENSION, "stage_ms needs 6 entries");
    check_outputs(outputs);
    State& S = state->s;
    Plan& P = *S.plan;
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and densities");
    require(!(outputs & FMMB_OUTPUT_POTENTIAL) || pot, FMMB_ERR_ARGUMENT, "null potential output");
    require(!(outputs & FMMB_OUTPUT_GRADIENT) || grad, FMMB_ERR_ARGUMENT, "null gradient output");
    set_device(*P.ctx);
    require_device_ptr(*P.ctx, xyz, "points");
    require_device_ptr(*P.ctx, tau, "densities");
    if (outputs & FMMB_OUTPUT_POTENTIAL) require_device_ptr(*P.ctx, pot, "potential output");
    if (outputs & FMMB_OUTPUT_GRADIENT) require_device_ptr(*P.ctx, grad, "gradient output");
    cudaStream_t s = P.ctx->stream;
    cudaEvent_t ev[7];
    for (auto& e : ev) FMMB_CUDA(cudaEventCreate(&e));
    int nl = 0;
    FMMB_CUDA(cudaEventRecord(ev[0], s));
    gather_inputs(S, xyz, tau);
    nl += 1;
    FMMB_CUDA(cudaEventRecord(ev[1], s));
    nl += p2m(S);
    FMMB_CUDA(cudaEventRecord(ev[2], s));
    nl += m2m_sweep(S);
    FMMB_CUDA(cudaEventRecord(ev[3], s));
    nl += m2l_stage(S);
    FMMB_CUDA(cudaEventRecord(ev[4], s));
    nl += l2l_sweep(S);
    FMMB_CUDA(cudaEventRecord(ev[5], s));
    S.built = true;
    evaluate_sources(S, outputs, pot, grad);
    nl += P.n_leaves > 0;
    FMMB_CUDA(cudaEventRecord(ev[6], s));
    FMMB_CUDA(cudaEventSynchronize(ev[6]));
    for (int i = 0; i < 6; ++i) {
      float ms = 0;
      FMMB_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      stage_ms[i] = ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    check_state_errors(S);
    if (launches) *launches = nl;
  });
}

int fmmb_state_expansions(const fmmb_state* state, double* multipoles, double* locals) {
  return guard([&] {
    require(state != nullptr, FMMB_ERR_ARGUMENT, "null argument");
    const State& S = state->s;
    const Plan& P = *S.plan;
    set_device(*P.ctx);
    // per node the nexp blocks of NP coefficients (Stokeslet states: Φ₁, Φ₂, Φ₃, Ψ̂)
    const int LD = P.cache->ld, NP = P.cache->np, n = P.nnodes, ne = P.cache->nexp;
    cudaStream_t s = P.ctx->stream;
    if (multipoles) {
      std::vector<double> h = to_host(S.M.p, (size_t)n * ne * LD, s);
      for (int i = 0; i < n; ++i)
        for (int a = 0; a < ne; ++a)
          std::memcpy(multipoles + ((size_t)i * ne + a) * NP, &h[((size_t)i * ne + a) * LD], sizeof(double) * NP);
    }
    if (locals) {
      std::vector<double> h = to_host(S.Pl.p, (size_t)n * ne * LD, s);
      for (int i = 0; i < n; ++i)
        for (int a = 0; a < ne; ++a) {
          double* dst = locals + ((size_t)i * ne + a) * NP;
          if (P.h_flags[i] & F_LEAF) std::memcpy(dst, &h[((size_t)i * ne + a) * LD], sizeof(double) * NP);
          else std::memset(dst, 0, sizeof(double) * NP);
        }
    }
  });
}

// stokes_fmm_eval!(velocities, plan; stokeslets) at the sources (src/stokes_api.jl:131-150):
// build_expansions! then evaluate_at_sources!, self excluded
int fmmb_stokes_eval_dev(fmmb_state* state, const double* xyz, const double* stokeslets, int64_t n, double* velocity) {
  return guard([&] {
    require(state && xyz && stokeslets && velocity, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    Plan& P = *S.plan;
    require(P.cache->kernel == FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "the state is not a Stokeslet state");
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and Stokeslets");
    set_device(*P.ctx);
    require_device_ptr(*P.ctx, xyz, "sources");
    require_device_ptr(*P.ctx, stokeslets, "stokeslets");
    require_device_ptr(*P.ctx, velocity, "velocities");
    StokesDensities d;
    d.stokeslets = stokeslets;
    stokes_build(S, xyz, d);
    stokes_evaluate_sources(S, FMMB_STOKES_VELOCITY, velocity);
  });
}

int fmmb_stokes_eval(fmmb_state* state, const double* xyz, const double* stokeslets, int64_t n, double* velocity) {
  return guard([&] {
    require(state && xyz && stokeslets && velocity, FMMB_ERR_ARGUMENT, "null argument");
    State& S = state->s;
    Plan& P = *S.plan;
    require(P.cache->kernel == FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "the state is not a Stokeslet state");
    require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and Stokeslets");
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    DBuf<double> x(3 * n), f(3 * n), v(3 * n);
    FMMB_CUDA(cudaMemcpyAsync(x.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(f.p, stokeslets, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    StokesDensities d;
    d.stokeslets = f.p;
    stokes_build(S, x.p, d);
    stokes_evaluate_sources(S, FMMB_STOKES_VELOCITY, v.p);
    FMMB_CUDA(cudaMemcpyAsync(velocity, v.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
  });
}

namespace {

// the checks of stokes_densities (src/stokes_api.jl:72-83) and of the state
void check_stokes_call(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n, int output,
                       const double* targets, int64_t nt, const double* out_src, const double* out_trg) {
  require(state && xyz && dens, FMMB_ERR_ARGUMENT, "null argument");
  require(out_src || out_trg, FMMB_ERR_ARGUMENT, "no output");
  require(nt >= 0, FMMB_ERR_DIMENSION, "negative target count");
  require(!out_trg || nt == 0 || targets, FMMB_ERR_ARGUMENT, "null targets");
  require((dens->stresslets == nullptr) == (dens->stressvecs == nullptr), FMMB_ERR_ARGUMENT,
          "stresslets and stressvecs must be given together");
  require(dens->stokeslets || dens->stresslets || dens->doublets, FMMB_ERR_ARGUMENT,
          "provide at least one of stokeslets, stresslets, doublets");
  require(output == FMMB_STOKES_VELOCITY || output == FMMB_STOKES_PRESSURE || output == FMMB_STOKES_GRADIENT,
          FMMB_ERR_UNSUPPORTED, "Stokes outputs are the velocity, the pressure and the velocity gradient");
  Plan& P = *state->s.plan;
  require(P.cache->kernel == FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "the state is not a Stokeslet state");
  require(n == P.N, FMMB_ERR_DIMENSION, "expected " + std::to_string(P.N) + " sources and densities");
}

// build_expansions! then the evaluations asked for (device pointers)
void stokes_run(State& S, const double* xyz, const StokesDensities& d, const double* tg, int64_t nt, int output,
                double* out_src, double* out_trg) {
  stokes_build(S, xyz, d);
  if (out_src) stokes_evaluate_sources(S, output, out_src);
  if (out_trg && nt > 0) stokes_evaluate_targets(S, tg, nt, output, out_trg);
}

int stokes_dev(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n, const double* tg,
               int64_t nt, int output, double* out_src, double* out_trg) {
  return guard([&] {
    check_stokes_call(state, xyz, dens, n, output, tg, nt, out_src, out_trg);
    State& S = state->s;
    Plan& P = *S.plan;
    set_device(*P.ctx);
    require_device_ptr(*P.ctx, xyz, "sources");
    const double* arrays[5] = {dens->stokeslets, dens->stresslets, dens->stressvecs, dens->doublets, dens->weights};
    for (const double* a : arrays)
      if (a) require_device_ptr(*P.ctx, a, "densities");
    if (out_src) require_device_ptr(*P.ctx, out_src, "outputs");
    if (out_trg && nt > 0) {
      require_device_ptr(*P.ctx, tg, "targets");
      require_device_ptr(*P.ctx, out_trg, "outputs");
    }
    StokesDensities d;
    d.stokeslets = dens->stokeslets;
    d.stresslets = dens->stresslets;
    d.stressvecs = dens->stressvecs;
    d.doublets = dens->doublets;
    d.weights = dens->weights;
    stokes_run(S, xyz, d, tg, nt, output, out_src, out_trg);
  });
}

int stokes_host(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n, const double* tg,
                int64_t nt, int output, double* out_src, double* out_trg) {
  return guard([&] {
    check_stokes_call(state, xyz, dens, n, output, tg, nt, out_src, out_trg);
    State& S = state->s;
    Plan& P = *S.plan;
    set_device(*P.ctx);
    cudaStream_t s = P.ctx->stream;
    const int w = output == FMMB_STOKES_PRESSURE ? 1 : output == FMMB_STOKES_GRADIENT ? 9 : 3;
    const bool trg = out_trg && nt > 0;
    DBuf<double> x(3 * n), os(out_src ? w * n : 0), t(trg ? 3 * nt : 0), ot(trg ? w * nt : 0);
    DBuf<double> a[5];
    const double* src[5] = {dens->stokeslets, dens->stresslets, dens->stressvecs, dens->doublets, dens->weights};
    const double* dev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    FMMB_CUDA(cudaMemcpyAsync(x.p, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    if (trg) FMMB_CUDA(cudaMemcpyAsync(t.p, tg, sizeof(double) * 3 * nt, cudaMemcpyHostToDevice, s));
    for (int k = 0; k < 5; ++k) {
      if (!src[k]) continue;
      const int64_t len = k == 4 ? n : 3 * n;
      a[k].alloc(len);
      FMMB_CUDA(cudaMemcpyAsync(a[k].p, src[k], sizeof(double) * len, cudaMemcpyHostToDevice, s));
      dev[k] = a[k].p;
    }
    StokesDensities d;
    d.stokeslets = dev[0];
    d.stresslets = dev[1];
    d.stressvecs = dev[2];
    d.doublets = dev[3];
    d.weights = dev[4];
    stokes_run(S, x.p, d, t.p, trg ? nt : 0, output, out_src ? os.p : nullptr, trg ? ot.p : nullptr);
    if (out_src) FMMB_CUDA(cudaMemcpyAsync(out_src, os.p, sizeof(double) * w * n, cudaMemcpyDeviceToHost, s));
    if (trg) FMMB_CUDA(cudaMemcpyAsync(out_trg, ot.p, sizeof(double) * w * nt, cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

int fmmb_stokes_eval_densities_dev(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                                   int output, double* out) {
  return stokes_dev(state, xyz, dens, n, nullptr, 0, output, out, nullptr);
}

int fmmb_stokes_eval_densities(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                               int output, double* out) {
  return stokes_host(state, xyz, dens, n, nullptr, 0, output, out, nullptr);
}

int fmmb_stokes_eval_src_trg_dev(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                                 const double* targets, int64_t nt, int output, double* out_src, double* out_trg) {
  return stokes_dev(state, xyz, dens, n, targets, nt, output, out_src, out_trg);
}

int fmmb_stokes_eval_src_trg(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                             const double* targets, int64_t nt, int output, double* out_src, double* out_trg) {
  return stokes_host(state, xyz, dens, n, targets, nt, output, out_src, out_trg);
}

int fmmb_direct_dev(fmmb_ctx* ctx, const double* src, const double* tau, int64_t ns, const double* tgt,
                    const int64_t* self_index, int64_t nt, double* pot, double* grad) {
  return guard([&] {
    require(ctx && src && tau && tgt, FMMB_ERR_ARGUMENT, "null argument");
    require(ns >= 0 && nt >= 0, FMMB_ERR_DIMENSION, "negative count");
    set_device(ctx->c);
    require_device_ptr(ctx->c, src, "sources");
    require_device_ptr(ctx->c, tau, "densities");
    require_device_ptr(ctx->c, tgt, "targets");
    require_device_ptr(ctx->c, self_index, "self index");
    require_device_ptr(ctx->c, pot, "potential output");
    require_device_ptr(ctx->c, grad, "gradient output");
    direct(ctx->c, src, tau, ns, tgt, self_index, nt, pot, grad);
  });
}

int fmmb_direct_noalloc_dev(fmmb_ctx* ctx, const double* src, const double* tau, int64_t ns, const double* tgt,
                            const int64_t* self_index, int64_t nt, double* pot, double* grad) {
  return guard([&] {
    require(ctx && src && tau && tgt, FMMB_ERR_ARGUMENT, "null argument");
    require(ns >= 0 && nt >= 0, FMMB_ERR_DIMENSION, "negative count");
    set_device(ctx->c);
    for (const void* p : {(const void*)src, (const void*)tau, (const void*)tgt, (const void*)self_index, (const void*)pot,
                          (const void*)grad})
      require_device_ptr(ctx->c, p, "fmmb_direct_noalloc_dev argument");
    direct_noalloc(ctx->c, src, tau, ns, tgt, self_index, nt, pot, grad);
  });
}

}  // extern "C"
