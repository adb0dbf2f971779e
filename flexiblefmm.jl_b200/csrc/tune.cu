// The autotuner of the launch shapes: tile and block shapes chosen by timing them on the
// caller's own inputs (the reference has no tuner).
//
// Three shapes are free, in that no result depends on them (each target's sums are taken in the
// list's order whatever the blocking, and a near-field warp owns its leaf group):
//   - the targets per M2L block (32, 64 or 128; a plan property: its blocks are re-cut from the
//     pairs per target), for both M2L kernels;
//   - the FP64 M2L's chunk width (two compiled widths per expansion length);
//   - the near-field warps per CTA (4 or 8).
// fmmb_autotune times each candidate on the state's own inputs (CUDA events on the context's
// stream, the median of three after one warm-up), keeps the fastest, applies it, and records it
// for every later plan and state of the same kind: method, kernel, order, precision path and the
// number of points rounded down to a power of two. Plans created afterwards take the recorded
// block size; states take the recorded chunk width and warps.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "passes.cuh"

namespace fmmb {
namespace {

struct Tuned {
  int tb = 0, nb_alt = 0, near_w = 4;
};
using Kind = std::tuple<int, int, int, int, int>;   // method, kernel, p, precision (-1: any), log2 N

std::mutex g_mu;
std::map<Kind, Tuned> g_tuned;

int log2_floor(int64_t n) {
  int b = 0;
  while ((int64_t)1 << (b + 1) <= n) ++b;
  return b;
}

Kind kind_of(const Plan& P, int precision) {
  const Cache& C = *P.cache;
  return Kind(C.method, C.kernel, C.p, precision, log2_floor(P.N));
}

// the median of three timed runs after one warm-up, in ms
template <class F>
double time_ms(cudaStream_t s, F&& f) {
  cudaEvent_t e0, e1;
  FMMB_CUDA(cudaEventCreate(&e0));
  FMMB_CUDA(cudaEventCreate(&e1));
  f();
  double t[3];
  for (double& x : t) {
    FMMB_CUDA(cudaEventRecord(e0, s));
    f();
    FMMB_CUDA(cudaEventRecord(e1, s));
    FMMB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    FMMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    x = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::sort(t, t + 3);
  return t[1];
}

}  // namespace

int tuned_block_size(const Plan& P) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_tuned.find(kind_of(P, -1));
  return it == g_tuned.end() ? 0 : it->second.tb;
}

void apply_tuned_state(State& S) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_tuned.find(kind_of(*S.plan, S.precision));
  if (it == g_tuned.end()) return;
  S.f64_nb_alt = it->second.nb_alt;
  S.near_warps = it->second.near_w;
}

void autotune(State& S, const double* xyz, const double* tau, bool tune_blocks, double* out) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  require(C.method == FMMB_METHOD_SPHERICAL_HARMONICS, FMMB_ERR_UNSUPPORTED, "the tuner takes the harmonic methods");
  cudaStream_t s = P.ctx->stream;
  // the multipoles of these inputs, which every M2L candidate reads (Stokeslet3D: Stokeslets)
  if (C.kernel == FMMB_KERNEL_STOKESLET3D) {
    StokesDensities d;
    d.stokeslets = tau;
    stokes_build(S, xyz, d);
  } else {
    gather_inputs(S, xyz, tau);
    upward_pass(S);
  }
  // the M2L: block sizes × (FP64) chunk widths
  std::vector<int> tbs = {P.TB};
  if (tune_blocks) tbs = {32, 64, 128};
  const bool f64 = S.precision == FMMB_PRECISION_FP64;
  double best = 1e300;
  int best_tb = P.TB, best_alt = S.f64_nb_alt;
  for (int tb : tbs) {
    if (tb != P.TB) build_blocks(P, tb);
    for (int alt = 0; alt < (f64 ? 2 : 1); ++alt) {
      S.f64_nb_alt = f64 ? alt : S.f64_nb_alt;
      const double ms = time_ms(s, [&] { m2l_stage(S); });
      if (ms < best) { best = ms; best_tb = tb; best_alt = S.f64_nb_alt; }
    }
  }
  if (P.TB != best_tb) build_blocks(P, best_tb);
  S.f64_nb_alt = best_alt;
  // the near field at the sources (harmonic methods with charges: Laplace3D and Yukawa3D)
  double best_near = 0;
  int best_w = S.near_warps;
  if (C.kernel != FMMB_KERNEL_STOKESLET3D && P.n_leaves > 0) {
    DBuf<double> pot(P.N), grad(3 * P.N);
    best_near = 1e300;
    for (int w : {4, 8}) {
      S.near_warps = w;
      const double ms = time_ms(s, [&] { near_sources(S, FMMB_OUTPUT_POTENTIAL | FMMB_OUTPUT_GRADIENT, pot.p, grad.p, s); });
      if (ms < best_near) { best_near = ms; best_w = w; }
    }
    FMMB_CUDA(cudaStreamSynchronize(s));
  }
  S.near_warps = best_w;
  S.built = false;                      // the timed stages left the expansions incomplete
  {
    std::lock_guard<std::mutex> lk(g_mu);
    Tuned t;
    t.tb = best_tb;
    t.nb_alt = best_alt;
    t.near_w = best_w;
    g_tuned[kind_of(P, S.precision)] = t;
    if (tune_blocks) g_tuned[kind_of(P, -1)] = t;
  }
  if (out) {
    out[0] = best_tb;
    out[1] = best_alt;
    out[2] = best_w;
    out[3] = best;
    out[4] = best_near;
  }
}

}  // namespace fmmb
