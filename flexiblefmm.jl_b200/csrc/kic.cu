// KernelIndependent(Laplace2D(); nequiv) on the device (src/operators/kifmm.jl,
// src/operators/ki_common.jl): the 2D method on circles. The points lie in the plane z = 0 of the
// octree (the binding embeds them), so the octree's sourced nodes are the quadtree's, their far
// pairs the in-plane offsets and their colleagues' sources the 2D near field. A multipole is a
// density on the node's small circle (N points, radius √2/2·w), a partial local the check
// potentials on that circle, a local a density on the large circle ((4 − √2)/2·w).
//   P2M     k_kic_check (check potentials of each childless node's sources on its large circle,
//           a warp per node, lanes over the circle's points) and V·(S⁺Uᴴ·check) per level (DMMA)
//   M2M/L2L the level's dense operators on the DMMA GEMM (the Laplace sweeps)
//   M2L     k_kic_m2l: a warp per target, its far pairs' dense N × N check maps applied in FP64
//   locals  V·(S⁺Uᴴ·check) per level over every real leaf
//   L2T     the large-circle sums (eval.cu) and the 2D near field
// The log kernel is not homogeneous: every width has its own operators (built on the host, FP64,
// when a plan first needs the width, kept by the cache).
#include <algorithm>

#include "passes.cuh"

namespace fmmb {

void gemm_columns(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                  int num_sms, cudaStream_t s);

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }
constexpr int CLD = 64;   // padded circle length

// check potentials pM[k] = Σ_j c·log|y_k − x_j|² τ_j at the large-circle points y_k of node g
__global__ void __launch_bounds__(128) k_kic_check(const int* __restrict__ nodes, int nn, int N,
                                                   const int4* __restrict__ cell, const int* __restrict__ plo,
                                                   const int* __restrict__ phi, const double* __restrict__ xs,
                                                   const double* __restrict__ ys, const double* __restrict__ q,
                                                   Geometry geo, double* __restrict__ pM) {
  const int wg = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (wg >= nn) return;
  const int node = nodes[wg];
  const int4 c = cell[node];
  const double w = ldexp(geo.W0, -c.w);
  const double cx = geo.center(0, c.x, w), cy = geo.center(1, c.y, w);
  double yx[2], yy[2], acc[2] = {0, 0};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = lane + 32 * h;
    double sn, cs;
    sincospi(2.0 * k / N, &sn, &cs);
    yx[h] = cx + KIC_LARGE * w * cs;
    yy[h] = cy + KIC_LARGE * w * sn;
  }
  for (int j = plo[node]; j <= phi[node]; ++j) {
    const double sx = xs[j], sy = ys[j], t = q[j];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const double dx = yx[h] - sx, dy = yy[h] - sy;
      acc[h] = fma(t, log(fma(dy, dy, dx * dx)), acc[h]);
    }
  }
  double* out = pM + (int64_t)wg * CLD;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = lane + 32 * h;
    out[k] = k < N ? -KC * acc[h] : 0.0;
  }
}

// the dense M2L: warp per target t, Pl[t] = Σ over its far pairs (s, f) of A_f(level) · M[s]
// (rows lane and lane + 32; the columns of M[s] broadcast by shuffles)
__global__ void __launch_bounds__(128) k_kic_m2l(int first, int last, int N, const int* __restrict__ ptr,
                                                 const int2* __restrict__ tp, const int4* __restrict__ cell,
                                                 const uint64_t* __restrict__ ops_lv, const double* __restrict__ M,
                                                 double* __restrict__ Pl) {
  const int t = first + blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= last) return;
  const int k0 = ptr[t], k1 = ptr[t + 1];
  if (k0 == k1) return;
  const double* ops = reinterpret_cast<const double*>(ops_lv[cell[t].w]);
  double a0 = 0, a1 = 0;
  for (int k = k0; k < k1; ++k) {
    const int2 pr = tp[k];
    const double* A = ops + (int64_t)pr.y * CLD * CLD;
    const double* x = M + (int64_t)pr.x * CLD;
    const double xl = x[lane], xh = x[lane + 32];
    for (int j = 0; j < N; ++j) {
      const double xj = __shfl_sync(0xffffffffu, j < 32 ? xl : xh, j & 31);
      a0 = fma(A[j * CLD + lane], xj, a0);
      a1 = fma(A[j * CLD + lane + 32], xj, a1);
    }
  }
  Pl[(int64_t)t * CLD + lane] = a0;
  Pl[(int64_t)t * CLD + lane + 32] = a1;
}

// the level ranges of a node-ordered list
std::vector<int> level_ranges(const std::vector<int>& nodes, const std::vector<int>& level_start, int L) {
  std::vector<int> r(L + 1, 0);
  size_t i = 0;
  for (int l = 0; l < L; ++l) {
    r[l] = (int)i;
    while (i < nodes.size() && nodes[i] < level_start[l + 1]) ++i;
  }
  r[L] = (int)i;
  return r;
}

}  // namespace

void kic_prepare(Plan& P) {
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  P.kic_upv.assign(P.L, nullptr);
  P.kic_upsu.assign(P.L, nullptr);
  P.kic_downv.assign(P.L, nullptr);
  P.kic_downsu.assign(P.L, nullptr);
  {
    std::lock_guard<std::mutex> lk(C.mu);
    for (int l = 2; l < P.L; ++l) {
      const int e = P.e0 - l;
      auto it = C.kic_levels.find(e);
      if (it == C.kic_levels.end()) {
        const KICircleLevel h = build_ki_circle_level(C.np, C.ki_rtol, std::ldexp(C.W0, e));
        std::unique_ptr<Cache::CircleLevel> d(new Cache::CircleLevel());
        to_device(d->upv, h.up_v, s);
        to_device(d->upsu, h.up_su, s);
        to_device(d->downv, h.down_v, s);
        to_device(d->downsu, h.down_su, s);
        to_device(d->m2m, h.m2m, s);
        to_device(d->l2l, h.l2l, s);
        to_device(d->m2l, h.m2l, s);
        FMMB_CUDA(cudaStreamSynchronize(s));
        it = C.kic_levels.emplace(e, std::move(d)).first;
      }
      const Cache::CircleLevel& d = *it->second;
      P.lv_reps[l] = d.m2l.p;
      P.lv_m2m[l] = d.m2m.p;
      P.lv_l2l[l] = d.l2l.p;
      P.kic_upv[l] = d.upv.p;
      P.kic_upsu[l] = d.upsu.p;
      P.kic_downv[l] = d.downv.p;
      P.kic_downsu[l] = d.downsu.p;
    }
  }
  std::vector<uint64_t> t(P.L);
  for (int l = 0; l < P.L; ++l) t[l] = (uint64_t)(uintptr_t)P.lv_reps[l];
  to_device(P.d_lv_reps, t, s);
  build_target_pairs(P);
  // the childless sourced nodes and every real leaf, with their level ranges
  std::vector<int> s2m, all;
  for (int g = 0; g < P.nnodes; ++g) {
    const int l = (int)(std::upper_bound(P.level_start.begin(), P.level_start.end(), g) - P.level_start.begin()) - 1;
    if (l >= 2 && P.h_cf[g] < 0 && (P.h_flags[g] & F_SOURCE)) s2m.push_back(g);
    if (P.h_flags[g] & F_LEAF) all.push_back(g);
  }
  P.s2m_level_start = level_ranges(s2m, P.level_start, P.L);
  P.ki_leaf_level_start = level_ranges(all, P.level_start, P.L);
  P.n_ki_leaves = (int)all.size();
  to_device(P.ki_leaves, all, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
}

void kic_state(State& S) {
  Plan& P = *S.plan;
  S.ki_pm.alloc((size_t)std::max(P.n_s2m, 1) * CLD);
  S.ki_y.alloc((size_t)std::max(std::max(P.n_s2m, P.n_ki_leaves), 1) * CLD);
  S.ki_ll.alloc((size_t)P.nnodes * CLD);
  // leaves above level 2 have no far field: their densities stay zero
  FMMB_CUDA(cudaMemsetAsync(S.ki_ll.p, 0, S.ki_ll.bytes(), P.ctx->stream));
}

// check potentials, then each level's multipoles V·(S⁺Uᴴ·check)
int kic_p2m(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  if (P.n_s2m == 0) return 0;
  k_kic_check<<<nblk(P.n_s2m, 4), 128, 0, s>>>(P.s2m_nodes.p, P.n_s2m, C.np, P.cell.p, P.plo.p, P.phi.p, S.xs.p, S.ys.p,
                                               S.q.p, geometry(P), S.ki_pm.p);
  FMMB_LAUNCH_CHECK();
  int launches = 1;
  for (int l = 2; l < P.L; ++l) {
    const int a = P.s2m_level_start[l], n = P.s2m_level_start[l + 1] - a;
    if (n == 0) continue;
    gemm_columns(CLD, CLD, P.kic_upsu[l], ColMap{S.ki_pm.p + (int64_t)a * CLD, nullptr, 0, 1, CLD},
                 ColMap{S.ki_y.p, nullptr, 0, 1, CLD}, n, CLD, CLD, 0, P.ctx->num_sms, s);
    gemm_columns(CLD, CLD, P.kic_upv[l], ColMap{S.ki_y.p, nullptr, 0, 1, CLD},
                 ColMap{S.M.p, P.s2m_nodes.p + a, 0, 0, CLD}, n, CLD, C.np, 0, P.ctx->num_sms, s);
    launches += 2;
  }
  return launches;
}

int kic_m2l(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  const int first = P.level_start[std::min(2, P.L)], last = P.nnodes;
  if (last <= first) return 0;
  k_kic_m2l<<<nblk(last - first, 4), 128, 0, P.ctx->stream>>>(first, last, C.np, P.tp_ptr.p, P.tp.p, P.cell.p,
                                                              P.d_lv_reps.p, S.M.p, S.Pl.p);
  FMMB_LAUNCH_CHECK();
  return 1;
}

// the leaves' densities on their large circles, per level
int kic_leaf_locals(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  int launches = 0;
  for (int l = 2; l < P.L; ++l) {
    const int a = P.ki_leaf_level_start[l], n = P.ki_leaf_level_start[l + 1] - a;
    if (n == 0) continue;
    gemm_columns(CLD, CLD, P.kic_downsu[l], ColMap{S.Pl.p, P.ki_leaves.p + a, 0, 0, CLD},
                 ColMap{S.ki_y.p, nullptr, 0, 1, CLD}, n, CLD, CLD, 0, P.ctx->num_sms, s);
    gemm_columns(CLD, CLD, P.kic_downv[l], ColMap{S.ki_y.p, nullptr, 0, 1, CLD},
                 ColMap{S.ki_ll.p, P.ki_leaves.p + a, 0, 0, CLD}, n, CLD, C.np, 0, P.ctx->num_sms, s);
    launches += 2;
  }
  return launches;
}

}  // namespace fmmb
