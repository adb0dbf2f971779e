// CubeKernelIndependent{3}(Laplace3D()) on the device (src/operators/cubeki.jl,
// src/operators/ki_common.jl, src/operators/spectral_m2l.jl). A multipole is a density on the
// box's small surface (p points per edge), a partial local the check potentials on the same
// surface, a local a density on the large surface (pc per edge).
//   P2M (a15)   k_ki_check: the check potentials of each childless node's sources on its large
//               surface; then the factored pseudo-inverse V·(S⁺Uᴴ·check) as two DMMA GEMMs
//   M2M, L2L    the dense width-invariant operators on the DMMA GEMM (the Laplace sweeps)
//   M2L (a19)   spectral: the multipole embedded in the zero-padded (2p)³ lattice and
//               transformed (k_ki_forward, half spectrum, FP32); per target the Hadamard sums
//               Σ κ̂_o ⊙ σ̂_s over its far pairs (k_ki_hadamard: one frequency block of 64 per
//               CTA, the block of the 316 kernel tables in shared memory, a warp per target,
//               float4 loads of the sources' spectra, 16 pairs in flight); the inverse transform at the target's
//               small-surface points added to its check potentials (k_ki_inverse)
//   locals      the leaves' densities on their large surfaces, V·(S⁺Uᴴ·check) (DMMA GEMMs)
//   L2T (a22)   the surface sums of the leaves' local densities (eval.cu) and the near field
// The operators are built at width 1 (Laplace3D is homogeneous of degree −1): at width w the
// surfaces scale by w, the pseudo-inverses by w and the M2L tables by 1/w.
#include <map>
#include <tuple>

#include "passes.cuh"

namespace fmmb {

void gemm_columns(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                  int num_sms, cudaStream_t s);

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }
inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

constexpr int FB = 64;             // frequencies per block of the Hadamard stage
constexpr int HAD_THREADS = 512;   // 16 warps, one target at a time each
constexpr int HAD_UNROLL = 16;
constexpr int SIDE = 2 * KI_PMAX;


// the host operators at width 1, by (p, pc, d, rtol): caches with the same parameters share them
std::mutex g_ki_mu;
std::map<std::tuple<int, int, double, double>, std::shared_ptr<const KIHost>> g_ki;

std::shared_ptr<const KIHost> host_operators(int p, int pc, double d, double rtol) {
  std::lock_guard<std::mutex> lk(g_ki_mu);
  auto key = std::make_tuple(p, pc, d, rtol);
  auto it = g_ki.find(key);
  if (it != g_ki.end()) return it->second;
  auto h = std::make_shared<const KIHost>(build_ki_operators(p, pc, d, rtol, 1.0));
  g_ki[key] = h;
  return h;
}

// a column-major rows × cols matrix zero-padded to R × C
std::vector<double> pad(const std::vector<double>& a, int rows, int cols, int R, int C) {
  std::vector<double> o((size_t)R * C, 0.0);
  for (int j = 0; j < cols; ++j)
    for (int i = 0; i < rows; ++i) o[(size_t)j * R + i] = a[(size_t)j * rows + i];
  return o;
}

// ---------------------------------------------------------------- P2M: check potentials
// one CTA per childless node with sources: pM[k] = w · Σ_j G(w·y_k − (x_j − c)) τ_j at the
// large-surface points y_k (width 1), the factor w being the pseudo-inverse's scale; the
// sources staged in shared memory 256 at a time, each thread owning its check points.
// R = float on the mixed path (box-centred FP32 terms and sums, the method's FP32 far field
// consumes them), double on the plain path.
constexpr int CHK_SRC = 256;
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
template <typename R>
__global__ void __launch_bounds__(128) k_ki_check(const int* __restrict__ nodes, const int4* __restrict__ cell,
                                                  const int* __restrict__ plo, const int* __restrict__ phi,
                                                  const double* __restrict__ xs, const double* __restrict__ ys,
                                                  const double* __restrict__ zs, const double* __restrict__ q,
                                                  Geometry geo, const double* __restrict__ large, int nl, int nld,
                                                  double* __restrict__ pM) {
  __shared__ R sx[CHK_SRC], sy[CHK_SRC], sz[CHK_SRC], sq[CHK_SRC];
  const int node = nodes[blockIdx.x];
  const int4 c = cell[node];
  const double w = ldexp(geo.W0, -c.w);
  const double cx = geo.center(0, c.x, w), cy = geo.center(1, c.y, w), cz = geo.center(2, c.z, w);
  double* out = pM + (int64_t)blockIdx.x * nld;
  const int j0 = plo[node], j1 = phi[node];
  for (int b = j0; b <= j1; b += CHK_SRC) {
    __syncthreads();
    for (int i = threadIdx.x; i < CHK_SRC && b + i <= j1; i += 128) {
      sx[i] = (R)(xs[b + i] - cx);
      sy[i] = (R)(ys[b + i] - cy);
      sz[i] = (R)(zs[b + i] - cz);
      sq[i] = (R)q[b + i];
    }
    __syncthreads();
    const int m = min(CHK_SRC, j1 - b + 1);
    for (int k = threadIdx.x; k < nl; k += 128) {
      const R yx = (R)(w * large[3 * k]), yy = (R)(w * large[3 * k + 1]), yz = (R)(w * large[3 * k + 2]);
      R a = b == j0 ? R(0) : (R)out[k];
      for (int s = 0; s < m; ++s) {
        const R dx = yx - sx[s], dy = yy - sy[s], dz = yz - sz[s];
        a = fma(sq[s], rsqrt_r(fma(dz, dz, fma(dy, dy, dx * dx))), a);
      }
      out[k] = (double)a;
    }
  }
  for (int k = threadIdx.x; k < nl; k += 128) out[k] *= w * KC;
}

// ---------------------------------------------------------------- the spectral M2L
// forward: the density of node g (its ns small-surface values, embedded in the p³ corner of the
// (2p)³ lattice) to its half spectrum, separable DFTs in shared memory
__global__ void __launch_bounds__(128) k_ki_forward(int first, int p, int ns, int LD, int nfp,
                                                    const double* __restrict__ M, const float2* __restrict__ tw,
                                                    const int* __restrict__ embed, float2* __restrict__ spec) {
  extern __shared__ float2 smf[];
  __shared__ float2 c_tw[SIDE * SIDE];              // [j·n + k] = e^{−2πi jk/n}, n = 2p
  const int g = first + blockIdx.x, n = 2 * p, nh = p + 1, tid = threadIdx.x;
  float2* a1 = smf;                                 // [nh·p·p]
  float2* a2 = a1 + nh * p * p;                     // [nh·n·p]
  float* x = reinterpret_cast<float*>(a2 + nh * n * p);   // [p³]
  for (int i = tid; i < n * n; i += 128) c_tw[i] = tw[(i / n) * (i % n) % n];
  for (int i = tid; i < p * p * p; i += 128) x[i] = 0.f;
  __syncthreads();
  const double* col = M + (int64_t)g * LD;
  for (int i = tid; i < ns; i += 128) {
    const int e = embed[i], j1 = e % n, j2 = (e / n) % n, j3 = e / (n * n);
    x[j1 + p * (j2 + p * j3)] = (float)col[i];
  }
  __syncthreads();
  // dim 1: real → k1 ≤ p
  for (int o = tid; o < nh * p * p; o += 128) {
    const int k1 = o % nh, r = o / nh;   // r = j2 + p·j3
    float re = 0.f, im = 0.f;
    for (int j1 = 0; j1 < p; ++j1) {
      const float v = x[j1 + p * r];
      const float2 t = c_tw[j1 * n + k1];
      re = fmaf(v, t.x, re);
      im = fmaf(v, t.y, im);
    }
    a1[o] = make_float2(re, im);         // a1[k1 + nh·(j2 + p·j3)]
  }
  __syncthreads();
  // dim 2: j2 < p → k2 < n
  for (int o = tid; o < nh * n * p; o += 128) {
    const int k1 = o % nh, k2 = (o / nh) % n, j3 = o / (nh * n);
    float re = 0.f, im = 0.f;
    for (int j2 = 0; j2 < p; ++j2) {
      const float2 a = a1[k1 + nh * (j2 + p * j3)], t = c_tw[j2 * n + k2];
      re = fmaf(a.x, t.x, fmaf(-a.y, t.y, re));
      im = fmaf(a.x, t.y, fmaf(a.y, t.x, im));
    }
    a2[o] = make_float2(re, im);         // a2[k1 + nh·(k2 + n·j3)]
  }
  __syncthreads();
  // dim 3: j3 < p → k3 < n, written to the node's spectrum (k1 fastest)
  float2* out = spec + (int64_t)g * nfp;
  const int nf = nh * n * n;
  for (int o = tid; o < nfp; o += 128) {
    if (o >= nf) { out[o] = make_float2(0.f, 0.f); continue; }
    const int k12 = o % (nh * n), k3 = o / (nh * n);
    float re = 0.f, im = 0.f;
    for (int j3 = 0; j3 < p; ++j3) {
      const float2 a = a2[k12 + nh * n * j3], t = c_tw[j3 * n + k3];
      re = fmaf(a.x, t.x, fmaf(-a.y, t.y, re));
      im = fmaf(a.x, t.y, fmaf(a.y, t.x, im));
    }
    out[o] = make_float2(re, im);
  }
}

// Hadamard sums: CTA (frequency block fb, range of targets); the 316 tables' block fb in shared
// memory; a warp per target, lane l the frequencies 2l, 2l + 1 of the block
__global__ void __launch_bounds__(HAD_THREADS) k_ki_hadamard(int first, int last, int per_cta, int nfp,
                                                             const int* __restrict__ ptr, const int2* __restrict__ tp,
                                                             const float2* __restrict__ tab,
                                                             const float2* __restrict__ spec, float2* __restrict__ U) {
  extern __shared__ float4 st[];   // [NFAR][FB / 2]
  const int fb = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < NFAR * (FB / 2); i += HAD_THREADS) {
    const int f = i / (FB / 2), l = i % (FB / 2);
    st[i] = reinterpret_cast<const float4*>(tab + (int64_t)f * nfp + fb * FB)[l];
  }
  __syncthreads();
  const int t0 = first + blockIdx.y * per_cta, t1 = min(last, t0 + per_cta);
  for (int t = t0 + warp; t < t1; t += HAD_THREADS / 32) {
    const int k0 = ptr[t], k1 = ptr[t + 1];
    if (k0 == k1) continue;
    float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;
    int k = k0;
    // HAD_UNROLL pairs' loads in flight per warp: the kernel is bound by their latency
    for (; k + HAD_UNROLL <= k1; k += HAD_UNROLL) {
      int2 pr[HAD_UNROLL];
      float4 sv[HAD_UNROLL];
#pragma unroll
      for (int u = 0; u < HAD_UNROLL; ++u) pr[u] = tp[k + u];
#pragma unroll
      for (int u = 0; u < HAD_UNROLL; ++u)
        sv[u] = __ldg(reinterpret_cast<const float4*>(spec + (int64_t)pr[u].x * nfp + fb * FB) + lane);
#pragma unroll
      for (int u = 0; u < HAD_UNROLL; ++u) {
        const float4 tv = st[pr[u].y * (FB / 2) + lane];
        ar = fmaf(tv.x, sv[u].x, fmaf(-tv.y, sv[u].y, ar));
        ai = fmaf(tv.x, sv[u].y, fmaf(tv.y, sv[u].x, ai));
        br = fmaf(tv.z, sv[u].z, fmaf(-tv.w, sv[u].w, br));
        bi = fmaf(tv.z, sv[u].w, fmaf(tv.w, sv[u].z, bi));
      }
    }
    for (; k < k1; ++k) {
      const int2 pr = tp[k];
      const float4 sv = __ldg(reinterpret_cast<const float4*>(spec + (int64_t)pr.x * nfp + fb * FB) + lane);
      const float4 tv = st[pr.y * (FB / 2) + lane];
      ar = fmaf(tv.x, sv.x, fmaf(-tv.y, sv.y, ar));
      ai = fmaf(tv.x, sv.y, fmaf(tv.y, sv.x, ai));
      br = fmaf(tv.z, sv.z, fmaf(-tv.w, sv.w, br));
      bi = fmaf(tv.z, sv.w, fmaf(tv.w, sv.z, bi));
    }
    reinterpret_cast<float4*>(U + (int64_t)t * nfp + fb * FB)[lane] = make_float4(ar, ai, br, bi);
  }
}

// inverse: target g's summed half spectrum back to the lattice at its p³ corner (inverse DFTs
// in dims 3 and 2, then the Hermitian sum over k1), the small-surface values added to its
// check potentials times 1/(w·n³) (the tables are at width 1)
__global__ void __launch_bounds__(128) k_ki_inverse(int first, int p, int ns, int LD, int nfp,
                                                    const int* __restrict__ ptr, const int4* __restrict__ cell,
                                                    double W0, const float2* __restrict__ tw,
                                                    const int* __restrict__ embed, const float2* __restrict__ U,
                                                    double* __restrict__ Pl) {
  extern __shared__ float2 sm2[];
  __shared__ float2 c_tw[SIDE * SIDE];              // [j·n + k] = e^{−2πi jk/n}
  const int g = first + blockIdx.x, n = 2 * p, nh = p + 1, tid = threadIdx.x;
  if (ptr[g] == ptr[g + 1]) return;                 // no far pairs: nothing to add
  for (int i = tid; i < n * n; i += 128) c_tw[i] = tw[(i / n) * (i % n) % n];
  float2* u = sm2;                                  // [nh·n·n]
  float2* b3 = u + nh * n * n;                      // [nh·n·p]: b3[k1 + nh·(k2 + n·j3)]
  float2* b2 = b3 + nh * n * p;                     // [nh·p·p]: b2[k1 + nh·(j2 + p·j3)]
  float* xo = reinterpret_cast<float*>(b2 + nh * p * p);   // [p³]
  const float2* src = U + (int64_t)g * nfp;
  for (int i = tid; i < nh * n * n; i += 128) u[i] = src[i];
  __syncthreads();
  for (int o = tid; o < nh * n * p; o += 128) {
    const int k12 = o % (nh * n), j3 = o / (nh * n);
    float re = 0.f, im = 0.f;
    for (int k3 = 0; k3 < n; ++k3) {
      const float2 a = u[k12 + nh * n * k3], t = c_tw[j3 * n + k3];   // × conj(t)
      re = fmaf(a.x, t.x, fmaf(a.y, t.y, re));
      im = fmaf(a.y, t.x, fmaf(-a.x, t.y, im));
    }
    b3[o] = make_float2(re, im);
  }
  __syncthreads();
  for (int o = tid; o < nh * p * p; o += 128) {
    const int k1 = o % nh, j2 = (o / nh) % p, j3 = o / (nh * p);
    float re = 0.f, im = 0.f;
    for (int k2 = 0; k2 < n; ++k2) {
      const float2 a = b3[k1 + nh * (k2 + n * j3)], t = c_tw[j2 * n + k2];
      re = fmaf(a.x, t.x, fmaf(a.y, t.y, re));
      im = fmaf(a.y, t.x, fmaf(-a.x, t.y, im));
    }
    b2[o] = make_float2(re, im);
  }
  __syncthreads();
  for (int o = tid; o < p * p * p; o += 128) {
    const int j1 = o % p, r = o / p;                // r = j2 + p·j3
    const float2* b = b2 + nh * r;
    float v = b[0].x + ((j1 & 1) ? -b[p].x : b[p].x);   // k1 = 0 and k1 = n/2 = p
    for (int k1 = 1; k1 < p; ++k1) {
      const float2 t = c_tw[j1 * n + k1];           // Re(b · e^{+iθ}) = b.x cos θ − b.y sin θ, t.y = −sin θ
      v += 2.f * fmaf(b[k1].x, t.x, b[k1].y * t.y);
    }
    xo[o] = v;
  }
  __syncthreads();
  const int4 c = cell[g];
  const double scale = 1.0 / (ldexp(W0, -c.w) * (double)(n * n * n));
  double* col = Pl + (int64_t)g * LD;
  for (int i = tid; i < ns; i += 128) {
    const int e = embed[i], j1 = e % n, j2 = (e / n) % n, j3 = e / (n * n);
    col[i] += scale * (double)xo[j1 + p * (j2 + p * j3)];
  }
}

}  // namespace

// the cache's device operators (once per cache, when the first plan has fixed its width) and
// the plan's per-level tables and target-major pair list
void ki_prepare(Plan& P) {
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  {
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.ki) {
      std::shared_ptr<const KIHost> h = host_operators(C.p, C.ki_pc, C.ki_d, C.ki_rtol);
      const int ns = h->ns, nl = h->nl, LD = C.ld;
      require(ns == C.np, FMMB_ERR_DEVICE, "surface size mismatch");
      C.ki_nl = nl;
      C.ki_nld = round_up(nl, 64);
      C.ki_ru = round_up(h->rank_up, 64);
      C.ki_rd = round_up(h->rank_down, 64);
      C.ki_nfp = round_up(h->nfreq, FB);
      to_device(C.ki_large, h->large, s);
      to_device(C.ki_upv, pad(h->up_v, ns, h->rank_up, LD, C.ki_ru), s);            // LD × RU
      to_device(C.ki_upsu, pad(h->up_su, h->rank_up, nl, C.ki_ru, nl), s);          // RU × nl
      to_device(C.ki_downv, pad(h->down_v, nl, h->rank_down, C.ki_nld, C.ki_rd), s); // NLD × RD
      to_device(C.ki_downsu, pad(h->down_su, h->rank_down, ns, C.ki_rd, ns), s);    // RD × ns
      // M2M (ns × 8ns) into LD × 8LD, L2L (8ns × ns) into 8LD × LD (child block k at k·LD)
      std::vector<double> m2m((size_t)LD * NCH * LD, 0.0), l2l((size_t)NCH * LD * LD, 0.0);
      for (int k = 0; k < NCH; ++k)
        for (int j = 0; j < ns; ++j)
          for (int i = 0; i < ns; ++i) {
            m2m[(size_t)(k * LD + j) * LD + i] = h->m2m[(size_t)(k * ns + j) * ns + i];
            l2l[(size_t)j * NCH * LD + k * LD + i] = h->l2l[(size_t)j * NCH * ns + k * ns + i];
          }
      to_device(C.ki_m2m, m2m, s);
      to_device(C.ki_l2l, l2l, s);
      std::vector<float2> tab((size_t)NFAR * C.ki_nfp, make_float2(0.f, 0.f));
      for (int f = 0; f < NFAR; ++f)
        for (int i = 0; i < h->nfreq; ++i)
          tab[(size_t)f * C.ki_nfp + i] = make_float2((float)h->tables[((size_t)f * h->nfreq + i) * 2],
                                                      (float)h->tables[((size_t)f * h->nfreq + i) * 2 + 1]);
      to_device(C.ki_tab, tab, s);
      const int n = 2 * C.p;
      std::vector<float2> tw(n);
      for (int k = 0; k < n; ++k)
        tw[k] = make_float2((float)std::cos(2 * M_PI * k / n), (float)-std::sin(2 * M_PI * k / n));
      to_device(C.ki_tw, tw, s);
      to_device(C.ki_embed, h->embed, s);
      FMMB_CUDA(cudaStreamSynchronize(s));
      C.ki = h;
    }
  }
  P.lv_m2m.assign(P.L, C.ki_m2m.p);
  P.lv_l2l.assign(P.L, C.ki_l2l.p);
  build_target_pairs(P);
  // every real leaf, sources or not: evaluate() may locate targets in the empty ones
  std::vector<int> all;
  for (int g = 0; g < P.nnodes; ++g)
    if (P.h_flags[g] & F_LEAF) all.push_back(g);
  P.n_ki_leaves = (int)all.size();
  to_device(P.ki_leaves, all, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// the state's buffers
void ki_state(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  S.ki_pm.alloc((size_t)std::max(P.n_s2m, 1) * C.ki_nld);
  S.ki_y.alloc((size_t)std::max(std::max(P.n_s2m, P.n_ki_leaves), 1) * std::max(C.ki_ru, C.ki_rd));
  S.ki_ll.alloc((size_t)P.nnodes * C.ki_nld);
  S.ki_spec.alloc((size_t)P.nnodes * C.ki_nfp);
  S.ki_u.alloc((size_t)P.nnodes * C.ki_nfp);
}

// P2M: check potentials, then the multipoles V·(S⁺Uᴴ·check) of the childless nodes
int ki_p2m(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  if (P.n_s2m == 0) return 0;
  auto chk = S.precision == FMMB_PRECISION_MIXED ? k_ki_check<float> : k_ki_check<double>;
  chk<<<P.n_s2m, 128, 0, s>>>(P.s2m_nodes.p, P.cell.p, P.plo.p, P.phi.p, S.xs.p, S.ys.p, S.zs.p, S.q.p, geometry(P),
                                     C.ki_large.p, C.ki_nl, C.ki_nld, S.ki_pm.p);
  FMMB_LAUNCH_CHECK();
  const int sms = P.ctx->num_sms;
  gemm_columns(C.ki_ru, C.ki_nl, C.ki_upsu.p, ColMap{S.ki_pm.p, nullptr, 0, 1, (int64_t)C.ki_nld},
               ColMap{S.ki_y.p, nullptr, 0, 1, (int64_t)C.ki_ru}, P.n_s2m, C.ki_ru, C.ki->rank_up, 0, sms, s);
  gemm_columns(C.ld, C.ki_ru, C.ki_upv.p, ColMap{S.ki_y.p, nullptr, 0, 1, (int64_t)C.ki_ru},
               ColMap{S.M.p, P.s2m_nodes.p, 0, 0, 0}, P.n_s2m, C.ld, C.np, 0, sms, s);
  return 3;
}

// the spectral M2L of every level into the (zeroed) check potentials
int ki_m2l(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  const int first = P.level_start[std::min(2, P.L)], last = P.nnodes, nt = last - first;
  if (nt <= 0) return 0;
  const int p = C.p, n = 2 * p, nh = p + 1;
  const size_t fsm = sizeof(float2) * (nh * p * p + nh * n * p) + sizeof(float) * p * p * p;
  FMMB_CUDA(cudaFuncSetAttribute(k_ki_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
  k_ki_forward<<<nt, 128, fsm, s>>>(first, p, C.np, C.ld, C.ki_nfp, S.M.p, C.ki_tw.p, C.ki_embed.p, S.ki_spec.p);
  FMMB_LAUNCH_CHECK();
  const size_t hsm = sizeof(float4) * NFAR * (FB / 2);
  FMMB_CUDA(cudaFuncSetAttribute(k_ki_hadamard, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
  const int per_cta = 256;
  k_ki_hadamard<<<dim3(C.ki_nfp / FB, (nt + per_cta - 1) / per_cta), HAD_THREADS, hsm, s>>>(
      first, last, per_cta, C.ki_nfp, P.tp_ptr.p, P.tp.p, C.ki_tab.p, S.ki_spec.p, S.ki_u.p);
  FMMB_LAUNCH_CHECK();
  const size_t ism = sizeof(float2) * (nh * n * n + nh * n * p + nh * p * p) + sizeof(float) * p * p * p;
  FMMB_CUDA(cudaFuncSetAttribute(k_ki_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ism));
  k_ki_inverse<<<nt, 128, ism, s>>>(first, p, C.np, C.ld, C.ki_nfp, P.tp_ptr.p, P.cell.p, P.W0, C.ki_tw.p, C.ki_embed.p,
                                    S.ki_u.p, S.Pl.p);
  FMMB_LAUNCH_CHECK();
  return 3;
}

// the leaves' local densities on their large surfaces: V·(S⁺Uᴴ·check), the width factor
// applied by the evaluation
int ki_leaf_locals(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  const int nlv = P.n_ki_leaves;
  if (nlv == 0) return 0;
  const int sms = P.ctx->num_sms;
  gemm_columns(C.ki_rd, C.np, C.ki_downsu.p, ColMap{S.Pl.p, P.ki_leaves.p, 0, 0, (int64_t)C.ld},
               ColMap{S.ki_y.p, nullptr, 0, 1, (int64_t)C.ki_rd}, nlv, C.ki_rd, C.ki->rank_down, 0, sms, s);
  gemm_columns(C.ki_nld, C.ki_rd, C.ki_downv.p, ColMap{S.ki_y.p, nullptr, 0, 1, (int64_t)C.ki_rd},
               ColMap{S.ki_ll.p, P.ki_leaves.p, 0, 0, (int64_t)C.ki_nld}, nlv, C.ki_nld, C.ki_nl, 0, sms, s);
  return 2;
}

}  // namespace fmmb
