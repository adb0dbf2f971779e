// The FP64 passes of the plain path (the drop-in) and the shared pieces of both paths:
//   gather    inputs into tree order                         (src/device_passes.jl:644-665)
//   P2M       multipoles of the childless nodes              (src/device_passes.jl:343-373)
//   M2M, L2L  one GEMM per level, gather/scatter fused       (src/device_passes.jl:539-611)
//   M2L       one launch for all levels: per block of targets and per symmetry class, the
//             signed-permutation gather, the class GEMM and the target-owned scatter
//                                                            (src/device_passes.jl:428-473,565-580)
//   L2P+P2P   the evaluation at the sources or at located targets
//                                                            (src/device.jl:89-100,189-206)
//   locate    the leaf of each target                        (src/tree/locate.jl:10-22)
//   direct    FP64 direct sums                               (src/kernels.jl:442-487)
// HBM layout: sources SoA (x, y, z, q) in tree order; expansions node-major with a padded
// leading dimension LD (a multiple of 64 ≥ (p+1)²), rows ≥ (p+1)² kept zero.
#include <algorithm>

#include "d4h.cuh"
#include "passes.cuh"
#include "scan_sort.cuh"

namespace fmmb {

__constant__ double c_tab[5 * TRI_MAX];  // a, b, cz, cm, cp of the Schmidt recurrences, up to degree PMAX
__constant__ double c_e[PMAX];           // the sectoral factors e_m, m = 1..PMAX
__constant__ float c_tabf[5 * TRI_MAX];
__constant__ float c_ef[PMAX];

void init_device_constants(cudaStream_t s) {
  std::vector<double> t(5 * TRI_MAX, 0.0), e(PMAX);
  for (int n = 0; n <= PMAX; ++n)
    for (int m = 0; m <= n; ++m) {
      int k = tri(n, m);
      double c = std::sqrt((double)((n - m) * (n + m)));
      t[2 * TRI_MAX + k] = c;
      if (n > m) {
        t[k] = (double)(2 * n - 1) / c;
        t[TRI_MAX + k] = std::sqrt((double)((n - m - 1) * (n + m - 1))) / c;
      }
      t[3 * TRI_MAX + k] = n + m >= 2 ? std::sqrt((double)((n + m) * (n + m - 1))) : 0.0;
      t[4 * TRI_MAX + k] = n - m >= 2 ? std::sqrt((double)((n - m) * (n - m - 1))) : 0.0;
    }
  for (int m = 1; m <= PMAX; ++m) e[m - 1] = std::sqrt((double)(2 * m - 1) / (double)(2 * m));
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_tab, t.data(), sizeof(double) * t.size(), 0, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_e, e.data(), sizeof(double) * e.size(), 0, cudaMemcpyHostToDevice, s));
  const std::vector<float> tf(t.begin(), t.end()), ef(e.begin(), e.end());
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_tabf, tf.data(), sizeof(float) * tf.size(), 0, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_ef, ef.data(), sizeof(float) * ef.size(), 0, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
}

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------- gather
__global__ void k_gather_inputs(const double* __restrict__ xyz, const double* __restrict__ tau, const int* __restrict__ perm,
                                int64_t n, double* __restrict__ xs, double* __restrict__ ys, double* __restrict__ zs,
                                double* __restrict__ q) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t j = perm[k];
  xs[k] = xyz[3 * j];
  ys[k] = xyz[3 * j + 1];
  zs[k] = xyz[3 * j + 2];
  q[k] = tau[j];
}

// charges (or zeros) and dipole moments into tree order
__global__ void k_gather_dipoles(const double* __restrict__ xyz, const double* __restrict__ tau,
                                 const double* __restrict__ dip, const int* __restrict__ perm, int64_t n,
                                 double* __restrict__ xs, double* __restrict__ ys, double* __restrict__ zs,
                                 double* __restrict__ q, double* __restrict__ d3) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int64_t j = perm[k];
  xs[k] = xyz[3 * j];
  ys[k] = xyz[3 * j + 1];
  zs[k] = xyz[3 * j + 2];
  q[k] = tau ? tau[j] : 0.0;
  d3[k] = dip ? dip[3 * j] : 0.0;
  d3[n + k] = dip ? dip[3 * j + 1] : 0.0;
  d3[2 * n + k] = dip ? dip[3 * j + 2] : 0.0;
}

// P2M of charges and dipoles d (src/operators/harmonics.jl:708-738): one thread per (node, order
// m); per source the charge's chain of order m, and the dipole's three terms from the chains of
// orders m − 1, m, m + 1 of degree n′ = n − 1 (the derivative identities, with the moment in box
// units d·s, harmonics.jl:436):
//   chain m − 1: (n, m) += ½ cm(n, m) · (−(dx ur − dy ui), dx ui + dy ur)
//   chain m:     (n, m) += cz(n, m) dz · (ur, −ui)
//   chain m + 1: (n, m) += ½ cp(n, m) · (dx ur + dy ui, dy ur − dx ui)   (m = 0: cp(n, 0) (dx ur + dy ui), 0)
template <int P>
__global__ void k_p2m_dip(const int* __restrict__ nodes, int nn, const int4* __restrict__ cell, const int* __restrict__ plo,
                          const int* __restrict__ phi, const double* __restrict__ xs, const double* __restrict__ ys,
                          const double* __restrict__ zs, const double* __restrict__ q, const double* __restrict__ d3,
                          int64_t npts, Geometry geo, const double* __restrict__ scale, int64_t pitch,
                          double* __restrict__ M) {
  __shared__ double s_t[5 * TRI_MAX];   // a, b, cz, cm, cp
  __shared__ double s_e[PMAX];
  for (int i = threadIdx.x; i < 5 * TRI_MAX; i += blockDim.x) s_t[i] = c_tab[i];
  for (int i = threadIdx.x; i < PMAX; i += blockDim.x) s_e[i] = c_e[i];
  __syncthreads();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = g / nn, qn = g % nn;
  if (m > P) return;
  const int node = nodes[qn];
  const int4 c = cell[node];
  const Geometry gn = geo.at(node);
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  double ar[P + 1], ai[P + 1];
#pragma unroll
  for (int n = 0; n <= P; ++n) { ar[n] = 0; ai[n] = 0; }
  for (int j = plo[node]; j <= phi[node]; ++j) {
    const double x = (xs[j] - cx) * s, y = (ys[j] - cy) * s, z = (zs[j] - cz) * s;
    const double r2 = x * x + y * y + z * z;
    const double tau = q[j], dx = d3[j] * s, dy = d3[npts + j] * s, dz = d3[2 * npts + j] * s;
    // sectoral values of orders m − 1, m, m + 1
    double sr = 1.0, si = 0.0, lr = 0, li = 0, mr = 1.0, mi = 0.0, hr = 0, hi = 0;
    for (int k = 1; k <= m + 1; ++k) {
      const double e = s_e[k - 1];
      const double nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      if (k == m) { lr = sr; li = si; }
      sr = nr; si = ni;
      if (k == m) { mr = sr; mi = si; }
      if (k == m + 1) { hr = sr; hi = si; }
    }
    if (m == 0) { mr = 1.0; mi = 0.0; }
    // the chain of order k from its sectoral value (vr, vi), calling f(n′, ur, ui) for n′ = k..nmax
    auto chain = [&](int k, double vr, double vi, int nmax, auto&& f) {
      double pr = 0, pi = 0, cr = vr, ci = vi;
#pragma unroll
      for (int n = 0; n <= P; ++n) {
        if (n < k || n > nmax) continue;
        if (n > k) {
          const int t = tri(n, k);
          const double az = s_t[t] * z, br = s_t[TRI_MAX + t] * r2;
          const double nr = az * cr - br * pr, ni = az * ci - br * pi;
          pr = cr; pi = ci; cr = nr; ci = ni;
        }
        f(n, cr, ci);
      }
    };
    chain(m, mr, mi, P, [&](int n, double ur, double ui) {
      ar[n] += tau * ur;
      ai[n] -= tau * ui;
      if (n < P) {
        const double cc = s_t[2 * TRI_MAX + tri(n + 1, m)] * dz;
        ar[n + 1] += cc * ur;
        ai[n + 1] -= cc * ui;
      }
    });
    if (m >= 1)
      chain(m - 1, lr, li, P - 1, [&](int n, double ur, double ui) {
        const double cc = 0.5 * s_t[3 * TRI_MAX + tri(n + 1, m)];
        ar[n + 1] += -cc * (dx * ur - dy * ui);
        ai[n + 1] += cc * (dx * ui + dy * ur);
      });
    if (m + 1 <= P - 1)
      chain(m + 1, hr, hi, P - 1, [&](int n, double ur, double ui) {
        if (m >= 1) {
          const double cc = 0.5 * s_t[4 * TRI_MAX + tri(n + 1, m)];
          ar[n + 1] += cc * (dx * ur + dy * ui);
          ai[n + 1] += cc * (dy * ur - dx * ui);
        } else {
          ar[n + 1] += s_t[4 * TRI_MAX + tri(n + 1, 0)] * (dx * ur + dy * ui);
        }
      });
  }
  double* col = M + (int64_t)node * pitch;
#pragma unroll
  for (int n = 0; n <= P; ++n) {
    if (n < m) continue;
    if (m == 0) col[n * n] = ar[n];
    else { col[n * n + 2 * m - 1] = ar[n]; col[n * n + 2 * m] = ai[n]; }
  }
}

// ---------------------------------------------------------------- P2M
// one thread per (node, order m): M_n^m += τ conj Υ̃_n^m((y − c)/w) over the node's sources,
// n = m..P, the chain of order m started from its own sectoral value (harmonics.jl:682-743)
// Yukawa3D (YK): the degree-n terms weighted by u_n(κ̂|x̂|), κ̂² = kh2[level]
// (harmonics_yukawa.jl:281-296). R = float on the mixed path of Laplace3D (box-centred, scaled
// coordinates in [−½, ½]³, sums over the box's sources in FP32, written as doubles: about 2⁻²⁴
// per coefficient, below the FP16x3 M2L's 2⁻²² that consumes them).
template <int P, bool YK, typename R>
__global__ void k_p2m(const int* __restrict__ nodes, int nn, const int4* __restrict__ cell, const int* __restrict__ plo,
                      const int* __restrict__ phi, const double* __restrict__ xs, const double* __restrict__ ys,
                      const double* __restrict__ zs, const double* __restrict__ q, Geometry geo,
                      const double* __restrict__ scale, int64_t pitch, double* __restrict__ M,
                      const double* __restrict__ kh2) {
  static_assert(!YK || sizeof(R) == 8, "Yukawa3D's P2M runs in FP64");
  // the recurrence tables in shared memory: the lanes of a warp run different orders and would
  // serialise on the constant cache
  __shared__ R s_ab[2 * TRI_MAX];
  __shared__ R s_e[PMAX];
  for (int i = threadIdx.x; i < 2 * TRI_MAX; i += blockDim.x) s_ab[i] = ctab<R>(i);
  for (int i = threadIdx.x; i < PMAX; i += blockDim.x) s_e[i] = ce<R>(i);
  __syncthreads();
  // thread g: order m = g / nn of node g % nn; the lanes of a warp share the order, so the
  // recurrence's branches on n versus m are uniform
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int m = g / nn, qn = g % nn;
  if (m > P) return;
  int node = nodes[qn];
  int4 c = cell[node];
  const Geometry gn = geo.at(node);
  double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  const double k2 = YK ? kh2[c.w] : 0.0;
  R ar[P + 1], ai[P + 1];
#pragma unroll
  for (int n = 0; n <= P; ++n) { ar[n] = 0; ai[n] = 0; }
  int j1 = phi[node];
  for (int j = plo[node]; j <= j1; ++j) {
    const R x = R((xs[j] - cx) * s), y = R((ys[j] - cy) * s), z = R((zs[j] - cz) * s);
    const R r2 = x * x + y * y + z * z;
    R sr = 1, si = 0;
    for (int k = 1; k <= m; ++k) {
      const R e = s_e[k - 1];
      const R nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      sr = nr; si = ni;
    }
    const R tau = R(q[j]);
    double u[P + 1];
    if constexpr (YK) yukawa_u<P>(k2 * (double)r2, u);
    R pr = 0, pi = 0, cr = 0, ci = 0;
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      R tn = tau;
      if constexpr (YK) tn = tau * u[n];
      if (n == m) {
        cr = sr; ci = si; pr = 0; pi = 0;
        ar[n] += tn * cr; ai[n] -= tn * ci;
      } else if (n > m) {
        int t = tri(n, m);
        const R az = s_ab[t] * z, br = s_ab[TRI_MAX + t] * r2;
        const R nr = az * cr - br * pr, ni = az * ci - br * pi;
        pr = cr; pi = ci; cr = nr; ci = ni;
        ar[n] += tn * nr; ai[n] -= tn * ni;
      }
    }
  }
  double* col = M + (int64_t)node * pitch;
#pragma unroll
  for (int n = 0; n <= P; ++n) {
    if (n < m) continue;
    if (m == 0) col[n * n] = (double)ar[n];
    else { col[n * n + 2 * m - 1] = (double)ar[n]; col[n * n + 2 * m] = (double)ai[n]; }
  }
}

// ---------------------------------------------------------------- GEMM over mapped columns (M2M, L2L)

// one FP64 tensor-core MMA, D(8×8) += A(8×4)·B(4×8): this lane holds A[g][t], B[t][g] and
// D[g][2t], D[g][2t+1] (g = lane / 4, t = lane % 4)
__device__ __forceinline__ void dmma_gemm(double* d, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// C(:, g) (=|+=) A · B(:, g) for mapped columns g; A column-major M × K; rows r with r mod LD ≥ NP
// written as 0. 128 × BN tiles on the FP64 tensor cores (DMMA): warp w the rows [16w, 16w + 16) ×
// all BN columns; K-slabs of 32 in shared memory (row strides of 4 mod 16 doubles: conflict-free
// fragment loads), the next slab prefetched into registers. Padding is not multiplied where it
// fills whole units of the loop: a warp whose 16 rows all have r mod LD ≥ NP (or lie past M)
// skips its MMAs, and, when KLD > 0, a slab whose columns k all have k mod KLD ≥ KNP is skipped —
// the caller guarantees that those columns of A are zero (M2M and L2L: the expansions' padded
// entries). The inner loop itself stays branch-free.
template <int BN>
__global__ void __launch_bounds__(256) k_gemm_tiles(int M, int K, const double* __restrict__ A, ColMap bm, ColMap cm,
                                                    int ncols, int LD, int NP, int accumulate, int KLD, int KNP) {
  constexpr int BM = 128, BK = 32, NT = BN / 8, LDA = BM + 4, LDB = BN + 4;
  constexpr int AL = BM * BK / 256, BL = (BK * BN + 255) / 256;
  __shared__ double As[BK * LDA];
  __shared__ double Bs[BK * LDB];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int row0 = blockIdx.y * BM, col0 = blockIdx.x * BN;
  // padding: rows (8-row sub-tiles of this warp) and K ranges with nothing to multiply
  auto pad_rows = [&](int r, int n) { const int m = r % LD; return r >= M || (m >= NP && m + n <= LD); };
  auto pad_k = [&](int k, int n) {
    if (KLD <= 0) return false;
    const int m = k % KLD;
    return m >= KNP && m + n <= KLD;
  };
  const bool live = !pad_rows(row0 + 16 * warp, 16);
  double acc[2][NT][2];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
  double ra[AL], rb[BL];
  const double* bcol[BL];
#pragma unroll
  for (int u = 0; u < BL; ++u) {
    const int e = tid + 256 * u, j = e / BK;
    bcol[u] = (e < BK * BN && col0 + j < ncols) ? bm.col(col0 + j, LD) : nullptr;
  }
  auto load = [&](int k0) {
#pragma unroll
    for (int u = 0; u < AL; ++u) {
      const int e = tid + 256 * u, i = e % BM, k = e / BM;
      ra[u] = (k0 + k < K && row0 + i < M) ? A[(int64_t)(k0 + k) * M + row0 + i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < BL; ++u) {
      const int e = tid + 256 * u, k = e % BK;
      rb[u] = (bcol[u] && k0 + k < K) ? bcol[u][k0 + k] : 0.0;
    }
  };
  // the slabs with something to multiply, in order
  auto next_slab = [&](int k) {
    while (k < K && pad_k(k, BK)) k += BK;
    return k;
  };
  int k0 = next_slab(0);
  if (k0 < K) load(k0);
  for (; k0 < K;) {
    const int k1 = next_slab(k0 + BK);
    __syncthreads();
#pragma unroll
    for (int u = 0; u < AL; ++u) { const int e = tid + 256 * u; As[(e / BM) * LDA + e % BM] = ra[u]; }
#pragma unroll
    for (int u = 0; u < BL; ++u) { const int e = tid + 256 * u; if (e < BK * BN) Bs[(e % BK) * LDB + e / BK] = rb[u]; }
    __syncthreads();
    if (k1 < K) load(k1);
    if (live) {                                        // uniform across the warp
#pragma unroll
      for (int ks = 0; ks < BK; ks += 4) {
        double af[2], bf[NT];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) af[mt] = As[(ks + t) * LDA + 16 * warp + 8 * mt + g];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) bf[nt] = Bs[(ks + t) * LDB + 8 * nt + g];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) dmma_gemm(acc[mt][nt], af[mt], bf[nt]);
      }
    }
    k0 = k1;
  }
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int gc = col0 + 8 * nt + 2 * t + i;
      if (gc >= ncols) continue;
      double* C = cm.col(gc, LD);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int row = row0 + 16 * warp + 8 * mt + g;
        if (row >= M) continue;
        const double v = (row % LD) < NP ? acc[mt][nt][i] : 0.0;
        C[row] = accumulate ? C[row] + v : v;
      }
    }
}

// the column-tile width: enough tiles to cover the SMs
void gemm_cols(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate, int num_sms,
               cudaStream_t s, int KLD = 0, int KNP = 0) {
  const int rows = (M + 127) / 128;
  if ((int64_t)rows * ((ncols + 31) / 32) >= num_sms) {
    k_gemm_tiles<32><<<dim3((ncols + 31) / 32, rows), 256, 0, s>>>(M, K, A, bm, cm, ncols, LD, NP, accumulate, KLD, KNP);
  } else if ((int64_t)rows * ((ncols + 15) / 16) >= num_sms) {
    k_gemm_tiles<16><<<dim3((ncols + 15) / 16, rows), 256, 0, s>>>(M, K, A, bm, cm, ncols, LD, NP, accumulate, KLD, KNP);
  } else {
    k_gemm_tiles<8><<<dim3((ncols + 7) / 8, rows), 256, 0, s>>>(M, K, A, bm, cm, ncols, LD, NP, accumulate, KLD, KNP);
  }
  FMMB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- locate and bucketing
__global__ void k_locate(const double* __restrict__ tg, int64_t nt, const int4* __restrict__ cell,
                         const int* __restrict__ cf, const uint8_t* __restrict__ flags, Geometry geo,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ idx, int* __restrict__ bad) {
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nt) return;
  double x[3] = {tg[3 * q], tg[3 * q + 1], tg[3 * q + 2]};
  bool inside = true;
  for (int d = 0; d < 3; ++d) inside = inside && geo.origin[d] <= x[d] && x[d] <= geo.origin[d] + geo.W0;
  int i = 0;
  if (!inside) { atomicExch(bad, 1); i = 0; }
  else {
    while (!(flags[i] & F_LEAF)) {
      int4 c = cell[i];
      double w = ldexp(geo.W0, -c.w);
      int k = (x[0] > geo.center(0, c.x, w)) | ((x[1] > geo.center(1, c.y, w)) << 1) | ((x[2] > geo.center(2, c.z, w)) << 2);
      i = cf[i] + k;
    }
  }
  keys[q] = ((uint64_t)i << 32) | (uint64_t)q;
  idx[q] = (uint32_t)q;
}

__global__ void k_bucket_gather(const uint64_t* __restrict__ keys, int64_t nt, const double* __restrict__ tg,
                                double* __restrict__ tx, double* __restrict__ ty, double* __restrict__ tz,
                                int* __restrict__ tout, int* __restrict__ start_flag) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  uint64_t key = keys[k];
  int64_t q = (int64_t)(uint32_t)key;
  tx[k] = tg[3 * q];
  ty[k] = tg[3 * q + 1];
  tz[k] = tg[3 * q + 2];
  tout[k] = (int)q;
  start_flag[k] = (k == 0) || ((keys[k - 1] >> 32) != (key >> 32));
}

__global__ void k_groups(const uint64_t* __restrict__ keys, const int* __restrict__ start_flag, const int* __restrict__ pos,
                         int64_t nt, int ng, int* __restrict__ gnode, int* __restrict__ gstart, int* __restrict__ gcount) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt || !start_flag[k]) return;
  int g = pos[k];
  gnode[g] = (int)(keys[k] >> 32);
  gstart[g] = (int)k;
  // the count: up to the next start
  int64_t e = k + 1;
  while (e < nt && !start_flag[e]) ++e;
  gcount[g] = (int)(e - k);
}

// ---------------------------------------------------------------- bounds
__global__ void k_bounds(const double* __restrict__ xyz, int64_t n, double* __restrict__ out, unsigned long long* __restrict__ bad) {
  __shared__ double s[6][256];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  unsigned long long nb = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      double v = xyz[3 * j + d];
      if (!isfinite(v)) { ++nb; continue; }
      lo[d] = fmin(lo[d], v);
      hi[d] = fmax(hi[d], v);
    }
  for (int d = 0; d < 3; ++d) { s[d][threadIdx.x] = lo[d]; s[3 + d][threadIdx.x] = hi[d]; }
  if (nb) atomicAdd(bad, nb);
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + h]);
        s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + h]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) out[blockIdx.x * 6 + threadIdx.x] = s[threadIdx.x][0];
}

// the bounds of each instance of a batch: blockIdx.y the instance (points [off[i], off[i + 1])),
// its gridDim.x blocks reduce over it as k_bounds does
__global__ void k_bounds_batch(const double* __restrict__ xyz, const int64_t* __restrict__ off, double* __restrict__ out,
                               unsigned long long* __restrict__ bad) {
  const int64_t a = off[blockIdx.y], n = off[blockIdx.y + 1] - a;
  __shared__ double s[6][256];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  unsigned long long nb = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      double v = xyz[3 * (a + j) + d];
      if (!isfinite(v)) { ++nb; continue; }
      lo[d] = fmin(lo[d], v);
      hi[d] = fmax(hi[d], v);
    }
  for (int d = 0; d < 3; ++d) { s[d][threadIdx.x] = lo[d]; s[3 + d][threadIdx.x] = hi[d]; }
  if (nb) atomicAdd(bad, nb);
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + h]);
        s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + h]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) out[((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = s[threadIdx.x][0];
}

// P2M of charges q (and, when d3 is given, dipoles d3: 3 × N planar) into M (pitch per node)
template <int P>
void launch_p2m(State& S, const double* q, const double* d3, double* M, int64_t pitch) {
  Plan& P_ = *S.plan;
  int nth = P_.n_s2m * (P + 1);
  if (nth == 0) return;
  if (d3) {
    k_p2m_dip<P><<<nblk(nth, 128), 128, 0, P_.ctx->stream>>>(P_.s2m_nodes.p, P_.n_s2m, P_.cell.p, P_.plo.p, P_.phi.p, S.xs.p,
                                                           S.ys.p, S.zs.p, q, d3, P_.N, geometry(P_), P_.d_scale.p,
                                                           pitch, M);
    FMMB_LAUNCH_CHECK();
    return;
  }
  // FP32 on the mixed path of Laplace3D (charges only), FP64 otherwise
  auto kern = P_.cache->kernel == FMMB_KERNEL_YUKAWA3D ? k_p2m<P, true, double>
              : (S.precision == FMMB_PRECISION_MIXED && P_.cache->kernel == FMMB_KERNEL_LAPLACE3D) ? k_p2m<P, false, float>
                                                                                                  : k_p2m<P, false, double>;
  kern<<<nblk(nth, 128), 128, 0, P_.ctx->stream>>>(P_.s2m_nodes.p, P_.n_s2m, P_.cell.p, P_.plo.p, P_.phi.p, S.xs.p, S.ys.p,
                                                 S.zs.p, q, geometry(P_), P_.d_scale.p, pitch, M, P_.d_kh2.p);
  FMMB_LAUNCH_CHECK();
}



}  // namespace

// ---------------------------------------------------------------- direct sums, FP64
// (shared by fmmb_direct_dev and fmmb_direct_noalloc_dev; declared in passes.cuh)
__global__ void __launch_bounds__(DT) k_direct(const double* __restrict__ src, const double* __restrict__ tau, int64_t ns,
                                               const double* __restrict__ tgt, const int64_t* __restrict__ self_idx,
                                               int64_t nt, int nsplit, double* __restrict__ part) {
  __shared__ double sx[DT], sy[DT], sz[DT], sq[DT];
  int64_t t = (int64_t)blockIdx.x * DT + threadIdx.x;
  int sp = blockIdx.y;
  int64_t s0 = ns * sp / nsplit, s1 = ns * (sp + 1) / nsplit;
  bool act = t < nt;
  double x = act ? tgt[3 * t] : 0, y = act ? tgt[3 * t + 1] : 0, z = act ? tgt[3 * t + 2] : 0;
  int64_t me = (act && self_idx) ? self_idx[t] : -1;
  double u = 0, gx = 0, gy = 0, gz = 0;
  for (int64_t b = s0; b < s1; b += DT) {
    __syncthreads();
    int64_t j = b + threadIdx.x;
    if (j < s1) { sx[threadIdx.x] = src[3 * j]; sy[threadIdx.x] = src[3 * j + 1]; sz[threadIdx.x] = src[3 * j + 2]; sq[threadIdx.x] = tau[j]; }
    __syncthreads();
    int m = (int)min((int64_t)DT, s1 - b);
    for (int i = 0; i < m; ++i) {
      double dx = x - sx[i], dy = y - sy[i], dz = z - sz[i];
      double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
      double ir = (b + i == me) ? 0.0 : 1.0 / sqrt(r2);
      double qi = sq[i] * ir, qi3 = qi * ir * ir;
      u += qi; gx += qi3 * dx; gy += qi3 * dy; gz += qi3 * dz;
    }
  }
  if (act) {
    double* o = part + ((int64_t)sp * nt + t) * 4;
    o[0] = u; o[1] = gx; o[2] = gy; o[3] = gz;
  }
}

__global__ void k_direct_reduce(const double* __restrict__ part, int64_t nt, int nsplit, double* __restrict__ pot,
                                double* __restrict__ grad) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double u = 0, gx = 0, gy = 0, gz = 0;
  for (int sp = 0; sp < nsplit; ++sp) {
    const double* o = part + ((int64_t)sp * nt + t) * 4;
    u += o[0]; gx += o[1]; gy += o[2]; gz += o[3];
  }
  if (pot) pot[t] = KC * u;
  if (grad) { grad[3 * t] = -KC * gx; grad[3 * t + 1] = -KC * gy; grad[3 * t + 2] = -KC * gz; }
}


Geometry geometry(const Plan& P) {
  Geometry g;
  for (int d = 0; d < 3; ++d) g.origin[d] = P.origin[d];
  g.W0 = P.W0;
  g.node_inst = P.ninst > 1 ? P.node_inst.p : nullptr;
  g.inst_box = P.ninst > 1 ? P.d_inst_box.p : nullptr;
  return g;
}

void upload_operators(Cache& C) {
  cudaStream_t s = C.ctx->stream;
  const HostOperators& h = C.host;
  to_device(C.m2m, h.m2m, s);
  to_device(C.l2l, h.l2l, s);
  to_device(C.reps, h.reps, s);
  to_device(C.tables, h.tables, s);
  to_device(C.gidx, h.gidx, s);
  to_device(C.gsgn, h.gsgn, s);
  to_device(C.sidx, h.sidx, s);
  to_device(C.ssgn, h.ssgn, s);
  to_device(C.cls, h.cls, s);
  upload_d4h(h, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
  C.uploaded = true;
}

void gather_inputs(State& S, const double* xyz_dev, const double* tau_dev) {
  Plan& P = *S.plan;
  require(P.cache->kernel != FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "a Stokeslet state takes fmmb_stokes_eval");
  k_gather_inputs<<<nblk(P.N), 256, 0, P.ctx->stream>>>(xyz_dev, tau_dev, P.perm.p, P.N, S.xs.p, S.ys.p, S.zs.p, S.q.p);
  FMMB_LAUNCH_CHECK();
  S.has_dip = false;
}

void gather_inputs_dipoles(State& S, const double* xyz_dev, const double* tau_dev, const double* dip_dev) {
  Plan& P = *S.plan;
  require(P.cache->kernel == FMMB_KERNEL_LAPLACE3D && P.cache->method == FMMB_METHOD_SPHERICAL_HARMONICS,
          FMMB_ERR_UNSUPPORTED, "dipole densities are provided for SphericalHarmonics(Laplace3D)");
  if (S.dip.n < (size_t)(3 * P.N)) S.dip.alloc(3 * P.N);
  k_gather_dipoles<<<nblk(P.N), 256, 0, P.ctx->stream>>>(xyz_dev, tau_dev, dip_dev, P.perm.p, P.N, S.xs.p, S.ys.p, S.zs.p,
                                                         S.q.p, S.dip.p);
  FMMB_LAUNCH_CHECK();
  S.has_dip = dip_dev != nullptr;
}


void p2m_block(State& S, const double* q, const double* d3, double* M, int64_t pitch) {
  switch (S.plan->cache->p) {
#define X(pp) case pp: launch_p2m<pp>(S, q, d3, M, pitch); break;
    FMMB_P_CASES(X)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "p out of range");
  }
}

void gemm_columns(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                  int num_sms, cudaStream_t s) {
  gemm_cols(M, K, A, bm, cm, ncols, LD, NP, accumulate, num_sms, s);
}

void gemm_expansions(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                     int num_sms, cudaStream_t s) {
  gemm_cols(M, K, A, bm, cm, ncols, LD, NP, accumulate, num_sms, s, LD, NP);
}

int p2m(State& S) {
  if (S.plan->cache->method == FMMB_METHOD_CUBE_KI) return ki_p2m(S);
  if (S.plan->cache->method == FMMB_METHOD_KI_CIRCLE) return kic_p2m(S);
  switch (S.plan->cache->p) {
#define X(pp) case pp: launch_p2m<pp>(S, S.q.p, S.has_dip ? S.dip.p : nullptr, S.M.p, (int64_t)S.plan->cache->ld); break;
    FMMB_P_CASES(X)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "p out of range");
  }
  return S.plan->n_s2m > 0;
}

int m2m_sweep(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  int launches = 0;
  for (int l = P.L - 2; l >= 2; --l) {
    int c0 = P.level_start[l + 1], ng = P.level_groups[l + 1];
    if (ng == 0) continue;
    ColMap bm{S.M.p, nullptr, c0, NCH}, cm{S.M.p, P.group_parent[l + 1].p, 0, 0};
    gemm_cols(C.ld, NCH * C.ld, P.lv_m2m[l], bm, cm, ng, C.ld, C.np, 0, P.ctx->num_sms, s, C.ld, C.np);
    ++launches;
  }
  return launches;
}

void State::Side::ensure() {
  if (s) return;
  int lo = 0, hi = 0;
  FMMB_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  FMMB_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, lo));   // the lowest priority
  FMMB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  FMMB_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
}

State::Side::~Side() {
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
}

void upward_pass(State& S) {
  p2m(S);
  m2m_sweep(S);
}


int l2l_sweep(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  int launches = 0;
  for (int l = 3; l < P.L; ++l) {
    int c0 = P.level_start[l], ng = P.level_groups[l];
    if (ng == 0) continue;
    ColMap bm{S.Pl.p, P.group_parent[l].p, 0, 0}, cm{S.Pl.p, nullptr, c0, NCH};
    gemm_cols(NCH * C.ld, C.ld, P.lv_l2l[l - 1], bm, cm, ng, C.ld, C.np, 1, P.ctx->num_sms, s, C.ld, C.np);
    ++launches;
  }
  // the kernel-independent method: the leaves' local densities from their check potentials
  if (C.method == FMMB_METHOD_CUBE_KI) launches += ki_leaf_locals(S);
  if (C.method == FMMB_METHOD_KI_CIRCLE) launches += kic_leaf_locals(S);
  return launches;
}

// the partial locals zeroed, then the M2L of every level in one launch (plus the FP16
// copy of the multipoles on the mixed path); returns the kernel launches
int m2l_stage(State& S) {
  Plan& P = *S.plan;
  FMMB_CUDA(cudaMemsetAsync(S.Pl.p, 0, S.Pl.bytes(), P.ctx->stream));
  if (P.cache->method == FMMB_METHOD_CUBE_KI) return ki_m2l(S);
  if (P.cache->method == FMMB_METHOD_KI_CIRCLE) return kic_m2l(S);
  if (P.h_blocks.empty()) return 0;
  if (S.precision == FMMB_PRECISION_MIXED) {
    m2l_mixed(S);
    return 4;
  }
  m2l_f64(S);
  return 1;
}

void downward_pass(State& S) {
  m2l_stage(S);
  l2l_sweep(S);
}


void evaluate_sources(State& S, int outputs, double* pot, double* grad) {
  Plan& P = *S.plan;
  require(P.cache->kernel != FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "a Stokeslet state takes fmmb_stokes_eval");
  evaluate_groups(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, S.xs.p, S.ys.p, S.zs.p, P.perm.p, true, outputs,
                  pot, grad);
}

void evaluate_targets(State& S, const double* tg, int64_t nt, int outputs, double* pot, double* grad) {
  Plan& P = *S.plan;
  require(P.cache->kernel != FMMB_KERNEL_STOKESLET3D, FMMB_ERR_UNSUPPORTED, "a Stokeslet state takes fmmb_stokes_eval");
  if (nt == 0) return;
  const int ng = group_targets(S, tg, nt);
  const int* gnode = S.t_groups.p;
  evaluate_groups(S, gnode, gnode + ng, gnode + 2 * ng, ng, S.t_x.p, S.t_y.p, S.t_z.p, S.t_out.p, false, outputs, pot, grad);
  FMMB_CUDA(cudaStreamSynchronize(P.ctx->stream));
}

int group_targets(State& S, const double* tg, int64_t nt) {
  Plan& P = *S.plan;
  cudaStream_t s = P.ctx->stream;
  require(P.ninst == 1, FMMB_ERR_UNSUPPORTED, "a batch plan evaluates at its sources only");
  require(nt < (1ll << 31) - 1, FMMB_ERR_ARGUMENT, "too many targets");
  if ((int64_t)S.t_x.n < nt) {
    S.t_x.alloc(nt); S.t_y.alloc(nt); S.t_z.alloc(nt); S.t_out.alloc(nt); S.t_node.alloc(nt);
    S.t_keys.alloc(nt); S.t_vals.alloc(nt); S.t_groups.alloc(3 * nt + 3);
  }
  DBuf<int> bad(1), pos(nt);
  FMMB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  k_locate<<<nblk(nt), 256, 0, s>>>(tg, nt, P.cell.p, P.cf.p, P.flags.p, geometry(P), S.t_keys.p, S.t_vals.p, bad.p);
  FMMB_LAUNCH_CHECK();
  require(read_one(bad.p, s) == 0, FMMB_ERR_ARGUMENT, "a target lies outside the tree's box");
  int nbits = 1;
  while ((1ll << nbits) < (int64_t)P.nnodes) ++nbits;
  radix_sort_pairs(S.t_keys.p, S.t_vals.p, nt, 32 + nbits, s);
  k_bucket_gather<<<nblk(nt), 256, 0, s>>>(S.t_keys.p, nt, tg, S.t_x.p, S.t_y.p, S.t_z.p, S.t_out.p, S.t_node.p);
  FMMB_LAUNCH_CHECK();
  int ng = (int)scan_exclusive_total(S.t_node.p, pos.p, nt, s);
  int* gnode = S.t_groups.p;
  int* gstart = gnode + ng;
  int* gcount = gstart + ng;
  k_groups<<<nblk(nt), 256, 0, s>>>(S.t_keys.p, S.t_node.p, pos.p, nt, ng, gnode, gstart, gcount);
  FMMB_LAUNCH_CHECK();
  return ng;   // pos and the flag are freed in stream order
}

void bounds(Ctx& ctx, const double* xyz, int64_t n, double lo[3], double hi[3], int64_t* nonfinite) {
  cudaStream_t s = ctx.stream;
  int nb = (int)std::min<int64_t>(std::max<int64_t>(1, (n + 255) / 256), 4 * ctx.num_sms);
  DBuf<double> out((size_t)nb * 6);
  DBuf<unsigned long long> bad(1);
  FMMB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(unsigned long long), s));
  k_bounds<<<nb, 256, 0, s>>>(xyz, n, out.p, bad.p);
  FMMB_LAUNCH_CHECK();
  std::vector<double> h = to_host(out.p, (size_t)nb * 6, s);
  *nonfinite = (int64_t)read_one(bad.p, s);
  for (int d = 0; d < 3; ++d) { lo[d] = INFINITY; hi[d] = -INFINITY; }
  for (int b = 0; b < nb; ++b)
    for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], h[b * 6 + d]); hi[d] = std::max(hi[d], h[b * 6 + 3 + d]); }
}

void bounds_batch(Ctx& ctx, const double* xyz, const std::vector<int64_t>& off, std::vector<double>& lo,
                  std::vector<double>& hi, int64_t* nonfinite) {
  cudaStream_t s = ctx.stream;
  const int ninst = (int)off.size() - 1;
  int64_t nmax = 1;
  for (int i = 0; i < ninst; ++i) nmax = std::max<int64_t>(nmax, off[i + 1] - off[i]);
  // blocks per instance: enough for the largest, and about four waves over all instances
  const int nbx = (int)std::max<int64_t>(1, std::min<int64_t>((nmax + 255) / 256, (4 * ctx.num_sms + ninst - 1) / ninst));
  DBuf<int64_t> d_off;
  to_device(d_off, off, s);
  DBuf<double> out((size_t)ninst * nbx * 6);
  DBuf<unsigned long long> bad(1);
  FMMB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(unsigned long long), s));
  k_bounds_batch<<<dim3(nbx, ninst), 256, 0, s>>>(xyz, d_off.p, out.p, bad.p);
  FMMB_LAUNCH_CHECK();
  std::vector<double> h = to_host(out.p, (size_t)ninst * nbx * 6, s);
  *nonfinite = (int64_t)read_one(bad.p, s);
  lo.assign(3 * ninst, INFINITY);
  hi.assign(3 * ninst, -INFINITY);
  for (int i = 0; i < ninst; ++i)
    for (int b = 0; b < nbx; ++b)
      for (int d = 0; d < 3; ++d) {
        lo[3 * i + d] = std::min(lo[3 * i + d], h[((size_t)i * nbx + b) * 6 + d]);
        hi[3 * i + d] = std::max(hi[3 * i + d], h[((size_t)i * nbx + b) * 6 + 3 + d]);
      }
}

void direct(Ctx& ctx, const double* src, const double* tau, int64_t ns, const double* tgt, const int64_t* self_idx,
            int64_t nt, double* pot, double* grad) {
  cudaStream_t s = ctx.stream;
  if (nt == 0) return;
  int tb = (int)((nt + DT - 1) / DT);
  int nsplit = std::max(1, std::min<int>(256, (4 * ctx.num_sms + tb - 1) / tb));
  DBuf<double> part((size_t)nsplit * nt * 4);
  k_direct<<<dim3(tb, nsplit), DT, 0, s>>>(src, tau, ns, tgt, self_idx, nt, nsplit, part.p);
  FMMB_LAUNCH_CHECK();
  k_direct_reduce<<<nblk(nt), 256, 0, s>>>(part.p, nt, nsplit, pot, grad);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb
