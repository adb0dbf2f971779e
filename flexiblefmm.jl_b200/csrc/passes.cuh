// Declarations shared by the pass kernels (passes.cu, m2l_f64.cu, m2l_tc.cu, eval.cu).
#pragma once
#include "plan.cuh"

namespace fmmb {

constexpr double KC = 0.079577471545947667884;  // 1/(4π), the Laplace3D constant (src/kernels.jl:182)
__host__ __device__ constexpr int tri(int n, int m) { return n * (n + 1) / 2 + m; }
constexpr int TRI_MAX = PMAX * (PMAX + 1) / 2 + PMAX + 1;

// the root box; centres formed exactly as the tree builder forms them. A batch's instances
// have boxes of their own: at(node) gives the geometry with the node's instance's origin.
struct Geometry {
  double origin[3];
  double W0;
  const int* node_inst;     // a batch: per node its instance, and per instance its box (4 each)
  const double* inst_box;
  __device__ __forceinline__ double center(int d, int c, double w) const {
    return __dadd_rn(origin[d], __dmul_rn(__dadd_rn((double)c, 0.5), w));
  }
  __device__ __forceinline__ Geometry at(int node) const {
    Geometry g = *this;
    if (node_inst) {
      const double* b = inst_box + 4 * node_inst[node];
      g.origin[0] = b[0]; g.origin[1] = b[1]; g.origin[2] = b[2];
    }
    return g;
  }
};
Geometry geometry(const Plan& P);

extern __constant__ double c_tab[5 * TRI_MAX];
extern __constant__ double c_e[PMAX];
extern __constant__ float c_tabf[5 * TRI_MAX];   // the same tables in FP32 (the mixed path's L2P)
extern __constant__ float c_ef[PMAX];
void init_device_constants(cudaStream_t s);

template <typename R> __device__ __forceinline__ R ctab(int i);
template <> __device__ __forceinline__ double ctab<double>(int i) { return c_tab[i]; }
template <> __device__ __forceinline__ float ctab<float>(int i) { return c_tabf[i]; }
template <typename R> __device__ __forceinline__ R ce(int i);
template <> __device__ __forceinline__ double ce<double>(int i) { return c_e[i]; }
template <> __device__ __forceinline__ float ce<float>(int i) { return c_ef[i]; }

// L2P at x̂ (potential and the gradient before the 1/w factor) from the local L in shared
// memory, in precision R (FP64 on the plain path, FP32 on the mixed path); the orders run as a
// loop (a full unroll keeps too many coefficients in registers)
template <int P, typename R>
__device__ __forceinline__ void l2p(const R* __restrict__ L, R x, R y, R z, R& u, R& gx, R& gy, R& gz) {
  R r2 = x * x + y * y + z * z;
  R sr = 1, si = 0;
  u = 0; gx = 0; gy = 0; gz = 0;
#pragma unroll 1
  for (int m = 0; m <= P; ++m) {
    R pr = 0, pi = 0, cr = sr, ci = si;
#pragma unroll 2
    for (int n = m; n <= P; ++n) {
      R vr, vi;
      if (n == m) { vr = sr; vi = si; }
      else {
        const int t = tri(n, m);
        R az = ctab<R>(t) * z, br = ctab<R>(TRI_MAX + t) * r2;
        vr = az * cr - br * pr; vi = az * ci - br * pi;
        pr = cr; pi = ci; cr = vr; ci = vi;
      }
      // potential: Σ L_n^m conj Υ̃ (harmonics.jl:455-462)
      if (m == 0) u += L[n * n] * vr;
      else u += 2 * (L[n * n + 2 * m - 1] * vr + L[n * n + 2 * m] * vi);
      // gradient from degree n + 1 (harmonics.jl:465-486)
      if (n < P) {
        const int n1 = n + 1;
        if (m == 0) {
          R cmv = ctab<R>(3 * TRI_MAX + tri(n1, 1));
          R lr = L[n1 * n1 + 1], li = L[n1 * n1 + 2];
          gx += -cmv * lr * vr;
          gy += -cmv * li * vr;
          gz += ctab<R>(2 * TRI_MAX + tri(n1, 0)) * L[n1 * n1] * vr;
        } else {
          R ur = L[n1 * n1 + 2 * (m + 1) - 1], ui = L[n1 * n1 + 2 * (m + 1)];
          R dr, di;
          if (m == 1) { dr = L[n1 * n1]; di = 0; }
          else { dr = L[n1 * n1 + 2 * (m - 1) - 1]; di = L[n1 * n1 + 2 * (m - 1)]; }
          R cu = R(0.5) * ctab<R>(3 * TRI_MAX + tri(n1, m + 1)), cd = R(0.5) * ctab<R>(4 * TRI_MAX + tri(n1, m - 1));
          R axr = -cu * ur + cd * dr, axi = -cu * ui + cd * di;
          R ayr = -(cu * ui + cd * di), ayi = cu * ur + cd * dr;
          R czv = ctab<R>(2 * TRI_MAX + tri(n1, m));
          R zr = L[n1 * n1 + 2 * m - 1], zi = L[n1 * n1 + 2 * m];
          gx += 2 * (axr * vr + axi * vi);
          gy += 2 * (ayr * vr + ayi * vi);
          gz += 2 * czv * (zr * vr + zi * vi);
        }
      }
    }
    if (m < P) {
      R e = ce<R>(m);
      R nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      sr = nr; si = ni;
    }
  }
}

// Yukawa3D's radial factors u_n(z), n = 0..NM, from z² (harmonics_yukawa.jl:224-245): Miller's
// backward recurrence u_n = u_{n+1} + z² u_{n+2}/((2n+3)(2n+5)) started at max(NM, ⌈z⌉) + 25 and
// normalised with u_0 = sinh z / z; 1 + z²/(2(2n+3)) for z² < 1e-8
template <int NM>
__device__ __forceinline__ void yukawa_u(double z2, double (&u)[NM + 1]) {
  if (z2 < 1e-8) {
#pragma unroll
    for (int n = 0; n <= NM; ++n) u[n] = 1 + z2 / (2 * (2 * n + 3));
    return;
  }
  const double z = sqrt(z2);
  const int N = max(NM, (int)ceil(z)) + 25;
  double a = 0, b = 1;
  for (int n = N - 1; n > NM; --n) {
    const double c = b + z2 * a / (double)((2 * n + 3) * (2 * n + 5));
    a = b;
    b = c;
  }
#pragma unroll
  for (int n = NM; n >= 0; --n) {
    const double c = b + z2 * a / (double)((2 * n + 3) * (2 * n + 5));
    u[n] = c;
    a = b;
    b = c;
  }
  const double s = (sinh(z) / z) / b;
#pragma unroll
  for (int n = 0; n <= NM; ++n) u[n] *= s;
}

// Yukawa3D's L2P at x̂ (harmonics_yukawa.jl:298-313): the potential Σ u_n(κ̂|x̂|) L_n^m conj Υ̃_n^m;
// the gradient (before the 1/w factor) the Laplace identities weighted by u_n of the local's
// degree, plus x̂ Σ κ̂² u_{n+1}/(2n+3) L_n^m conj Υ̃_n^m (from u_n'(z) = z u_{n+1}(z)/(2n+3))
template <int P>
__device__ __forceinline__ void l2p_yukawa(const double* __restrict__ L, double kh2, double x, double y, double z, double& u,
                                           double& gx, double& gy, double& gz) {
  const double r2 = x * x + y * y + z * z;
  double w[P + 2];
  yukawa_u<P + 1>(kh2 * r2, w);
  double sr = 1, si = 0, rad = 0;
  u = 0; gx = 0; gy = 0; gz = 0;
#pragma unroll 1
  for (int m = 0; m <= P; ++m) {
    double pr = 0, pi = 0, cr = sr, ci = si;
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      if (n < m) continue;
      double vr, vi;
      if (n == m) { vr = sr; vi = si; }
      else {
        const int t = tri(n, m);
        const double az = c_tab[t] * z, br = c_tab[TRI_MAX + t] * r2;
        vr = az * cr - br * pr; vi = az * ci - br * pi;
        pr = cr; pi = ci; cr = vr; ci = vi;
      }
      const double term = m == 0 ? L[n * n] * vr : 2 * (L[n * n + 2 * m - 1] * vr + L[n * n + 2 * m] * vi);
      u += w[n] * term;
      rad += kh2 * w[n + 1] / (2 * n + 3) * term;
      if (n < P) {
        const int n1 = n + 1;
        const double wn = w[n1];
        if (m == 0) {
          const double cmv = c_tab[3 * TRI_MAX + tri(n1, 1)];
          gx += wn * (-cmv * L[n1 * n1 + 1] * vr);
          gy += wn * (-cmv * L[n1 * n1 + 2] * vr);
          gz += wn * (c_tab[2 * TRI_MAX + tri(n1, 0)] * L[n1 * n1] * vr);
        } else {
          const double ur = L[n1 * n1 + 2 * (m + 1) - 1], ui = L[n1 * n1 + 2 * (m + 1)];
          double dr, di;
          if (m == 1) { dr = L[n1 * n1]; di = 0; }
          else { dr = L[n1 * n1 + 2 * (m - 1) - 1]; di = L[n1 * n1 + 2 * (m - 1)]; }
          const double cu = 0.5 * c_tab[3 * TRI_MAX + tri(n1, m + 1)], cd = 0.5 * c_tab[4 * TRI_MAX + tri(n1, m - 1)];
          const double axr = -cu * ur + cd * dr, axi = -cu * ui + cd * di;
          const double ayr = -(cu * ui + cd * di), ayi = cu * ur + cd * dr;
          const double czv = c_tab[2 * TRI_MAX + tri(n1, m)];
          const double zr = L[n1 * n1 + 2 * m - 1], zi = L[n1 * n1 + 2 * m];
          gx += 2 * wn * (axr * vr + axi * vi);
          gy += 2 * wn * (ayr * vr + ayi * vi);
          gz += 2 * wn * czv * (zr * vr + zi * vi);
        }
      }
    }
    if (m < P) {
      const double e = c_e[m];
      const double nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      sr = nr; si = ni;
    }
  }
  gx += x * rad;
  gy += y * rad;
  gz += z * rad;
}

// the orders with compiled kernels
#define FMMB_P_CASES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) X(20)

// a column of a GEMM over mapped columns (M2M, L2L): column g at base + (idx ? idx[g] : off +
// stride·g)·pitch (pitch 0: the expansion length LD)
struct ColMap {
  double* base;
  const int* idx;
  int off, stride;
  int64_t pitch = 0;
  __device__ __forceinline__ double* col(int g, int LD) const {
    return base + (int64_t)(idx ? idx[g] : off + stride * g) * (pitch ? pitch : (int64_t)LD);
  }
};
// C(:, g) (=|+=) A · B(:, g) on the FP64 tensor cores; rows r with r mod LD ≥ NP written as 0
void gemm_columns(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                  int num_sms, cudaStream_t s);
// the same over expansions (K in blocks of LD whose entries k mod LD ≥ NP are zero columns of A:
// M2M and L2L), without multiplying that padding
void gemm_expansions(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                     int num_sms, cudaStream_t s);
// P2M of the childless sourced nodes with charges q (tree order) into the block at M (node pitch)
// P2M of charges q and, when d3 (3 × N planar) is given, dipoles into M (pitch doubles per node)
void p2m_block(State& S, const double* q, const double* d3, double* M, int64_t pitch);

void m2l_f64(State& S);
int p2m(State& S);          // the stages of the passes; each returns its kernel launches
int m2m_sweep(State& S);
int m2l_stage(State& S);
int l2l_sweep(State& S);
void evaluate_groups(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx,
                     const double* ty, const double* tz, const int* tout, bool self, int outputs, double* pot, double* grad);
// the mixed path (m2l_tc.cu)
void prepare_mixed_operators(Cache& C);
void prepare_mixed_levels(Plan& P);   // the cache locked by the caller
void m2l_mixed(State& S);
int mixed_error_flag(State& S);   // 1 when a bounded wait of the tensor-core M2L gave up since the last call (then cleared)
void set_m2l_stall(long long slab, double wait_s);   // the test hook of fmmb_test_m2l_stall

// FP64 direct sums at nt targets (passes.cu): per (source range sp of nsplit, target) the partial
// potential and gradient sums into part[(sp·nt + t)·4 ..], then their reduction; DT targets per CTA
constexpr int DT = 128;
__global__ void k_direct(const double* __restrict__ src, const double* __restrict__ tau, int64_t ns,
                         const double* __restrict__ tgt, const int64_t* __restrict__ self_idx, int64_t nt, int nsplit,
                         double* __restrict__ part);
__global__ void k_direct_reduce(const double* __restrict__ part, int64_t nt, int nsplit, double* __restrict__ pot,
                                double* __restrict__ grad);
// resolves the no-allocation scratch array's device address for the current device and context
// (direct_noalloc.cu; called when a context is created)
void direct_noalloc_prepare();

}  // namespace fmmb
