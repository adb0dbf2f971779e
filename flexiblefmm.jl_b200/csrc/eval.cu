// Evaluation at the targets of one leaf (src/evaluate.jl:12-48, src/device.jl:89-100,185-206),
// in two kernels:
//   k_l2p   the far field: L2P of the leaf's local expansion (harmonics.jl:447-486), one warp
//           per leaf group with the local staged in shared memory, lanes over the targets; FP64 on
//           the plain path, FP32 on the mixed path (tolerances ≥ 1e-8); writes the outputs
//   k_near  the near field: the sources of the 27 colleagues, flattened into batches of 32 that
//           each warp stages once in shared memory while the next batch's loads are in flight;
//           lanes over the targets; adds to the outputs. The self term is skipped by index
//           (evaluate_at_sources, src/evaluate.jl:1-10), checked only in the batches that hold
//           the leaf's own points.
// Two precisions of the near field:
//   double  the plain path: absolute coordinates, the reference's FMA square norm
//           (src/kernels.jl:20-24) and its summation order (colleagues in order, points in order)
//   float   the mixed path: coordinates relative to the target leaf's centre, converted from FP64
//           when staged (the FP32 differences carry an absolute error of ~2⁻²⁴·w instead of
//           2⁻²⁴·|x|, so close pairs keep their accuracy); two sources per packed f32x2
//           instruction; each batch summed in FP32, the batch sums accumulated in FP64
// Splitting the two keeps the near-field loop at a low register count (high occupancy); the
// outputs are u then u + KC·near, the same arithmetic as one fused pass.
#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int NEAR_WARPS = 4;

// The leaf's local expansion prepared for L2P (harmonics.jl:447-486): per (m, n), m-major, eight
// values — the potential's coefficient pair and the three gradient components' pairs (each from
// the degree-(n+1) coefficients and the recurrence tables), the factor 2 of the m ≥ 1 terms
// folded in — so that every term of the point loop is a complex dot product a·v with the
// regular harmonic v = Υ̃_n^m(x̂). Built once per leaf (FP64, then rounded to R).
template <int P>
__host__ __device__ constexpr int l2p_entries() { return (P + 1) * (P + 2) / 2; }
__device__ __forceinline__ int l2p_entry(int P, int m, int n) { return m * (P + 1) - m * (m - 1) / 2 + n - m; }

template <int P, typename R>
__device__ void l2p_prepare(const double* __restrict__ L, R* __restrict__ E, int lane) {
  for (int q = lane; q < l2p_entries<P>(); q += 32) {
    int m = 0, rem = q;
    while (rem >= P + 1 - m) { rem -= P + 1 - m; ++m; }
    const int n = m + rem;
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // potential: Σ L_n^m conj Υ̃ (harmonics.jl:455-462)
    if (m == 0) v[0] = L[n * n];
    else { v[0] = 2 * L[n * n + 2 * m - 1]; v[1] = 2 * L[n * n + 2 * m]; }
    // gradient from degree n + 1 (harmonics.jl:465-486)
    if (n < P) {
      const int n1 = n + 1;
      if (m == 0) {
        const double cmv = ctab<double>(3 * TRI_MAX + tri(n1, 1));
        v[2] = -cmv * L[n1 * n1 + 1];
        v[4] = -cmv * L[n1 * n1 + 2];
        v[6] = ctab<double>(2 * TRI_MAX + tri(n1, 0)) * L[n1 * n1];
      } else {
        const double ur = L[n1 * n1 + 2 * (m + 1) - 1], ui = L[n1 * n1 + 2 * (m + 1)];
        double dr, di;
        if (m == 1) { dr = L[n1 * n1]; di = 0; }
        else { dr = L[n1 * n1 + 2 * (m - 1) - 1]; di = L[n1 * n1 + 2 * (m - 1)]; }
        const double cu = 0.5 * ctab<double>(3 * TRI_MAX + tri(n1, m + 1));
        const double cd = 0.5 * ctab<double>(4 * TRI_MAX + tri(n1, m - 1));
        const double czv = ctab<double>(2 * TRI_MAX + tri(n1, m));
        v[2] = 2 * (-cu * ur + cd * dr); v[3] = 2 * (-cu * ui + cd * di);
        v[4] = -2 * (cu * ui + cd * di); v[5] = 2 * (cu * ur + cd * dr);
        v[6] = 2 * czv * L[n1 * n1 + 2 * m - 1]; v[7] = 2 * czv * L[n1 * n1 + 2 * m];
      }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) E[8 * q + i] = (R)v[i];
  }
}

template <typename R> struct alignas(4 * sizeof(R)) Quad { R a, b, c, d; };

// L2P at x̂ from the prepared entries (potential and the gradient before the 1/w factor)
template <int P, typename R>
__device__ __forceinline__ void l2p_prepared(const R* __restrict__ E, R x, R y, R z, R& u, R& gx, R& gy, R& gz) {
  const R r2 = x * x + y * y + z * z;
  R sr = 1, si = 0;
  u = 0; gx = 0; gy = 0; gz = 0;
#pragma unroll 1
  for (int m = 0; m <= P; ++m) {
    R pr = 0, pi = 0, cr = sr, ci = si;
    const Quad<R>* Em = reinterpret_cast<const Quad<R>*>(E + 8 * l2p_entry(P, m, m));
#pragma unroll 2
    for (int n = m; n <= P; ++n) {
      R vr, vi;
      if (n == m) { vr = sr; vi = si; }
      else {
        const int t = tri(n, m);
        const R az = ctab<R>(t) * z, br = ctab<R>(TRI_MAX + t) * r2;
        vr = az * cr - br * pr; vi = az * ci - br * pi;
        pr = cr; pi = ci; cr = vr; ci = vi;
      }
      const Quad<R> a = Em[2 * (n - m)], b = Em[2 * (n - m) + 1];
      u += a.a * vr + a.b * vi;
      gx += a.c * vr + a.d * vi;
      gy += b.a * vr + b.b * vi;
      gz += b.c * vr + b.d * vi;
    }
    if (m < P) {
      const R e = ce<R>(m);
      const R nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      sr = nr; si = ni;
    }
  }
}

// per-warp shared memory of k_l2p: the prepared entries, or (Yukawa3D) the local itself
template <int P, typename R, bool YK>
size_t l2p_warp_bytes(int LD) { return YK ? sizeof(R) * LD : sizeof(R) * 8 * l2p_entries<P>(); }

// YK: Yukawa3D's weighted L2P (FP64), κ̂² = kh2[level]
template <int P, typename R, bool YK>
__global__ void __launch_bounds__(256) k_l2p(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                             const int* __restrict__ gcount, int ngroups, const double* __restrict__ tx,
                                             const double* __restrict__ ty, const double* __restrict__ tz,
                                             const int* __restrict__ tout, const int4* __restrict__ cell,
                                             const double* __restrict__ Pl, int LD, Geometry geo,
                                             const double* __restrict__ scale, int outputs, double* __restrict__ pot,
                                             double* __restrict__ grad, const double* __restrict__ kh2, int acc) {
  extern __shared__ __align__(16) unsigned char sl_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * (blockDim.x >> 5) + warp;
  if (grp >= ngroups) return;
  const int leaf = gnode[grp];
  R* L = reinterpret_cast<R*>(sl_raw) + warp * (YK ? LD : 8 * l2p_entries<P>());
  if constexpr (YK) {
    for (int i = lane; i < LD; i += 32) L[i] = (R)Pl[(int64_t)leaf * LD + i];
  } else {
    l2p_prepare<P, R>(Pl + (int64_t)leaf * LD, L, lane);
  }
  __syncwarp();
  const int4 c = cell[leaf];
  const Geometry gn = geo.at(leaf);
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : cx, y = act ? ty[k] : cy, z = act ? tz[k] : cz;
    R u, gx, gy, gz;
    if constexpr (YK) l2p_yukawa<P>(L, kh2[c.w], (x - cx) * s, (y - cy) * s, (z - cz) * s, u, gx, gy, gz);
    else l2p_prepared<P, R>(L, (R)((x - cx) * s), (R)((y - cy) * s), (R)((z - cz) * s), u, gx, gy, gz);
    if (act) {
      const int o = tout[k];
      // acc: the near field is already in the outputs (x + y = y + x: the same sums either way)
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = (acc ? pot[o] : 0.0) + (double)u;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        const int64_t o3 = 3 * (int64_t)o;
        grad[o3] = (acc ? grad[o3] : 0.0) + (double)gx * s;
        grad[o3 + 1] = (acc ? grad[o3 + 1] : 0.0) + (double)gy * s;
        grad[o3 + 2] = (acc ? grad[o3 + 2] : 0.0) + (double)gz * s;
      }
    }
  }
}

// one staged source: aligned so that it is read with one 16-byte (FP32) or two 16-byte (FP64)
// shared-memory loads
template <typename R>
struct alignas(4 * sizeof(R)) R4 { R x, y, z, w; };

// the hardware reciprocal square root (PTX rsqrt.approx, relative error below 2^-22), with
// subnormal inputs flushed: squared distances of distinct points in leaf-centred coordinates are
// far above FP32's subnormal range, and the self term (r² = 0 → ∞) is masked by index
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <typename R>
struct NearWarp {
  R4<R> stg[2][32];   // double-buffered batch of staged sources
  int lo[32];         // first point of each colleague (27 used)
  int pre[32];        // flat index of each colleague's first point (total for the unused slots)
};

// the sources of batch b (flat indices 32b + lane) from global memory, in FP64
template <typename R>
__device__ __forceinline__ void load_batch(const NearWarp<R>& sw, int b, int lane, int S, const double* __restrict__ xs,
                                           const double* __restrict__ ys, const double* __restrict__ zs,
                                           const double* __restrict__ q, double& x, double& y, double& z, double& w) {
  const int f = 32 * b + lane;
  x = y = z = w = 0.0;
  if (f < S) {
    int idx = 0;   // the last colleague whose flat start is ≤ f
#pragma unroll
    for (int step = 16; step; step >>= 1)
      if (sw.pre[idx + step] <= f) idx += step;
    const int j = sw.lo[idx] + (f - sw.pre[idx]);
    x = xs[j];
    y = ys[j];
    z = zs[j];
    w = q[j];
  }
}

// one batch of m staged sources against this lane's target; CHECK skips flat index `is`.
// YK (FP64): the Yukawa pair e^{−κr}/r and its radial derivative −e^{−κr}(1 + κr)/r²
// (src/kernels.jl:235-242)
// KIND 2 (FP64): the Laplace2D pair c·log r², c = −1/(4π), as KC·(−τ log r²) and gradient
// −KC·(2τ/r²)·d (src/kernels.jl:58-66; the points share z, so r² is the planar distance)
template <typename R, bool CHECK, int YK = 0>
__device__ __forceinline__ void near_batch(const R4<R>* __restrict__ stg, int m, int is, R fx, R fy, R fz, R& bp, R& bx,
                                           R& by, R& bz, double kappa = 0) {
  auto body = [&](int i) {
    const R4<R> sv = stg[i];
    const R dx = fx - sv.x, dy = fy - sv.y, dz = fz - sv.z;
    R r2, ir;
    if constexpr (sizeof(R) == 8) {
      r2 = fma(dz, dz, fma(dy, dy, dx * dx));
      ir = rsqrt(r2);
    } else {
      r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      ir = rsqrt_ftz(r2);
    }
    if (CHECK && i == is) ir = R(0);
    R qir, qir3;
    if constexpr (YK == 2) {
      const bool self = CHECK && i == is;
      qir = self ? R(0) : -sv.w * log(r2);
      qir3 = self ? R(0) : 2 * sv.w / r2;
    } else if constexpr (YK == 1) {
      const double r = r2 * ir, e = exp(-kappa * r);
      qir = sv.w * e * ir;
      qir3 = qir * (1 + kappa * r) * ir * ir;
    } else {
      qir = sv.w * ir;
      qir3 = qir * ir * ir;
    }
    bp += qir;
    bx = fma(qir3, dx, bx);
    by = fma(qir3, dy, by);
    bz = fma(qir3, dz, bz);
  };
  if (m == 32) {
#pragma unroll 8
    for (int i = 0; i < 32; ++i) body(i);
  } else {
#pragma unroll 4
    for (int i = 0; i < m; ++i) body(i);
  }
}

// packed FP32 pairs (the f32x2 instructions of sm_100: two lanes of arithmetic per instruction)
__device__ __forceinline__ uint64_t pk2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(uint64_t v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// The FP32 batch with two sources per instruction: the batch staged as 16 source pairs
// {x₀ x₁ y₀ y₁}{z₀ z₁ w₀ w₁}; each pair's arithmetic in packed f32x2 (the same operations and
// per-element rounding as near_batch), the two running sums of every quantity added at the end;
// an odd last source takes the scalar body. CHECK skips flat index `is`.
template <bool CHECK>
__device__ __forceinline__ void near_batch_f32x2(const float4* __restrict__ pr, int m, int is, float fx, float fy,
                                                 float fz, float& bp, float& bx, float& by, float& bz) {
  const uint64_t fx2 = pk2(fx, fx), fy2 = pk2(fy, fy), fz2 = pk2(fz, fz);
  uint64_t p2 = pk2(0.f, 0.f), x2 = p2, y2 = p2, z2 = p2;
  const int np = m >> 1;
  auto body = [&](int k) {
    const float4 a = pr[2 * k], b = pr[2 * k + 1];
    const uint64_t dx = sub2(fx2, pk2(a.x, a.y)), dy = sub2(fy2, pk2(a.z, a.w)), dz = sub2(fz2, pk2(b.x, b.y));
    const uint64_t r2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
    float ra, rb;
    upk2(r2, ra, rb);
    float ia = rsqrt_ftz(ra), ib = rsqrt_ftz(rb);
    if (CHECK && 2 * k == is) ia = 0.f;
    if (CHECK && 2 * k + 1 == is) ib = 0.f;
    const uint64_t ir = pk2(ia, ib);
    const uint64_t qir = mul2(pk2(b.z, b.w), ir);
    const uint64_t qir3 = mul2(mul2(qir, ir), ir);
    p2 = add2(p2, qir);
    x2 = fma2(qir3, dx, x2);
    y2 = fma2(qir3, dy, y2);
    z2 = fma2(qir3, dz, z2);
  };
  if (np == 16) {
#pragma unroll 8
    for (int k = 0; k < 16; ++k) body(k);
  } else {
#pragma unroll 2
    for (int k = 0; k < np; ++k) body(k);
  }
  float a0, a1;
  upk2(p2, a0, a1); bp += a0 + a1;
  upk2(x2, a0, a1); bx += a0 + a1;
  upk2(y2, a0, a1); by += a0 + a1;
  upk2(z2, a0, a1); bz += a0 + a1;
  if (m & 1) {                                   // the odd last source
    const float* f = reinterpret_cast<const float*>(pr + 2 * np);
    const float dx = fx - f[0], dy = fy - f[2], dz = fz - f[4];
    float ir = rsqrt_ftz(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
    if (CHECK && m - 1 == is) ir = 0.f;
    const float qir = f[6] * ir, qir3 = qir * ir * ir;
    bp += qir;
    bx = fmaf(qir3, dx, bx);
    by = fmaf(qir3, dy, by);
    bz = fmaf(qir3, dz, bz);
  }
}

// W warps (leaf groups) per CTA: 4 or 8, chosen per state by the tuner (tune.cu)
template <typename R, bool SELF, int YK, int W>
__global__ void __launch_bounds__(W * 32, W == 4 ? 5 : 2) k_near(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                         const int* __restrict__ gcount, int ngroups,
                                                         const double* __restrict__ tx, const double* __restrict__ ty,
                                                         const double* __restrict__ tz, const int* __restrict__ tout,
                                                         const double* __restrict__ xs, const double* __restrict__ ys,
                                                         const double* __restrict__ zs, const double* __restrict__ q,
                                                         const int4* __restrict__ cell, const int* __restrict__ plo,
                                                         const int* __restrict__ phi, const int* __restrict__ col,
                                                         Geometry geo, int outputs, double* __restrict__ pot,
                                                         double* __restrict__ grad, double kappa, int first) {
  constexpr bool REL = sizeof(R) == 4;   // the mixed path works relative to the leaf's centre
  __shared__ NearWarp<R> sws[W];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * W + warp;
  if (grp >= ngroups) return;                      // the whole warp
  NearWarp<R>& sw = sws[warp];
  const int leaf = gnode[grp];
  double cx = 0, cy = 0, cz = 0;
  if (REL) {
    const int4 c = cell[leaf];
    const Geometry gn = geo.at(leaf);
    const double w = ldexp(geo.W0, -c.w);
    cx = gn.center(0, c.x, w);
    cy = gn.center(1, c.y, w);
    cz = gn.center(2, c.z, w);
  }
  // the colleagues' point ranges, flattened in colleague order
  const int cn = lane < NCOL ? col[(int64_t)leaf * NCOL + lane] : -1;
  int lo = 0, len = 0;
  if (cn >= 0) {
    lo = plo[cn];
    len = max(0, phi[cn] - lo + 1);
  }
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int S = __shfl_sync(0xffffffffu, incl, 31);
  sw.lo[lane] = lo;
  sw.pre[lane] = incl - len;
  // the leaf's own slot: its points are the self terms
  const unsigned selfm = __ballot_sync(0xffffffffu, cn == leaf);
  const int slot = selfm ? __ffs(selfm) - 1 : 0;
  const int pself = selfm ? __shfl_sync(0xffffffffu, incl - len, slot) : -1;
  const int loself = __shfl_sync(0xffffffffu, lo, slot), lenself = selfm ? __shfl_sync(0xffffffffu, len, slot) : 0;
  __syncwarp();
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : cx, y = act ? ty[k] : cy, z = act ? tz[k] : cz;
    const R fx = (R)(x - cx), fy = (R)(y - cy), fz = (R)(z - cz);
    const int fself = SELF && act && selfm ? pself + (k - loself) : -1;
    double np = 0, nx = 0, ny = 0, nz = 0;
    double sx, sy, sz, sq;
    load_batch(sw, 0, lane, S, xs, ys, zs, q, sx, sy, sz, sq);
    for (int b = 0; 32 * b < S; ++b) {
      R4<R>* stg = sw.stg[b & 1];
      if constexpr (sizeof(R) == 4) {
        // the FP32 path stages source pairs: lane l into pair l/2, slot l%2
        float* f = reinterpret_cast<float*>(stg) + 8 * (lane >> 1) + (lane & 1);
        f[0] = (float)(sx - cx);
        f[2] = (float)(sy - cy);
        f[4] = (float)(sz - cz);
        f[6] = (float)sq;
      } else {
        stg[lane] = R4<R>{(R)(sx - cx), (R)(sy - cy), (R)(sz - cz), (R)sq};
      }
      __syncwarp();
      if (32 * (b + 1) < S) load_batch(sw, b + 1, lane, S, xs, ys, zs, q, sx, sy, sz, sq);
      const int m = min(32, S - 32 * b);
      const bool chk = SELF && selfm && 32 * b < pself + lenself && 32 * b + 32 > pself;   // uniform
      if constexpr (sizeof(R) == 8) {
        // the plain path sums straight into the FP64 totals, in the reference's order
        if (chk) near_batch<R, true, YK>(stg, m, fself - 32 * b, fx, fy, fz, np, nx, ny, nz, kappa);
        else near_batch<R, false, YK>(stg, m, 0, fx, fy, fz, np, nx, ny, nz, kappa);
      } else {
        float bp = 0, bx = 0, by = 0, bz = 0;
        const float4* pr = reinterpret_cast<const float4*>(stg);
        if (chk) near_batch_f32x2<true>(pr, m, fself - 32 * b, fx, fy, fz, bp, bx, by, bz);
        else near_batch_f32x2<false>(pr, m, 0, fx, fy, fz, bp, bx, by, bz);
        np += bp;
        nx += bx;
        ny += by;
        nz += bz;
      }
    }
    if (act) {
      const int o = tout[k];
      // first: the far field comes after (and adds to) these
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = (first ? 0.0 : pot[o]) + KC * np;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        const int64_t o3 = 3 * (int64_t)o;
        grad[o3] = (first ? 0.0 : grad[o3]) - KC * nx;
        grad[o3 + 1] = (first ? 0.0 : grad[o3 + 1]) - KC * ny;
        grad[o3 + 2] = (first ? 0.0 : grad[o3 + 2]) - KC * nz;
      }
    }
    __syncwarp();   // the staging buffers are reused by the next group of targets
  }
}

// The kernel-independent far field (l2t, src/operators/ki_common.jl:293-327): at each target
// Σ_k G(x − y_k) L_k over the leaf's large surface y_k = c + w·ŷ_k (ŷ at width 1), times w (the
// pseudo-inverse's scale). A warp per leaf, lanes over the surface points (a lane takes every
// 32nd): each lane reads its points and densities once per batch of up to TB targets held in
// registers, then the batch's sums are reduced across the lanes in FP64. (Leaves of the adaptive
// configurations hold a few points each, so lanes over the targets would mostly idle.)
// R = float: leaf-centred FP32 terms, each lane's partial sums in FP32, the reduction in FP64;
// R = double: FP64 throughout. Writes the outputs (the near field adds to them).
template <typename R, int TB>
__device__ __forceinline__ void ki_l2t_batch(int k0, int nb, const double* __restrict__ tx, const double* __restrict__ ty,
                                             const double* __restrict__ tz, const int* __restrict__ tout,
                                             const double* __restrict__ L, const double* __restrict__ large, int nl,
                                             double w, double cx, double cy, double cz, int lane, int outputs,
                                             double* __restrict__ pot, double* __restrict__ grad) {
  R px[TB], py[TB], pz[TB], au[TB], ax[TB], ay[TB], az[TB];
#pragma unroll
  for (int i = 0; i < TB; ++i) {
    const int k = k0 + (i < nb ? i : 0);             // slots past the batch repeat its first target
    px[i] = (R)(tx[k] - cx); py[i] = (R)(ty[k] - cy); pz[i] = (R)(tz[k] - cz);
    au[i] = 0; ax[i] = 0; ay[i] = 0; az[i] = 0;
  }
  for (int q = lane; q < nl; q += 32) {
    const R yx = (R)(w * large[3 * q]), yy = (R)(w * large[3 * q + 1]), yz = (R)(w * large[3 * q + 2]);
    const R l = (R)L[q];
#pragma unroll
    for (int i = 0; i < TB; ++i) {
      const R dx = px[i] - yx, dy = py[i] - yy, dz = pz[i] - yz;
      const R ir = rsqrt(dx * dx + dy * dy + dz * dz);
      const R li = l * ir;
      au[i] += li;
      const R li3 = li * ir * ir;
      ax[i] += li3 * dx;
      ay[i] += li3 * dy;
      az[i] += li3 * dz;
    }
  }
#pragma unroll
  for (int i = 0; i < TB; ++i) {
    double u = au[i], gx = ax[i], gy = ay[i], gz = az[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      u += __shfl_xor_sync(0xffffffffu, u, o);
      gx += __shfl_xor_sync(0xffffffffu, gx, o);
      gy += __shfl_xor_sync(0xffffffffu, gy, o);
      gz += __shfl_xor_sync(0xffffffffu, gz, o);
    }
    if (lane == i && i < nb) {
      const int t = tout[k0 + i];
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[t] = KC * w * u;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        grad[3 * (int64_t)t] = -KC * w * gx;
        grad[3 * (int64_t)t + 1] = -KC * w * gy;
        grad[3 * (int64_t)t + 2] = -KC * w * gz;
      }
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(128) k_ki_l2t(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                const int* __restrict__ gcount, int ngroups, const double* __restrict__ tx,
                                                const double* __restrict__ ty, const double* __restrict__ tz,
                                                const int* __restrict__ tout, const int4* __restrict__ cell,
                                                const double* __restrict__ Ll, int nl, int nld,
                                                const double* __restrict__ large, Geometry geo, int outputs,
                                                double* __restrict__ pot, double* __restrict__ grad) {
  constexpr int TB = sizeof(R) == 4 ? 8 : 4;         // targets per batch
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * (blockDim.x >> 5) + warp;
  if (grp >= ngroups) return;
  const int leaf = gnode[grp];
  const int4 c = cell[leaf];
  const Geometry gn = geo.at(leaf);
  const double w = ldexp(geo.W0, -c.w);
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  const double* L = Ll + (int64_t)leaf * nld;
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int b = 0; b < nt; b += TB) {
    const int nb = min(TB, nt - b);                  // uniform across the warp
    if (nb > TB / 2)
      ki_l2t_batch<R, TB>(t0 + b, nb, tx, ty, tz, tout, L, large, nl, w, cx, cy, cz, lane, outputs, pot, grad);
    else if (nb > TB / 4)
      ki_l2t_batch<R, TB / 2>(t0 + b, nb, tx, ty, tz, tout, L, large, nl, w, cx, cy, cz, lane, outputs, pot, grad);
    else
      ki_l2t_batch<R, TB / 4>(t0 + b, nb, tx, ty, tz, tout, L, large, nl, w, cx, cy, cz, lane, outputs, pot, grad);
  }
}

// The circle method's far field (l2t over the large circle, src/operators/ki_common.jl:293-327):
// Σ_k c·log|x − y_k|² L_k and its gradient Σ_k 2c (x − y_k)/|x − y_k|² L_k, y_k on the leaf's
// circle of radius (4 − √2)/2·w, FP64; writes the outputs (the near field adds to them)
__global__ void __launch_bounds__(128) k_kic_l2t(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                 const int* __restrict__ gcount, int ngroups, const double* __restrict__ tx,
                                                 const double* __restrict__ ty, const int* __restrict__ tout,
                                                 const int4* __restrict__ cell, const double* __restrict__ Ll, int N,
                                                 Geometry geo, int outputs, double* __restrict__ pot,
                                                 double* __restrict__ grad) {
  __shared__ double sL[4][64], sx[4][64], sy[4][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * 4 + warp;
  if (grp >= ngroups) return;
  const int leaf = gnode[grp];
  const int4 c = cell[leaf];
  const Geometry gn = geo.at(leaf);
  const double w = ldexp(geo.W0, -c.w);
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w);
  for (int k = lane; k < N; k += 32) {
    double sn, cs;
    sincospi(2.0 * k / N, &sn, &cs);
    sL[warp][k] = Ll[(int64_t)leaf * 64 + k];
    sx[warp][k] = cx + KIC_LARGE * w * cs;
    sy[warp][k] = cy + KIC_LARGE * w * sn;
  }
  __syncwarp();
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : cx, y = act ? ty[k] : cy;
    double u = 0, gx = 0, gy = 0;
    for (int q = 0; q < N; ++q) {
      const double dx = x - sx[warp][q], dy = y - sy[warp][q];
      const double r2 = fma(dy, dy, dx * dx);
      u = fma(sL[warp][q], log(r2), u);
      const double g = sL[warp][q] / r2;
      gx = fma(g, dx, gx);
      gy = fma(g, dy, gy);
    }
    if (act) {
      const int o = tout[k];
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = -KC * u;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        grad[3 * (int64_t)o] = -2 * KC * gx;
        grad[3 * (int64_t)o + 1] = -2 * KC * gy;
        grad[3 * (int64_t)o + 2] = 0.0;
      }
    }
  }
}

// The near field of charges and dipoles (source_field / target_field of src/sources.jl:137-155 with
// Laplace3D): per source q/r + (d·v)/r³ and the gradient −q v/r³ + d/r³ − 3 v (d·v)/r⁵, v = t − s,
// as KC times the sums below (pot += KC·Σ, grad −= KC·Σ). Same flattening of the colleagues'
// ranges as k_near, one batch of 32 staged sources (positions and moments) at a time; R as there
// (FP32 relative to the leaf's centre with FP64 batch sums, or FP64).
template <typename R, bool SELF>
__global__ void __launch_bounds__(NEAR_WARPS * 32) k_near_dip(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                             const int* __restrict__ gcount, int ngroups,
                                                             const double* __restrict__ tx, const double* __restrict__ ty,
                                                             const double* __restrict__ tz, const int* __restrict__ tout,
                                                             const double* __restrict__ xs, const double* __restrict__ ys,
                                                             const double* __restrict__ zs, const double* __restrict__ q,
                                                             const double* __restrict__ d3, int64_t npts,
                                                             const int4* __restrict__ cell, const int* __restrict__ plo,
                                                             const int* __restrict__ phi, const int* __restrict__ col,
                                                             Geometry geo, int outputs, double* __restrict__ pot,
                                                             double* __restrict__ grad) {
  constexpr bool REL = sizeof(R) == 4;
  __shared__ R4<R> sp[NEAR_WARPS][32], sd[NEAR_WARPS][32];
  __shared__ int slo[NEAR_WARPS][32], spre[NEAR_WARPS][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * NEAR_WARPS + warp;
  if (grp >= ngroups) return;
  const int leaf = gnode[grp];
  double cx = 0, cy = 0, cz = 0;
  if (REL) {
    const int4 c = cell[leaf];
    const Geometry gn = geo.at(leaf);
    const double w = ldexp(geo.W0, -c.w);
    cx = gn.center(0, c.x, w);
    cy = gn.center(1, c.y, w);
    cz = gn.center(2, c.z, w);
  }
  const int cn = lane < NCOL ? col[(int64_t)leaf * NCOL + lane] : -1;
  int lo = 0, len = 0;
  if (cn >= 0) {
    lo = plo[cn];
    len = max(0, phi[cn] - lo + 1);
  }
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int S = __shfl_sync(0xffffffffu, incl, 31);
  slo[warp][lane] = lo;
  spre[warp][lane] = incl - len;
  __syncwarp();
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : cx, y = act ? ty[k] : cy, z = act ? tz[k] : cz;
    const R fx = (R)(x - cx), fy = (R)(y - cy), fz = (R)(z - cz);
    double np = 0, nx = 0, ny = 0, nz = 0;
    for (int b = 0; 32 * b < S; ++b) {
      const int f = 32 * b + lane;
      int src = -1;
      if (f < S) {
        int idx = 0;
#pragma unroll
        for (int step = 16; step; step >>= 1)
          if (spre[warp][idx + step] <= f) idx += step;
        src = slo[warp][idx] + (f - spre[warp][idx]);
      }
      __syncwarp();
      if (src >= 0) {
        sp[warp][lane] = R4<R>{(R)(xs[src] - cx), (R)(ys[src] - cy), (R)(zs[src] - cz), (R)q[src]};
        sd[warp][lane] = R4<R>{(R)d3[src], (R)d3[npts + src], (R)d3[2 * npts + src], (R)0};
      }
      // the source index of each staged slot, for the self check
      const int sidx = src;
      __syncwarp();
      const int m = min(32, S - 32 * b);
      R bp = 0, bx = 0, by = 0, bz = 0;
      for (int i = 0; i < m; ++i) {
        const R4<R> sv = sp[warp][i], dv = sd[warp][i];
        const int si = __shfl_sync(0xffffffffu, sidx, i);
        const R vx = fx - sv.x, vy = fy - sv.y, vz = fz - sv.z;
        const R r2 = vx * vx + vy * vy + vz * vz;
        R ir = r2 > R(0) ? R(1) / sqrt(r2) : R(0);
        if (SELF && act && si == k) ir = R(0);     // the target's own source: k is its tree index
        const R ir2 = ir * ir, ir3 = ir2 * ir;
        const R dd = dv.x * vx + dv.y * vy + dv.z * vz;
        bp += sv.w * ir + dd * ir3;
        const R cv = sv.w * ir3 + 3 * dd * ir3 * ir2;
        bx += cv * vx - dv.x * ir3;
        by += cv * vy - dv.y * ir3;
        bz += cv * vz - dv.z * ir3;
      }
      np += bp; nx += bx; ny += by; nz += bz;
    }
    if (act) {
      const int o = tout[k];
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = pot[o] + KC * np;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        grad[3 * (int64_t)o] = grad[3 * (int64_t)o] - KC * nx;
        grad[3 * (int64_t)o + 1] = grad[3 * (int64_t)o + 1] - KC * ny;
        grad[3 * (int64_t)o + 2] = grad[3 * (int64_t)o + 2] - KC * nz;
      }
    }
    __syncwarp();
  }
}

template <int P>
void launch_l2p(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx, const double* ty,
                const double* tz, const int* tout, int outputs, double* pot, double* grad, int acc = 0) {
  Plan& P_ = *S.plan;
  // the mixed path evaluates Laplace3D in FP32; Yukawa3D keeps its radial weights in FP64 (its
  // mixed path is the tensor-core M2L only)
  const bool yk = P_.cache->kernel == FMMB_KERNEL_YUKAWA3D;
  const bool mixed = S.precision == FMMB_PRECISION_MIXED && !yk;
  const size_t per_warp = mixed ? l2p_warp_bytes<P, float, false>(P_.cache->ld)
                                : (yk ? l2p_warp_bytes<P, double, true>(P_.cache->ld) : l2p_warp_bytes<P, double, false>(P_.cache->ld));
  const int warps = per_warp > 8192 ? 4 : 8;
  const size_t smem = per_warp * warps;
  auto kern = mixed ? k_l2p<P, float, false> : (yk ? k_l2p<P, double, true> : k_l2p<P, double, false>);
  FMMB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(ng + warps - 1) / warps, 32 * warps, smem, P_.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, P_.cell.p,
                                                                      S.Pl.p, P_.cache->ld, geometry(P_), P_.d_scale.p,
                                                                      outputs, pot, grad, P_.d_kh2.p, acc);
  FMMB_LAUNCH_CHECK();
}

template <typename R, bool SELF, int YK = 0>
void launch_near(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx, const double* ty,
                 const double* tz, const int* tout, int outputs, double* pot, double* grad, int first = 0,
                 cudaStream_t st = nullptr) {
  Plan& P_ = *S.plan;
  const cudaStream_t s = st ? st : P_.ctx->stream;
  if (S.near_warps == 8)
    k_near<R, SELF, YK, 8><<<(ng + 7) / 8, 32 * 8, 0, s>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, S.xs.p, S.ys.p, S.zs.p,
                                                          S.q.p, P_.cell.p, P_.plo.p, P_.phi.p, P_.col.p, geometry(P_),
                                                          outputs, pot, grad, P_.cache->kappa, first);
  else
    k_near<R, SELF, YK, 4><<<(ng + 3) / 4, 32 * 4, 0, s>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, S.xs.p, S.ys.p, S.zs.p,
                                                          S.q.p, P_.cell.p, P_.plo.p, P_.phi.p, P_.col.p, geometry(P_),
                                                          outputs, pot, grad, P_.cache->kappa, first);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

void evaluate_groups(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx,
                     const double* ty, const double* tz, const int* tout, bool self, int outputs, double* pot, double* grad) {
  if (ng == 0) return;
  if (S.plan->cache->method == FMMB_METHOD_KI_CIRCLE) {
    Plan& P_ = *S.plan;
    k_kic_l2t<<<(ng + 3) / 4, 128, 0, P_.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tout, P_.cell.p, S.ki_ll.p,
                                                        P_.cache->np, geometry(P_), outputs, pot, grad);
    FMMB_LAUNCH_CHECK();
    if (self) launch_near<double, true, 2>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    else launch_near<double, false, 2>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    return;
  }
  if (S.plan->cache->method == FMMB_METHOD_CUBE_KI) {
    Plan& P_ = *S.plan;
    Cache& C = *P_.cache;
    const bool mixed = S.precision == FMMB_PRECISION_MIXED;
    const int warps = 4;
    auto kern = mixed ? k_ki_l2t<float> : k_ki_l2t<double>;
    kern<<<(ng + warps - 1) / warps, 32 * warps, 0, P_.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout,
                                                                       P_.cell.p, S.ki_ll.p, C.ki_nl, C.ki_nld,
                                                                       C.ki_large.p, geometry(P_), outputs, pot, grad);
    FMMB_LAUNCH_CHECK();
    if (mixed && self) launch_near<float, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    else if (mixed) launch_near<float, false>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    else if (self) launch_near<double, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    else launch_near<double, false>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    return;
  }
  switch (S.plan->cache->p) {
#define X(pp) case pp: launch_l2p<pp>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad); break;
    FMMB_P_CASES(X)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "p out of range");
  }
  const bool mixed = S.precision == FMMB_PRECISION_MIXED;
  if (S.has_dip) {
    Plan& P_ = *S.plan;
    const unsigned nb = (ng + NEAR_WARPS - 1) / NEAR_WARPS;
#define FMMB_NEAR_DIP(R, SELF)                                                                                  \
  k_near_dip<R, SELF><<<nb, 32 * NEAR_WARPS, 0, P_.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, S.xs.p, \
                                                                  S.ys.p, S.zs.p, S.q.p, S.dip.p, P_.N, P_.cell.p,     \
                                                                  P_.plo.p, P_.phi.p, P_.col.p, geometry(P_), outputs, \
                                                                  pot, grad)
    if (mixed && self) FMMB_NEAR_DIP(float, true);
    else if (mixed) FMMB_NEAR_DIP(float, false);
    else if (self) FMMB_NEAR_DIP(double, true);
    else FMMB_NEAR_DIP(double, false);
#undef FMMB_NEAR_DIP
    FMMB_LAUNCH_CHECK();
    return;
  }
  if (S.plan->cache->kernel == FMMB_KERNEL_YUKAWA3D) {   // the near field in FP64 on both paths
    if (self) launch_near<double, true, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    else launch_near<double, false, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
    return;
  }
  if (mixed && self) launch_near<float, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
  else if (mixed) launch_near<float, false>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
  else if (self) launch_near<double, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
  else launch_near<double, false>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);
}

// the harmonic method's evaluation at the sources in two halves: the near field on stream st
// (writing the outputs) and, after it, the far field (adding to them); charges only
bool split_evaluation(const State& S) {
  const Cache& C = *S.plan->cache;
  return C.method == FMMB_METHOD_SPHERICAL_HARMONICS && !S.has_dip &&
         (C.kernel == FMMB_KERNEL_LAPLACE3D || C.kernel == FMMB_KERNEL_YUKAWA3D);
}

void near_sources(State& S, int outputs, double* pot, double* grad, cudaStream_t st) {
  Plan& P = *S.plan;
  if (P.n_leaves == 0) return;
  const bool mixed = S.precision == FMMB_PRECISION_MIXED;
  const double *tx = S.xs.p, *ty = S.ys.p, *tz = S.zs.p;
  if (P.cache->kernel == FMMB_KERNEL_YUKAWA3D)
    launch_near<double, true, 1>(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, tx, ty, tz, P.perm.p, outputs,
                                 pot, grad, 1, st);
  else if (mixed)
    launch_near<float, true>(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, tx, ty, tz, P.perm.p, outputs, pot,
                             grad, 1, st);
  else
    launch_near<double, true>(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, tx, ty, tz, P.perm.p, outputs, pot,
                              grad, 1, st);
}

void far_sources(State& S, int outputs, double* pot, double* grad) {
  Plan& P = *S.plan;
  if (P.n_leaves == 0) return;
  switch (P.cache->p) {
#define X(pp)                                                                                                    \
  case pp:                                                                                                       \
    launch_l2p<pp>(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, S.xs.p, S.ys.p, S.zs.p, P.perm.p, outputs, \
                   pot, grad, 1);                                                                                \
    break;
    FMMB_P_CASES(X)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "p out of range");
  }
}

}  // namespace fmmb
