// SphericalHarmonics(Yukawa3D(κ)): the kernel e^{−κr}/(4πr) on the harmonic basis
// (src/operators/harmonics_yukawa.jl). With the modified spherical Bessel functions normalised
// to the Laplace limit,
//   u_n(z) = (2n+1)!! i_n(z)/z^n,   v_n(z) = (2/π) z^{n+1} k_n(z)/(2n−1)!!,
// e^{−κ|x−y|}/|x−y| = Σ_n u_n(κ r_<) v_n(κ r_>) Σ_m S̃_n^m(x̂) conj S̃_n^m(ŷ), so the multipoles and
// locals are the Laplace folds weighted per degree by u_n(κ̂|x̂|) (κ̂ = κ·w in box coordinates),
// and the symmetry classes still hold. The translations couple all degrees, so M2M, L2L and the
// 34 class representatives are built per box width by projection on a sphere, where the real
// surface harmonics are orthogonal: a Gauss–Legendre × trapezoid rule of (2p+10) × (4p+20)
// points (harmonics_yukawa.jl:94-110).
//
// The reference builds those operators on the host per width. Here the quadrature rule is
// computed on the host and everything else on the device in FP64: the basis of each translated
// sphere (one thread per quadrature point) and the projections, which are GEMMs of
// (p+1)² × (2p+10)(4p+20) by (2p+10)(4p+20) × (p+1)² on the FP64 tensor cores (the same DMMA
// GEMM as M2M and L2L). Each width's operators are built once, when a plan first needs that
// width, and kept in a process-wide store shared by the operator caches of the same device,
// order and κ.
#include <cmath>
#include <map>
#include <tuple>

#include "passes.cuh"

namespace fmmb {

void gemm_columns(int M, int K, const double* A, ColMap bm, ColMap cm, int ncols, int LD, int NP, int accumulate,
                  int num_sms, cudaStream_t s);

namespace {

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// u_n(z), n = 0..nmax, from z²: Miller's backward recurrence u_n = u_{n+1} + z² u_{n+2}/((2n+3)(2n+5))
// started above max(nmax, z), normalised with u_0 = sinh z / z; the series' first two terms for
// z² < 1e-8 (harmonics_yukawa.jl:41-59)
__device__ void yk_u(double z2, int nmax, double* u) {
  if (z2 < 1e-8) {
    for (int n = 0; n <= nmax; ++n) u[n] = 1 + z2 / (2 * (2 * n + 3));
    return;
  }
  const double z = sqrt(z2);
  const int N = max(nmax, (int)ceil(z)) + 25;
  double a = 0, b = 1;
  for (int n = N - 1; n >= 0; --n) {
    const double c = b + z2 * a / (double)((2 * n + 3) * (2 * n + 5));
    if (n <= nmax) u[n] = c;
    a = b;
    b = c;
  }
  const double s = (sinh(z) / z) / b;
  for (int n = 0; n <= nmax; ++n) u[n] *= s;
}

// v_n(z), n = 0..nmax: v_0 = e^{−z}, v_1 = e^{−z}(1 + z), v_{n+1} = v_n + z² v_{n−1}/((2n−1)(2n+1))
// (harmonics_yukawa.jl:61-73)
__device__ void yk_v(double z, int nmax, double* v) {
  const double e = exp(-z), z2 = z * z;
  v[0] = e;
  if (nmax >= 1) v[1] = e * (1 + z);
  for (int n = 1; n < nmax; ++n) v[n + 1] = v[n] + z2 * v[n - 1] / (double)((2 * n - 1) * (2 * n + 1));
}

// Re, Im Υ̃_n^m(x) for 0 ≤ m ≤ n ≤ p at triangular index tri(n, m): the Schmidt recurrences of
// the P2M and L2P folds (harmonics.jl:682-700)
__device__ void fold_all(double x, double y, double z, int p, double* vr, double* vi) {
  const double r2 = x * x + y * y + z * z;
  double sr = 1, si = 0;
  for (int m = 0; m <= p; ++m) {
    if (m > 0) {
      const double e = c_e[m - 1];
      const double nr = -e * (x * sr - y * si), ni = -e * (x * si + y * sr);
      sr = nr;
      si = ni;
    }
    vr[tri(m, m)] = sr;
    vi[tri(m, m)] = si;
    double pr = 0, pi = 0, cr = sr, ci = si;
    for (int n = m + 1; n <= p; ++n) {
      const int t = tri(n, m);
      const double az = c_tab[t] * z, br = c_tab[TRI_MAX + t] * r2;
      const double nr = az * cr - br * pr, ni = az * ci - br * pi;
      vr[t] = nr;
      vi[t] = ni;
      pr = cr; pi = ci; cr = nr; ci = ni;
    }
  }
}

// One column set of a projection's right operand: at quadrature point q the real basis of
// expansion coefficient i (rows i < (p+1)², column-major over q: F[i·nq + q]) at
// y = bs·(a·x̂_q + sh), times mult:
//   regular   u_n(κ̂|y|) {Υ̃_n^0, 2 Re Υ̃_n^m, 2 Im Υ̃_n^m}(y)                  (harmonics_yukawa.jl:111-125)
//   irregular v_n(κ̂|y|) |y|^{−(2n+1)} {Υ̃_n^0, 2 Re Υ̃_n^m, −2 Im Υ̃_n^m}(y)    (harmonics_yukawa.jl:126-142)
__global__ void k_yk_basis(int p, int nq, const double* __restrict__ xq, double a, double shx, double shy, double shz,
                           double bs, double kh, int irregular, double mult, double* __restrict__ F) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  double vr[TRI_MAX], vi[TRI_MAX], rad[PMAX + 1];
  const double x = bs * (a * xq[3 * q] + shx), y = bs * (a * xq[3 * q + 1] + shy), z = bs * (a * xq[3 * q + 2] + shz);
  fold_all(x, y, z, p, vr, vi);
  const double r = sqrt(x * x + y * y + z * z);
  if (irregular) {
    yk_v(kh * r, p, rad);
    const double ir = 1 / r;
    double f = ir;                                 // |y|^{−(2n+1)}
    for (int n = 0; n <= p; ++n) {
      rad[n] *= f;
      f *= ir * ir;
    }
  } else {
    yk_u((kh * r) * (kh * r), p, rad);
  }
  const double sim = irregular ? -2.0 : 2.0;
  for (int n = 0; n <= p; ++n) {
    const double w = mult * rad[n];
    F[(int64_t)(n * n) * nq + q] = w * vr[tri(n, 0)];
    for (int m = 1; m <= n; ++m) {
      F[(int64_t)(n * n + 2 * m - 1) * nq + q] = 2 * w * vr[tri(n, m)];
      F[(int64_t)(n * n + 2 * m) * nq + q] = sim * w * vi[tri(n, m)];
    }
  }
}

// The projection onto the regular (or irregular) basis on the sphere of radius ρ, as the left
// operand (LD × nq, column-major; rows ≥ (p+1)² zero): coefficient i = Σ_q Φ(ρ x̂_q) β_i(x̂_q) w_q /
// (γ_i f_n), β = {Υ̃⁰, 2 Re Υ̃, 2 Im Υ̃} on the unit sphere, γ = 4π/(2n+1) (m = 0) or 8π/(2n+1),
// f_n = u_n(κ̂ρ) ρ^n or v_n(κ̂ρ) ρ^{−n−1}, the irregular basis' imaginary rows negated
// (harmonics_yukawa.jl:143-163); times mult
__global__ void k_yk_projection(int p, int LD, int nq, const double* __restrict__ xq, const double* __restrict__ wq,
                                double kh, double rho, int irregular, double mult, double* __restrict__ P) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  double vr[TRI_MAX], vi[TRI_MAX], rad[PMAX + 1];
  fold_all(xq[3 * q], xq[3 * q + 1], xq[3 * q + 2], p, vr, vi);
  if (irregular) yk_v(kh * rho, p, rad);
  else yk_u((kh * rho) * (kh * rho), p, rad);
  double* col = P + (int64_t)q * LD;
  const double wt = mult * wq[q];
  for (int n = 0; n <= p; ++n) {
    const double f = irregular ? rad[n] * pow(rho, -n - 1) : rad[n] * pow(rho, n);
    const double g0 = 4 * M_PI / (2 * n + 1);
    col[n * n] = vr[tri(n, 0)] * wt / (g0 * f);
    for (int m = 1; m <= n; ++m) {
      col[n * n + 2 * m - 1] = 2 * vr[tri(n, m)] * wt / (2 * g0 * f);
      col[n * n + 2 * m] = (irregular ? -1.0 : 1.0) * 2 * vi[tri(n, m)] * wt / (2 * g0 * f);
    }
  }
  for (int i = (p + 1) * (p + 1); i < LD; ++i) col[i] = 0;
}

// the Gauss–Legendre rule on [−1, 1] of n points by Newton's iteration on P_n (the reference
// takes the Golub–Welsch eigenvalues, harmonics_yukawa.jl:89-93: the same rule to rounding)
void gauss_legendre(int n, std::vector<double>& t, std::vector<double>& w) {
  t.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double x = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1, p1 = x;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1);
      const double dx = p1 / dp;
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    double p0 = 1, p1 = x;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = n * (x * p1 - p0) / (x * x - 1);
    t[i] = -x;
    t[n - 1 - i] = x;
    w[i] = w[n - 1 - i] = 2 / ((1 - x * x) * dp * dp);
  }
}

// the product rule on the unit sphere (harmonics_yukawa.jl:94-110), uploaded once per cache
void sphere_rule(Cache& C, cudaStream_t s) {
  if (C.yk_nq) return;
  const int nt = 2 * C.p + 10, nf = 4 * C.p + 20;
  std::vector<double> t, wt;
  gauss_legendre(nt, t, wt);
  std::vector<double> xq, wq;
  for (int i = 0; i < nt; ++i)
    for (int k = 0; k < nf; ++k) {
      const double ph = 2 * M_PI * k / nf, st = std::sqrt(std::max(0.0, 1 - t[i] * t[i]));
      xq.push_back(st * std::cos(ph));
      xq.push_back(st * std::sin(ph));
      xq.push_back(t[i]);
      wq.push_back(wt[i] * 2 * M_PI / nf);
    }
  to_device(C.yk_xq, xq, s);
  to_device(C.yk_wq, wq, s);
  C.yk_nq = nt * nf;
}

// the operators of width w = ldexp(W0, e) (harmonics_yukawa.jl:164-207): projection spheres of
// radius ½ about the target (M2L), 2 about the parent (M2M) and 1 about the child (L2L)
void build_level(Cache& C, int e, YukawaLevel& out, cudaStream_t s) {
  const int p = C.p, N = C.np, LD = C.ld, nq = C.yk_nq, sms = C.ctx->num_sms;
  const double w = std::ldexp(C.W0, e), kh = C.kappa * w, cw = KC / w;
  const double* xq = C.yk_xq.p;
  DBuf<double> Preg((size_t)LD * nq), Pirr((size_t)LD * nq), Pregc((size_t)LD * nq), F((size_t)N * nq);
  k_yk_projection<<<nblk(nq, 128), 128, 0, s>>>(p, LD, nq, xq, C.yk_wq.p, kh, 0.5, 0, cw, Preg.p);
  FMMB_LAUNCH_CHECK();
  k_yk_projection<<<nblk(nq, 128), 128, 0, s>>>(p, LD, nq, xq, C.yk_wq.p, kh, 2.0, 1, 1.0, Pirr.p);
  FMMB_LAUNCH_CHECK();
  k_yk_projection<<<nblk(nq, 128), 128, 0, s>>>(p, LD, nq, xq, C.yk_wq.p, kh / 2, 1.0, 0, 1.0, Pregc.p);
  FMMB_LAUNCH_CHECK();
  out.reps.alloc((size_t)NCLASS * LD * LD);
  out.m2m.alloc((size_t)LD * NCH * LD);
  out.l2l.alloc((size_t)NCH * LD * LD);
  FMMB_CUDA(cudaMemsetAsync(out.reps.p, 0, out.reps.bytes(), s));
  FMMB_CUDA(cudaMemsetAsync(out.m2m.p, 0, out.m2m.bytes(), s));
  FMMB_CUDA(cudaMemsetAsync(out.l2l.p, 0, out.l2l.bytes(), s));
  const ColMap bm{F.p, nullptr, 0, 1, (int64_t)nq};
  // M2L: the source's irregular basis (κ̂) on the target sphere, source centre at the offset o
  for (int c = 0; c < NCLASS; ++c) {
    const int* o = &C.host.reps_off[3 * c];
    k_yk_basis<<<nblk(nq, 128), 128, 0, s>>>(p, nq, xq, 0.5, -(double)o[0], -(double)o[1], -(double)o[2], 1.0, kh, 1, 1.0,
                                             F.p);
    FMMB_LAUNCH_CHECK();
    gemm_columns(LD, nq, Preg.p, bm, ColMap{out.reps.p + (int64_t)c * LD * LD, nullptr, 0, 1, 0}, N, LD, N, 0, sms, s);
  }
  for (int k = 0; k < NCH; ++k) {
    double dh[3];
    for (int d = 0; d < 3; ++d) dh[d] = ((double)((k >> d) & 1) - 0.5) / 2;
    // M2M: the child's irregular basis (κ̂/2, child coordinates 2(x̂ − δ̂)) on the parent sphere,
    // times 2 for the child's c_K·2/w against the parent's c_K/w
    k_yk_basis<<<nblk(nq, 128), 128, 0, s>>>(p, nq, xq, 2.0, -dh[0], -dh[1], -dh[2], 2.0, kh / 2, 1, 2.0, F.p);
    FMMB_LAUNCH_CHECK();
    gemm_columns(LD, nq, Pirr.p, bm, ColMap{out.m2m.p + (int64_t)k * LD * LD, nullptr, 0, 1, 0}, N, LD, N, 0, sms, s);
    // L2L: the parent's regular basis (κ̂) at the child sphere δ̂ + x̂/2
    k_yk_basis<<<nblk(nq, 128), 128, 0, s>>>(p, nq, xq, 0.5, dh[0], dh[1], dh[2], 1.0, kh, 0, 1.0, F.p);
    FMMB_LAUNCH_CHECK();
    gemm_columns(LD, nq, Pregc.p, bm, ColMap{out.l2l.p + (int64_t)k * LD, nullptr, 0, 1, (int64_t)NCH * LD}, N, LD, N, 0,
                 sms, s);
  }
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// the operators of every width built so far, by (device, p, κ, width): caches on different
// contexts (the request server's slots, successive servers) share them rather than rebuilding.
// The store keeps them after their last cache is gone, up to STORE_BYTES; beyond that the
// oldest that no cache holds are released.
constexpr size_t STORE_BYTES = size_t(4) << 30;
std::mutex g_store_mu;
std::map<std::tuple<int, int, double, double>, std::shared_ptr<YukawaLevel>> g_store;
std::vector<std::tuple<int, int, double, double>> g_store_order;   // insertion order
size_t g_store_bytes = 0;

size_t level_bytes(const YukawaLevel& lv) { return lv.reps.bytes() + lv.m2m.bytes() + lv.l2l.bytes(); }

void store_trim() {
  for (size_t i = 0; i < g_store_order.size() && g_store_bytes > STORE_BYTES;) {
    auto it = g_store.find(g_store_order[i]);
    if (it != g_store.end() && it->second.use_count() == 1) {
      g_store_bytes -= level_bytes(*it->second);
      g_store.erase(it);
      g_store_order.erase(g_store_order.begin() + i);
    } else {
      ++i;
    }
  }
}

std::shared_ptr<YukawaLevel> level_operators(Cache& C, int e, cudaStream_t s) {
  const auto key = std::make_tuple(C.ctx->device, C.p, C.kappa, std::ldexp(C.W0, e));
  std::lock_guard<std::mutex> lk(g_store_mu);
  auto it = g_store.find(key);
  if (it != g_store.end()) return it->second;
  // allocated outside the stream-ordered pool (freed by whichever cache releases it last)
  const cudaStream_t keep = g_alloc_stream;
  g_alloc_stream = nullptr;
  std::shared_ptr<YukawaLevel> lv;
  try {
    lv = std::make_shared<YukawaLevel>();
    build_level(C, e, *lv, s);
  } catch (...) {
    lv.reset();
    g_alloc_stream = keep;
    throw;
  }
  g_alloc_stream = keep;
  g_store[key] = lv;
  g_store_order.push_back(key);
  g_store_bytes += level_bytes(*lv);
  store_trim();
  return lv;
}

}  // namespace

void yukawa_prepare(Plan& P) {
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  std::vector<double> kh2(P.L, 0.0);
  {
    std::lock_guard<std::mutex> lk(C.mu);
    sphere_rule(C, s);
    for (int l = 0; l < P.L; ++l) {
      const int e = P.e0 - l;                       // the level's width is ldexp(cache W0, e)
      const double kh = C.kappa * std::ldexp(C.W0, e);
      kh2[l] = kh * kh;
      if (l < 2) continue;                          // no translations touch levels 0 and 1
      auto it = C.yk_levels.find(e);
      if (it == C.yk_levels.end()) it = C.yk_levels.emplace(e, level_operators(C, e, s)).first;
      if ((int)P.lv_yukawa.size() < P.L) P.lv_yukawa.resize(P.L);
      P.lv_yukawa[l] = it->second;
      P.lv_reps[l] = it->second->reps.p;
      P.lv_m2m[l] = it->second->m2m.p;
      P.lv_l2l[l] = it->second->l2l.p;
    }
  }
  to_device(P.d_kh2, kh2, s);
}

}  // namespace fmmb
