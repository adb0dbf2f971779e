// Host precompute of CubeKernelIndependent{3}(Laplace3D(); p, pc, d) (src/operators/cubeki.jl,
// src/operators/ki_common.jl), in FP64 at the cache's base width:
//   - the small surface (p points per edge, half-width (1+d)·w/2: upward equivalent, downward
//     check) and the large one (pc per edge, (3−2d)·w/2: upward check, downward equivalent),
//     the boundary points of the lattices in CartesianIndices order (coordinate 1 fastest), and
//     each small point's index in the zero-padded (2p)³ lattice (cubeki.jl:52-67,
//     spectral_m2l.jl:159-172);
//   - the truncated pseudo-inverses of the two check maps (pinv_rtol, ki_common.jl:38-44) kept
//     as factors V and diag(1/σ)·Uᴴ, by a one-sided Jacobi SVD;
//   - M2M and L2L with the pseudo-inverses folded in the reference's order
//     (ki_common.jl:176-199): V·(diag(1/σ)·(Uᴴ·M2Mc)) and ((L2Lc·V)·diag(1/σ))·Uᴴ.
// Laplace3D is homogeneous of degree −1: M2M and L2L are width-invariant, the pseudo-inverses
// scale by λ = w/w_ref and the M2L by 1/λ (ki_common.jl:207-218).
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "ki.h"

namespace fmmb {
namespace {

constexpr double KCL = 0.079577471545947667884;   // 1/(4π)

int nthreads() { return std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }

// run f(t, T) on T threads
template <class F>
void parallel(F&& f) {
  const int T = nthreads();
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) th.emplace_back([&, t] { f(t, T); });
  f(0, T);
  for (auto& x : th) x.join();
}

// a reusable barrier for the Jacobi rounds
struct Barrier {
  std::mutex m;
  std::condition_variable cv;
  int n, count = 0, gen = 0;
  explicit Barrier(int k) : n(k) {}
  void wait() {
    std::unique_lock<std::mutex> lk(m);
    const int g = gen;
    if (++count == n) { count = 0; ++gen; cv.notify_all(); }
    else cv.wait(lk, [&] { return gen != g; });
  }
};

// One-sided Jacobi (Hestenes) SVD of a column-major m × n matrix A, m ≥ n: A·V = U·Σ. The
// columns are rotated pairwise in round-robin order (n/2 disjoint pairs per round, run on
// several threads) until every pair is orthogonal to rounding. Returns σ (descending), U
// (m × n) and V (n × n), column-major.
void jacobi_svd(int m, int n, std::vector<double> A, std::vector<double>& sigma, std::vector<double>& U,
                std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  const int nn = n + (n & 1);               // a dummy column when n is odd
  std::vector<int> ring(nn);
  for (int i = 0; i < nn; ++i) ring[i] = i;
  const int T = nthreads();
  const double tol = 4 * 2.220446049250313e-16 * std::sqrt((double)m);   // orthogonal to rounding
  Barrier bar(T);
  std::atomic<int> rotated{0};
  bool done = false;
  auto worker = [&](int t) {
    for (int sweep = 0; sweep < 40; ++sweep) {
      for (int round = 0; round < nn - 1; ++round) {
        for (int k = t; k < nn / 2; k += T) {
          int i = ring[k], j = ring[nn - 1 - k];
          if (i >= n || j >= n) continue;
          if (i > j) std::swap(i, j);
          double* a = &A[(size_t)i * m];
          double* b = &A[(size_t)j * m];
          double al = 0, be = 0, ga = 0;
          for (int r = 0; r < m; ++r) { al += a[r] * a[r]; be += b[r] * b[r]; ga += a[r] * b[r]; }
          if (ga == 0 || std::fabs(ga) <= tol * std::sqrt(al * be)) continue;
          const double ze = (be - al) / (2 * ga);
          const double tt = (ze >= 0 ? 1.0 : -1.0) / (std::fabs(ze) + std::sqrt(1 + ze * ze));
          const double c = 1 / std::sqrt(1 + tt * tt), s = c * tt;
          for (int r = 0; r < m; ++r) {
            const double x = a[r], y = b[r];
            a[r] = c * x - s * y;
            b[r] = s * x + c * y;
          }
          double* va = &V[(size_t)i * n];
          double* vb = &V[(size_t)j * n];
          for (int r = 0; r < n; ++r) {
            const double x = va[r], y = vb[r];
            va[r] = c * x - s * y;
            vb[r] = s * x + c * y;
          }
          rotated.fetch_add(1, std::memory_order_relaxed);
        }
        bar.wait();
        if (t == 0) {                       // next round of the tournament: fix ring[0], rotate the rest
          const int last = ring[nn - 1];
          for (int k = nn - 1; k > 1; --k) ring[k] = ring[k - 1];
          ring[1] = last;
        }
        bar.wait();
      }
      if (t == 0) {
        done = rotated.load() == 0;
        rotated = 0;
      }
      bar.wait();
      if (done) return;
      bar.wait();
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) th.emplace_back(worker, t);
  worker(0);
  for (auto& x : th) x.join();
  // σ and U, sorted by σ descending
  std::vector<double> s(n);
  for (int j = 0; j < n; ++j) {
    double q = 0;
    for (int r = 0; r < m; ++r) q += A[(size_t)j * m + r] * A[(size_t)j * m + r];
    s[j] = std::sqrt(q);
  }
  std::vector<int> ord(n);
  for (int j = 0; j < n; ++j) ord[j] = j;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return s[a] > s[b]; });
  sigma.resize(n);
  U.assign((size_t)m * n, 0.0);
  std::vector<double> V2((size_t)n * n);
  for (int k = 0; k < n; ++k) {
    const int j = ord[k];
    sigma[k] = s[j];
    for (int r = 0; r < m; ++r) U[(size_t)k * m + r] = s[j] > 0 ? A[(size_t)j * m + r] / s[j] : 0.0;
    for (int r = 0; r < n; ++r) V2[(size_t)k * n + r] = V[(size_t)j * n + r];
  }
  V.swap(V2);
}

// the boundary points of the p³ lattice spanning [−a, a]³, coordinate 1 fastest, and their
// linear indices in the zero-padded (2p)³ lattice (spectral_m2l.jl:159-172)
void cube_boundary_points(int p, double a, std::vector<double>& pts, std::vector<int>* embed) {
  pts.clear();
  if (embed) embed->clear();
  for (int i3 = 0; i3 < p; ++i3)
    for (int i2 = 0; i2 < p; ++i2)
      for (int i1 = 0; i1 < p; ++i1) {
        if (!(i1 == 0 || i1 == p - 1 || i2 == 0 || i2 == p - 1 || i3 == 0 || i3 == p - 1)) continue;
        const int ii[3] = {i1, i2, i3};
        for (int d = 0; d < 3; ++d) pts.push_back(-a + 2 * a * (double)ii[d] / (p - 1));
        if (embed) embed->push_back(i1 + 2 * p * (i2 + 2 * p * i3));
      }
}

inline double lap(const double* x, const double* y) {
  const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
  return KCL / std::sqrt(dx * dx + dy * dy + dz * dz);
}

// the kernel matrix (targets × sources, column-major) of unit densities at `src` (+ shift cs)
// seen at `tgt` (+ shift ct)
std::vector<double> kernel_matrix(const std::vector<double>& src, const double* cs, const std::vector<double>& tgt,
                                  const double* ct) {
  const int ns = (int)src.size() / 3, nt = (int)tgt.size() / 3;
  std::vector<double> K((size_t)nt * ns);
  parallel([&](int t, int T) {
    for (int j = t; j < ns; j += T) {
      const double y[3] = {src[3 * j] + cs[0], src[3 * j + 1] + cs[1], src[3 * j + 2] + cs[2]};
      for (int i = 0; i < nt; ++i) {
        const double x[3] = {tgt[3 * i] + ct[0], tgt[3 * i + 1] + ct[1], tgt[3 * i + 2] + ct[2]};
        K[(size_t)j * nt + i] = lap(x, y);
      }
    }
  });
  return K;
}

// C (m × n) = A (m × k) · B (k × n), column-major, threaded over columns
std::vector<double> matmul(int m, int k, int n, const std::vector<double>& A, const std::vector<double>& B) {
  std::vector<double> C((size_t)m * n, 0.0);
  parallel([&](int t, int T) {
    for (int j = t; j < n; j += T) {
      double* c = &C[(size_t)j * m];
      for (int q = 0; q < k; ++q) {
        const double b = B[(size_t)j * k + q];
        if (b == 0) continue;
        const double* a = &A[(size_t)q * m];
        for (int i = 0; i < m; ++i) c[i] += a[i] * b;
      }
    }
  });
  return C;
}

// the truncated pseudo-inverse of a column-major m × n matrix (either shape), as V (n × r) and
// S⁺Uᴴ (r × m)
void pinv_factors(int m, int n, const std::vector<double>& A, double rtol, std::vector<double>& Vf,
                  std::vector<double>& SU, int& r) {
  std::vector<double> sigma, U, V;
  if (m >= n) {
    jacobi_svd(m, n, A, sigma, U, V);             // A = U Σ Vᵀ: U m × n, V n × n
  } else {
    std::vector<double> At((size_t)n * m);        // Aᵀ (n × m) = U' Σ V'ᵀ  ⇒  A = V' Σ U'ᵀ
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) At[(size_t)i * n + j] = A[(size_t)j * m + i];
    std::vector<double> Up, Vp;
    jacobi_svd(n, m, At, sigma, Up, Vp);
    U.swap(Vp);                                   // m × m
    V.swap(Up);                                   // n × m
  }
  const int kmax = (int)sigma.size();
  r = 0;
  while (r < kmax && sigma[r] >= rtol * sigma[0]) ++r;
  const int ucols = m >= n ? n : m;               // columns of U, length m each
  const int vrows = n;
  (void)ucols;
  Vf.assign((size_t)vrows * r, 0.0);
  SU.assign((size_t)r * m, 0.0);
  for (int k = 0; k < r; ++k) {
    for (int i = 0; i < vrows; ++i) Vf[(size_t)k * vrows + i] = V[(size_t)k * vrows + i];
    for (int i = 0; i < m; ++i) SU[(size_t)i * r + k] = U[(size_t)k * m + i] / sigma[k];
  }
}

// the 2D Laplace kernel c·log(r²), c = −1/(4π) (src/kernels.jl:58-66), between points in the plane
inline double lap2(const double* x, const double* y) {
  const double dx = x[0] - y[0], dy = x[1] - y[1];
  return -KCL * std::log(dx * dx + dy * dy);
}

// N equispaced points on the circle of radius r about (cx, cy), angle 2πk/N (kifmm.jl:69-71)
std::vector<double> circle(int N, double r, double cx = 0, double cy = 0) {
  std::vector<double> p(2 * N);
  for (int k = 0; k < N; ++k) {
    const double t = 2 * M_PI / N * k;
    p[2 * k] = cx + r * std::cos(t);
    p[2 * k + 1] = cy + r * std::sin(t);
  }
  return p;
}

// targets × sources, column-major, of the 2D kernel
std::vector<double> kernel_matrix2(const std::vector<double>& src, const std::vector<double>& tgt) {
  const int ns = (int)src.size() / 2, nt = (int)tgt.size() / 2;
  std::vector<double> K((size_t)nt * ns);
  for (int j = 0; j < ns; ++j)
    for (int i = 0; i < nt; ++i) K[(size_t)j * nt + i] = lap2(&tgt[2 * i], &src[2 * j]);
  return K;
}

}  // namespace

KICircleLevel build_ki_circle_level(int n, double rtol, double w) {
  require(n >= 4 && n <= 64, FMMB_ERR_ARGUMENT, "nequiv must lie in 4..64");
  KICircleLevel c;
  c.n = n;
  c.ld = 64;
  const int L = c.ld;
  const std::vector<double> small = circle(n, KIC_SMALL * w), large = circle(n, KIC_LARGE * w);
  std::vector<double> uv, usu, dv, dsu;
  pinv_factors(n, n, kernel_matrix2(small, large), rtol, uv, usu, c.rank_up);
  pinv_factors(n, n, kernel_matrix2(large, small), rtol, dv, dsu, c.rank_down);
  // M2Mc: each child slot's small circle (centre (δx − ½, δy − ½)·w/2) seen on the large one;
  // L2Lc: the large circle seen on each child's small one
  std::vector<double> M2Mc((size_t)n * NCH * n), L2Lc((size_t)NCH * n * n);
  for (int k = 0; k < NCH; ++k) {
    const double cx = ((k & 1) - 0.5) * (w / 2), cy = (((k >> 1) & 1) - 0.5) * (w / 2);
    const std::vector<double> ch = circle(n, KIC_SMALL * w / 2, cx, cy);
    const std::vector<double> a = kernel_matrix2(ch, large), b = kernel_matrix2(large, ch);
    std::copy(a.begin(), a.end(), M2Mc.begin() + (size_t)k * n * n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) L2Lc[(size_t)j * NCH * n + k * n + i] = b[(size_t)j * n + i];
  }
  const int ru = c.rank_up, rd = c.rank_down;
  const std::vector<double> m2m = matmul(n, ru, NCH * n, uv, matmul(ru, n, NCH * n, usu, M2Mc));
  const std::vector<double> l2l = matmul(NCH * n, rd, n, matmul(NCH * n, n, rd, L2Lc, dv), dsu);
  // zero-padded copies
  auto padm = [](const std::vector<double>& a, int rows, int cols, int R, int C) {
    std::vector<double> o((size_t)R * C, 0.0);
    for (int j = 0; j < cols; ++j)
      for (int i = 0; i < rows; ++i) o[(size_t)j * R + i] = a[(size_t)j * rows + i];
    return o;
  };
  c.up_v = padm(uv, n, ru, L, L);
  c.up_su = padm(usu, ru, n, L, L);
  c.down_v = padm(dv, n, rd, L, L);
  c.down_su = padm(dsu, rd, n, L, L);
  c.m2m.assign((size_t)L * NCH * L, 0.0);
  c.l2l.assign((size_t)NCH * L * L, 0.0);
  for (int k = 0; k < NCH; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        c.m2m[(size_t)(k * L + j) * L + i] = m2m[(size_t)(k * n + j) * n + i];
        c.l2l[(size_t)j * NCH * L + k * L + i] = l2l[(size_t)j * NCH * n + k * n + i];
      }
  // M2L: the source's small circle at offset o·w seen on the target's small circle
  c.m2l.assign((size_t)NFAR * L * L, 0.0);
  int f = 0;
  for (int t = 0; t < 343; ++t) {
    const int o[3] = {t % 7 - 3, (t / 7) % 7 - 3, (t / 49) % 7 - 3};
    if (std::max({std::abs(o[0]), std::abs(o[1]), std::abs(o[2])}) < 2) continue;
    if (o[2] == 0) {
      const std::vector<double> src = circle(n, KIC_SMALL * w, o[0] * w, o[1] * w);
      const std::vector<double> A = kernel_matrix2(src, small);
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) c.m2l[(size_t)f * L * L + (size_t)j * L + i] = A[(size_t)j * n + i];
    }
    ++f;
  }
  return c;
}

KIHost build_ki_operators(int p, int pc, double d, double rtol, double w) {
  require(p >= 2 && p <= KI_PMAX, FMMB_ERR_ARGUMENT, "the cube KI method takes 2 ≤ p ≤ " + std::to_string(KI_PMAX));
  require(pc >= p && pc <= 4 * KI_PMAX, FMMB_ERR_ARGUMENT, "pc must lie in p..4·p_max");
  require(d > 0 && d < 2.0 / 3.0, FMMB_ERR_ARGUMENT, "d must lie in (0, 2/3)");
  KIHost h;
  h.p = p;
  h.pc = pc;
  h.d = d;
  h.w = w;
  const double as = (1 + d) * w / 2, al = (3 - 2 * d) * w / 2;
  cube_boundary_points(p, as, h.small, &h.embed);
  cube_boundary_points(pc, al, h.large, nullptr);
  std::vector<double> child;
  cube_boundary_points(p, as / 2, child, nullptr);
  h.ns = (int)h.small.size() / 3;
  h.nl = (int)h.large.size() / 3;
  h.h = 2 * as / (p - 1);
  const int ns = h.ns, nl = h.nl;
  const double zero[3] = {0, 0, 0};
  // upward: unit densities on the small surface seen on the large (check) surface
  pinv_factors(nl, ns, kernel_matrix(h.small, zero, h.large, zero), rtol, h.up_v, h.up_su, h.rank_up);
  // downward: unit densities on the large surface seen on the small (check) surface
  pinv_factors(ns, nl, kernel_matrix(h.large, zero, h.small, zero), rtol, h.down_v, h.down_su, h.rank_down);
  // M2Mc: the children's small surfaces (centres (δ − ½)·w/2) seen on the parent's large one;
  // L2Lc: the parent's large surface seen on the children's small ones
  std::vector<double> M2Mc((size_t)nl * NCH * ns), L2Lc((size_t)NCH * ns * nl);
  for (int k = 0; k < NCH; ++k) {
    double c[3];
    for (int dd = 0; dd < 3; ++dd) c[dd] = ((double)((k >> dd) & 1) - 0.5) * (w / 2);
    std::vector<double> a = kernel_matrix(child, c, h.large, zero);     // nl × ns
    std::copy(a.begin(), a.end(), M2Mc.begin() + (size_t)k * nl * ns);
    std::vector<double> b = kernel_matrix(h.large, zero, child, c);     // ns × nl
    for (int j = 0; j < nl; ++j)
      for (int i = 0; i < ns; ++i) L2Lc[(size_t)j * NCH * ns + k * ns + i] = b[(size_t)j * ns + i];
  }
  const int ru = h.rank_up, rd = h.rank_down;
  h.m2m = matmul(ns, ru, NCH * ns, h.up_v, matmul(ru, nl, NCH * ns, h.up_su, M2Mc));        // ns × 8ns
  h.l2l = matmul(NCH * ns, rd, ns, matmul(NCH * ns, nl, rd, L2Lc, h.down_v), h.down_su);   // 8ns × ns
  // the kernel tables of the 316 far offsets (coordinate 1 fastest, as the far-offset
  // enumeration), transformed by separable DFTs (forward sign −, no normalisation)
  const int n = 2 * p, nh = p + 1;
  h.nfreq = nh * n * n;
  h.tables.assign((size_t)NFAR * h.nfreq * 2, 0.0);
  std::vector<std::array<int, 3>> offs;
  for (int t = 0; t < 343; ++t) {
    std::array<int, 3> o{t % 7 - 3, (t / 7) % 7 - 3, (t / 49) % 7 - 3};
    if (std::max({std::abs(o[0]), std::abs(o[1]), std::abs(o[2])}) >= 2) offs.push_back(o);
  }
  std::vector<double> cs(n), sn(n);
  for (int k = 0; k < n; ++k) { cs[k] = std::cos(2 * M_PI * k / n); sn[k] = std::sin(2 * M_PI * k / n); }
  parallel([&](int t, int T) {
    std::vector<double> x((size_t)n * n * n), a1r((size_t)nh * n * n), a1i((size_t)nh * n * n),
        a2r((size_t)nh * n * n), a2i((size_t)nh * n * n);
    for (int f = t; f < NFAR; f += T) {
      std::fill(x.begin(), x.end(), 0.0);
      const double src[3] = {(double)offs[f][0] * w, (double)offs[f][1] * w, (double)offs[f][2] * w};
      for (int m3 = -(p - 1); m3 <= p - 1; ++m3)
        for (int m2 = -(p - 1); m2 <= p - 1; ++m2)
          for (int m1 = -(p - 1); m1 <= p - 1; ++m1) {
            const double tg[3] = {h.h * m1, h.h * m2, h.h * m3};
            const int j1 = (m1 + n) % n, j2 = (m2 + n) % n, j3 = (m3 + n) % n;
            x[(size_t)j1 + n * (j2 + (size_t)n * j3)] = lap(tg, src);
          }
      // dim 1 (real → half), then dims 2 and 3 (complex)
      for (int j3 = 0; j3 < n; ++j3)
        for (int j2 = 0; j2 < n; ++j2)
          for (int k1 = 0; k1 < nh; ++k1) {
            double re = 0, im = 0;
            for (int j1 = 0; j1 < n; ++j1) {
              const double v = x[(size_t)j1 + n * (j2 + (size_t)n * j3)];
              const int q = (j1 * k1) % n;
              re += v * cs[q];
              im -= v * sn[q];
            }
            a1r[(size_t)k1 + nh * (j2 + (size_t)n * j3)] = re;
            a1i[(size_t)k1 + nh * (j2 + (size_t)n * j3)] = im;
          }
      for (int j3 = 0; j3 < n; ++j3)
        for (int k2 = 0; k2 < n; ++k2)
          for (int k1 = 0; k1 < nh; ++k1) {
            double re = 0, im = 0;
            for (int j2 = 0; j2 < n; ++j2) {
              const size_t i = (size_t)k1 + nh * (j2 + (size_t)n * j3);
              const int q = (j2 * k2) % n;
              re += a1r[i] * cs[q] + a1i[i] * sn[q];
              im += a1i[i] * cs[q] - a1r[i] * sn[q];
            }
            a2r[(size_t)k1 + nh * (k2 + (size_t)n * j3)] = re;
            a2i[(size_t)k1 + nh * (k2 + (size_t)n * j3)] = im;
          }
      double* out = &h.tables[(size_t)f * h.nfreq * 2];
      for (int k3 = 0; k3 < n; ++k3)
        for (int k2 = 0; k2 < n; ++k2)
          for (int k1 = 0; k1 < nh; ++k1) {
            double re = 0, im = 0;
            for (int j3 = 0; j3 < n; ++j3) {
              const size_t i = (size_t)k1 + nh * (k2 + (size_t)n * j3);
              const int q = (j3 * k3) % n;
              re += a2r[i] * cs[q] + a2i[i] * sn[q];
              im += a2i[i] * cs[q] - a2r[i] * sn[q];
            }
            const size_t o = (size_t)k1 + nh * (k2 + (size_t)n * k3);
            out[2 * o] = re;
            out[2 * o + 1] = im;
          }
    }
  });
  return h;
}

}  // namespace fmmb
