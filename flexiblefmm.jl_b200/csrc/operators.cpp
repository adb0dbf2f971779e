// Host precompute of the SphericalHarmonics(Laplace3D) operators, in FP64 (they stay on the
// host side of the product and are uploaded once per operator cache):
//   - the exact M2M and L2L blocks of the eight child slots (src/operators/harmonics.jl:376-397)
//   - the 34 class representatives of the D4h symmetry classes of the 316 far offsets, with
//     the kernel constant c_K / W_ref folded in (harmonics.jl:365-374, 398-401)
//   - the signed permutations of each far offset (src/operators/symmetry.jl:252-319), stored
//     as gathers: the source side P_sᵀ and the target side P_t (the inverse of idx_t)
//   - the coefficient tables of the Schmidt recurrences (harmonics.jl:172-188)
// The complex solid harmonics use the Hobson normalisation and are rescaled to the Schmidt
// semi-normalised real storage (harmonics.jl:1-27).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>

#include "common.cuh"

namespace fmmb {
namespace {

using cd = std::complex<double>;
inline int ci(int n, int m) { return n * n + n + m; }                 // complex index
inline int tri(int n, int m) { return n * (n + 1) / 2 + m; }          // triangular index
inline int rr(int n, int m) { return m == 0 ? n * n : n * n + 2 * m - 1; }  // real part slot
inline int ri(int n, int m) { return n * n + 2 * m; }                 // imaginary part slot

// Υ_n^m (regular, Hobson) by the upward recurrence in n for each m
std::vector<cd> regular(const double* x, int p) {
  std::vector<cd> Y((p + 1) * (p + 1));
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
  cd w(x[0], x[1]), s(1.0, 0.0);
  for (int m = 0; m <= p; ++m) {
    Y[ci(m, m)] = s;
    cd a(0.0, 0.0), b = s;
    for (int n = m + 1; n <= p; ++n) {
      cd c = ((double)(2 * n - 1) * x[2] * b - r2 * a) / (double)((n - m) * (n + m));
      Y[ci(n, m)] = c;
      a = b;
      b = c;
    }
    s *= -w / (double)(2 * (m + 1));
  }
  for (int n = 1; n <= p; ++n)
    for (int m = 1; m <= n; ++m) Y[ci(n, -m)] = ((m & 1) ? -1.0 : 1.0) * std::conj(Y[ci(n, m)]);
  return Y;
}

// Θ_n^m (irregular, Hobson)
std::vector<cd> irregular(const double* x, int p) {
  std::vector<cd> T((p + 1) * (p + 1));
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2], q = 1.0 / r2;
  cd w(x[0], x[1]), s(1.0 / std::sqrt(r2), 0.0);
  for (int m = 0; m <= p; ++m) {
    T[ci(m, m)] = s;
    cd a(0.0, 0.0), b = s;
    for (int n = m + 1; n <= p; ++n) {
      cd c = ((double)(2 * n - 1) * x[2] * b - (double)((n - 1) * (n - 1) - m * m) * a) * q;
      T[ci(n, m)] = c;
      a = b;
      b = c;
    }
    s *= -(double)(2 * m + 1) * q * w;
  }
  for (int n = 1; n <= p; ++n)
    for (int m = 1; m <= n; ++m) T[ci(n, -m)] = ((m & 1) ? -1.0 : 1.0) * std::conj(T[ci(n, m)]);
  return T;
}

// √((n−|m|)!(n+|m|)!), the Hobson → Schmidt factors
std::vector<double> schmidt(int p) {
  std::vector<double> s((p + 1) * (p + 1));
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      double f = 1.0;
      for (int k = 2; k <= n - std::abs(m); ++k) f *= k;
      for (int k = 2; k <= n + std::abs(m); ++k) f *= k;
      s[ci(n, m)] = std::sqrt(f);
    }
  return s;
}

// the real matrix (NP × NP, column-major) of a complex operator A (NP × NP, column-major)
// that commutes with the conjugate symmetry of real densities
std::vector<double> realify(const std::vector<cd>& A, int p) {
  int N = (p + 1) * (p + 1);
  std::vector<double> R((size_t)N * N, 0.0);
  std::vector<cd> v(N);
  for (int n1 = 0; n1 <= p; ++n1)
    for (int m1 = 0; m1 <= n1; ++m1)
      for (int part = 0; part < (m1 == 0 ? 1 : 2); ++part) {
        int j = m1 == 0 ? n1 * n1 : rr(n1, m1) + part;
        const cd* a = &A[(size_t)ci(n1, m1) * N];
        const cd* b = &A[(size_t)ci(n1, -m1) * N];
        double sg = (m1 & 1) ? -1.0 : 1.0;
        for (int i = 0; i < N; ++i)
          v[i] = m1 == 0 ? a[i] : (part == 0 ? a[i] + sg * b[i] : cd(0, 1) * (a[i] - sg * b[i]));
        double* col = &R[(size_t)j * N];
        for (int n = 0; n <= p; ++n) {
          col[n * n] = v[ci(n, 0)].real();
          for (int m = 1; m <= n; ++m) {
            col[rr(n, m)] = v[ci(n, m)].real();
            col[ri(n, m)] = v[ci(n, m)].imag();
          }
        }
      }
  return R;
}

struct SPerm { int perm[3], sign[3]; };

// the signed permutation of the real storage for z → u·[conj]^εy z, u = i^{mk}(−1)^{(n+m)εz}
// (target side) or its conjugate (source side), as (destination index, sign) per entry
void d4h_permutation(int p, int k, bool ey, bool ez, bool target, std::vector<int>& idx, std::vector<int>& sgn) {
  int N = (p + 1) * (p + 1);
  idx.assign(N, 0);
  sgn.assign(N, 1);
  for (int n = 0; n <= p; ++n) {
    idx[n * n] = n * n;
    sgn[n * n] = (ez && (n & 1)) ? -1 : 1;
    for (int m = 1; m <= n; ++m) {
      int a = rr(n, m), b = a + 1;
      int q = ((target ? m * k : -m * k) % 4 + 4) % 4;
      int s = (ez && ((n + m) & 1)) ? -1 : 1;
      int c = ey ? -1 : 1;
      switch (q) {
        case 0: idx[a] = a; sgn[a] = s;  idx[b] = b; sgn[b] = s * c;  break;
        case 1: idx[a] = b; sgn[a] = s;  idx[b] = a; sgn[b] = -s * c; break;
        case 2: idx[a] = a; sgn[a] = -s; idx[b] = b; sgn[b] = -s * c; break;
        default: idx[a] = b; sgn[a] = -s; idx[b] = a; sgn[b] = s * c; break;
      }
    }
  }
}

}  // namespace

HostOperators build_operators(int p, double ref_width) {
  require(p >= 1 && p <= PMAX, FMMB_ERR_ARGUMENT, "p must lie in 1.." + std::to_string(PMAX));
  HostOperators op;
  op.p = p;
  op.np = (p + 1) * (p + 1);
  op.ld = ld_of(p);
  const int N = op.np, LD = op.ld;
  std::vector<double> s = schmidt(2 * p);

  // M2M / L2L blocks per child slot: δ̂ = (slot offset − ½)/2
  op.m2m.assign((size_t)LD * 8 * LD, 0.0);
  op.l2l.assign((size_t)8 * LD * LD, 0.0);
  for (int k = 0; k < NCH; ++k) {
    double dh[3];
    for (int d = 0; d < 3; ++d) dh[d] = ((double)((k >> d) & 1) - 0.5) / 2;
    std::vector<cd> Y = regular(dh, p);
    std::vector<cd> A((size_t)N * N), B((size_t)N * N);
    for (int n1 = 0; n1 <= p; ++n1)
      for (int m1 = -n1; m1 <= n1; ++m1)
        for (int n = n1; n <= p; ++n) {
          int d = n - n1;
          for (int mm = std::max(-n, m1 - d); mm <= std::min(n, m1 + d); ++mm) {
            cd v = std::conj(Y[ci(d, mm - m1)]) * (s[ci(n, mm)] / s[ci(n1, m1)]) * std::ldexp(1.0, -n1);
            A[(size_t)ci(n1, m1) * N + ci(n, mm)] = v;
            B[(size_t)ci(n, mm) * N + ci(n1, m1)] = v;
          }
        }
    std::vector<double> RA = realify(A, p), RB = realify(B, p);
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        op.m2m[(size_t)(k * LD + j) * LD + i] = RA[(size_t)j * N + i];
        op.l2l[(size_t)j * 8 * LD + k * LD + i] = RB[(size_t)j * N + i];
      }
  }

  // the far offsets in table order, their classes and signed permutations
  std::vector<std::array<int, 3>> offs;
  for (int t = 0; t < 343; ++t) {
    std::array<int, 3> o{t % 7 - 3, (t / 7) % 7 - 3, (t / 49) % 7 - 3};
    if (std::max({std::abs(o[0]), std::abs(o[1]), std::abs(o[2])}) >= 2) offs.push_back(o);
  }
  // D4h: the signed permutations fixing the z axis, in the reference's enumeration order
  std::vector<SPerm> G;
  const int perms[2][3] = {{0, 1, 2}, {1, 0, 2}};
  for (auto& pp : perms)
    for (int sb = 0; sb < 8; ++sb) {
      SPerm R;
      for (int d = 0; d < 3; ++d) { R.perm[d] = pp[d]; R.sign[d] = ((sb >> d) & 1) ? -1 : 1; }
      G.push_back(R);
    }
  std::vector<std::array<int, 3>> reps;
  op.cls.resize(NFAR);
  op.gidx.assign((size_t)NFAR * LD, -1);
  op.gsgn.assign((size_t)NFAR * LD, 0);
  op.sidx.assign((size_t)NFAR * LD, -1);
  op.ssgn.assign((size_t)NFAR * LD, 0);
  for (int f = 0; f < NFAR; ++f) {
    const auto& o = offs[f];
    for (int d = 0; d < 3; ++d) op.faroff.push_back((int8_t)o[d]);
    int a = std::abs(o[0]), b = std::abs(o[1]);
    std::array<int, 3> r{std::max(a, b), std::min(a, b), std::abs(o[2])};
    int c = (int)(std::find(reps.begin(), reps.end(), r) - reps.begin());
    if (c == (int)reps.size()) reps.push_back(r);
    op.cls[f] = c;
    const SPerm* g = nullptr;
    for (auto& R : G) {
      bool ok = true;
      for (int k = 0; k < 3; ++k) ok = ok && R.sign[k] * r[R.perm[k]] == o[k];
      if (ok) { g = &R; break; }
    }
    require(g != nullptr, FMMB_ERR_DEVICE, "no D4h element maps the class representative");
    // g = Rot_z(kπ/2) ∘ Refl_y^εy ∘ Refl_z^εz
    bool ez = g->sign[2] == -1;
    int A2[2][2] = {{0, 0}, {0, 0}};
    A2[0][g->perm[0]] = g->sign[0];
    A2[1][g->perm[1]] = g->sign[1];
    bool ey = A2[0][0] * A2[1][1] - A2[0][1] * A2[1][0] == -1;
    if (ey) { A2[0][1] = -A2[0][1]; A2[1][1] = -A2[1][1]; }
    // the rotation index: A2 = [[cos, −sin], [sin, cos]] of kπ/2
    int k = (A2[0][0] == 1) ? 0 : (A2[1][0] == 1) ? 1 : (A2[0][0] == -1) ? 2 : 3;
    op.d4h.push_back((uint8_t)(k | (ey ? 4 : 0) | (ez ? 8 : 0)));
    std::vector<int> is, ss, it, st;
    d4h_permutation(p, k, ey, ez, false, is, ss);
    d4h_permutation(p, k, ey, ez, true, it, st);
    for (int i = 0; i < N; ++i) {
      op.gidx[(size_t)f * LD + i] = (int16_t)is[i];
      op.gsgn[(size_t)f * LD + i] = (int8_t)ss[i];
      // (P_t y)[it[i]] = st[i] y[i]  ⇔  (P_t y)[j] = st[i] y[i] with i = it⁻¹[j]
      op.sidx[(size_t)f * LD + it[i]] = (int16_t)i;
      op.ssgn[(size_t)f * LD + it[i]] = (int8_t)st[i];
    }
  }
  require((int)reps.size() == NCLASS, FMMB_ERR_DEVICE, "expected 34 harmonic classes");
  for (auto& r : reps) op.reps_off.insert(op.reps_off.end(), r.begin(), r.end());

  // the class representatives: M2L of offset o in the Schmidt real basis, times c_K / W_ref
  const double cK = 1.0 / (4.0 * M_PI);
  double c = cK / ref_width;
  op.reps.assign((size_t)NCLASS * LD * LD, 0.0);
  for (int q = 0; q < NCLASS; ++q) {
    double od[3] = {(double)reps[q][0], (double)reps[q][1], (double)reps[q][2]};
    std::vector<cd> T = irregular(od, 2 * p);
    std::vector<cd> A((size_t)N * N);
    for (int k2 = 0; k2 <= p; ++k2)
      for (int l = -k2; l <= k2; ++l) {
        double sk = ((k2 & 1) ? -1.0 : 1.0) * c / s[ci(k2, l)];
        for (int n = 0; n <= p; ++n)
          for (int mm = -n; mm <= n; ++mm) A[(size_t)ci(k2, l) * N + ci(n, mm)] = sk * T[ci(n + k2, mm + l)] / s[ci(n, mm)];
      }
    std::vector<double> R = realify(A, p);
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) op.reps[(size_t)q * LD * LD + (size_t)j * LD + i] = R[(size_t)j * N + i];
  }

  // recurrence tables
  op.ntri = tri(p, p) + 1;
  int nt = op.ntri;
  op.tables.assign((size_t)5 * nt + p, 0.0);
  double* ta = &op.tables[0];
  double* tb = &op.tables[nt];
  double* tz = &op.tables[2 * nt];
  double* tm = &op.tables[3 * nt];
  double* tp = &op.tables[4 * nt];
  double* te = &op.tables[5 * nt];
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      int t = tri(n, m);
      double cc = std::sqrt((double)((n - m) * (n + m)));
      tz[t] = cc;
      if (n > m) {
        ta[t] = (double)(2 * n - 1) / cc;
        tb[t] = std::sqrt((double)((n - m - 1) * (n + m - 1))) / cc;
      }
      tm[t] = n + m >= 2 ? std::sqrt((double)((n + m) * (n + m - 1))) : 0.0;
      tp[t] = n - m >= 2 ? std::sqrt((double)((n - m) * (n - m - 1))) : 0.0;
    }
  for (int m = 1; m <= p; ++m) te[m - 1] = std::sqrt((double)(2 * m - 1) / (double)(2 * m));
  return op;
}

}  // namespace fmmb
