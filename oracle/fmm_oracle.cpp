// CPU ORACLE — test infrastructure only.
//
// A restatement, in C++/OpenMP, of the reference CPU path of FlexibleFMM.jl for the
// Laplace3D `SphericalHarmonics` method: the ghost-cell tree, the interaction lists,
// the analytic operators with the 34 D4h symmetry classes, the upward and downward
// passes with the class-wise M2L in 32-target blocks, the evaluation at sources and
// at targets, and the FP64 direct sums. Only the tests, the smoke check and the CPU
// baseline leg of the benchmark load this library; the product path never does.
//
// Parity anchor: the reference cannot run here (no Julia). The restatement is pinned
// by the reference's own known-answer tests and tolerances (Hobson values and
// identities, class reconstruction, orbit sizes, tree invariants, FMM vs direct sums),
// restated in tests/test_oracle.py. Citations are file:line within the reference.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <numeric>
#include <omp.h>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

using cplx = std::complex<double>;
typedef int64_t i64;

// ---------------------------------------------------------------- indices
// src/operators/harmonics.jl:29-30 (0-based here)
static inline int cidx(int n, int m) { return n * n + n + m; }
static inline int tidx(int n, int m) { return (n * (n + 1)) / 2 + m; }
// real storage (src/operators/harmonics.jl:20-27): M_n^0 at n², Re/Im M_n^m at n²+2m-1, n²+2m
static inline int rre(int n, int m) { return m == 0 ? n * n : n * n + 2 * m - 1; }
static inline int rim(int n, int m) { return n * n + 2 * m; }

// ---------------------------------------------------------------- util.jl
static const int NCH = 8, NCOL = 27, NFAR = 316;
struct I3 { int v[3]; };
// colleague offsets, coordinate 1 fastest (src/util.jl:12-16,53)
static I3 coll_off(int k) { I3 o; for (int d = 0, b = 1; d < 3; ++d, b *= 3) o.v[d] = (k / b) % 3 - 1; return o; }
// child offsets: slot k has bit d = coordinate d (src/util.jl:24-27)
static I3 child_off(int k) { I3 o; for (int d = 0; d < 3; ++d) o.v[d] = (k >> d) & 1; return o; }
// m2l table index (src/util.jl:65-71)
static int table_index(const int o[3]) { int k = 0; for (int d = 0, b = 1; d < 3; ++d, b *= 7) k += (o[d] + 3) * b; return k; }
static bool is_far(const int o[3]) { int m = 0; for (int d = 0; d < 3; ++d) m = std::max(m, std::abs(o[d])); return m >= 2; }
// far offsets in table order and the table → far index map (src/util.jl:79,87-97)
static std::vector<I3> far_offsets() {
  std::vector<I3> out;
  for (int i = 0; i < 343; ++i) {
    I3 o; for (int d = 0, b = 1; d < 3; ++d, b *= 7) o.v[d] = (i / b) % 7 - 3;
    if (is_far(o.v)) out.push_back(o);
  }
  return out;
}
static std::vector<int> far_index_table() {
  std::vector<int> t(343, -1); int n = 0;
  for (int i = 0; i < 343; ++i) {
    int o[3]; for (int d = 0, b = 1; d < 3; ++d, b *= 7) o[d] = (i / b) % 7 - 3;
    if (is_far(o)) t[i] = n++;
  }
  return t;
}
// child slot: coordinate strictly above the centre goes up (src/util.jl:39-45)
static inline int child_slot(const double* x, const double* c) {
  int k = 0; for (int d = 0; d < 3; ++d) k += (x[d] > c[d]) << d; return k;
}
// centre of a lattice cell at width w (src/tree/tree.jl:81-83); built without contraction
static inline void cell_center(const double* origin, const int* cell, double w, double* c) {
  for (int d = 0; d < 3; ++d) { double t = (double)cell[d] + 0.5; t = t * w; c[d] = origin[d] + t; }
}
static uint64_t morton_key(const int* cell, int nbits) {   // src/util.jl:132-138
  uint64_t key = 0;
  for (int b = 0; b < nbits; ++b) for (int k = 0; k < 3; ++k) key |= (uint64_t)((cell[k] >> b) & 1) << (3 * b + k);
  return key;
}

struct Error : std::runtime_error { int code; Error(int c, const std::string& s) : std::runtime_error(s), code(c) {} };

// ---------------------------------------------------------------- tree builder (src/tree/builder.jl)
struct LevelB {
  std::vector<int> cell, parent, cf, lo, hi, depth, col;
  std::vector<uint8_t> leaf, ghost, xlist;
  int n() const { return (int)parent.size(); }
  void push(const int* c, int par, int l0, int h0, bool lf, bool gh) {
    cell.insert(cell.end(), c, c + 3); parent.push_back(par); cf.push_back(-1); lo.push_back(l0); hi.push_back(h0);
    leaf.push_back(lf); ghost.push_back(gh); xlist.push_back(0); depth.push_back(0);
  }
};

// split_nodes! (builder.jl:45-69): stable counting sort by child slot, children appended in
// the order of `which`, each sibling group in slot order
static void split_nodes(LevelB& par, const std::vector<int>& which, int l, LevelB& chi, std::vector<double>& pts,
                        std::vector<int>& perm, std::vector<double>& spts, std::vector<int>& sperm,
                        const double* origin, double W0, bool ghost) {
  double w = std::ldexp(W0, -l);
  for (int i : which) {
    if (par.cf[i] != -1) throw Error(4, "node already has children");
    double c[3]; cell_center(origin, &par.cell[3 * i], w, c);
    int lo = par.lo[i], hi = par.hi[i];
    int counts[NCH] = {0}, starts[NCH], pos[NCH];
    for (int j = lo; j <= hi; ++j) counts[child_slot(&pts[3 * j], c)]++;
    int s = lo; for (int k = 0; k < NCH; ++k) { starts[k] = s; pos[k] = s; s += counts[k]; }
    for (int j = lo; j <= hi; ++j) {
      int k = child_slot(&pts[3 * j], c);
      int p = pos[k]++;
      spts[3 * p] = pts[3 * j]; spts[3 * p + 1] = pts[3 * j + 1]; spts[3 * p + 2] = pts[3 * j + 2]; sperm[p] = perm[j];
    }
    for (int j = lo; j <= hi; ++j) { pts[3 * j] = spts[3 * j]; pts[3 * j + 1] = spts[3 * j + 1]; pts[3 * j + 2] = spts[3 * j + 2]; perm[j] = sperm[j]; }
    par.cf[i] = chi.n();
    if (!ghost) par.leaf[i] = 0;
    for (int k = 0; k < NCH; ++k) {
      I3 o = child_off(k);
      int cc[3] = {2 * par.cell[3 * i] + o.v[0], 2 * par.cell[3 * i + 1] + o.v[1], 2 * par.cell[3 * i + 2] + o.v[2]};
      chi.push(cc, i, starts[k], starts[k] + counts[k] - 1, !ghost, ghost);
    }
  }
}

// tag_colleagues! by the parent rule (builder.jl:212-248)
static void tag_colleagues(LevelB& lev, const LevelB& par) {
  int n = lev.n();
  lev.col.assign((size_t)NCOL * n, -1);
  for (int i = 0; i < n; ++i) {
    const int* c = &lev.cell[3 * i];
    int p = lev.parent[i];
    int pc[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
    for (int k = 0; k < NCOL; ++k) {
      I3 o = coll_off(k);
      int cc[3] = {c[0] + o.v[0], c[1] + o.v[1], c[2] + o.v[2]};
      int oi = 0; for (int j = 0, b = 1; j < 3; ++j, b *= 3) oi += (((cc[j] >> 1) - pc[j]) + 1) * b;
      int q = par.col[(size_t)NCOL * p + oi];
      int sb = (cc[0] & 1) | ((cc[1] & 1) << 1) | ((cc[2] & 1) << 2);
      lev.col[(size_t)NCOL * i + k] = (q < 0 || par.cf[q] < 0) ? -1 : par.cf[q] + sb;
    }
  }
}
static void tag_root(LevelB& root) { root.col.assign(NCOL, -1); root.col[13] = 0; }

static void compute_depths(std::vector<LevelB>& levels) {   // builder.jl:260-280
  int L = (int)levels.size();
  std::fill(levels[L - 1].depth.begin(), levels[L - 1].depth.end(), 0);
  for (int l = L - 2; l >= 0; --l) {
    LevelB& lev = levels[l]; LevelB& nxt = levels[l + 1];
    for (int i = 0; i < lev.n(); ++i) {
      int f = lev.cf[i];
      if (f < 0) { lev.depth[i] = 0; continue; }
      int m = 0; for (int k = 0; k < NCH; ++k) m = std::max(m, nxt.depth[f + k]);
      lev.depth[i] = m + 1;
    }
  }
}

struct Tree {
  double origin[3], W0;
  int L, N, n;
  std::vector<int> level_start;                  // L+1
  std::vector<int> cell, level, parent, cf, plo, phi, col, perm, point_node;
  std::vector<uint8_t> leaf, ghost, xlist, has_source;
  // interaction lists per level by target: tptr[node-local], tsrc, tfar (fill order)
  std::vector<std::vector<int>> ptr, src, far;
};

static Tree build_tree(const double* xyz, int N, int ppl, const double* origin, double W0, int max_levels) {
  if (ppl < 1) throw Error(1, "ppl must be positive");
  if (N <= 0) throw Error(1, "no points");
  if (!(W0 > 0)) throw Error(1, "box width must be positive");
  for (int j = 0; j < N; ++j)
    for (int d = 0; d < 3; ++d) {
      double x = xyz[3 * j + d];
      if (!(origin[d] <= x && x <= origin[d] + W0)) throw Error(1, "point lies outside the box");
    }
  std::vector<double> pts(xyz, xyz + 3 * (size_t)N), spts(3 * (size_t)N);
  std::vector<int> perm(N), sperm(N);
  std::iota(perm.begin(), perm.end(), 0);
  std::vector<LevelB> levels(1);
  int zero[3] = {0, 0, 0};
  levels[0].push(zero, -1, 0, N - 1, true, false);
  while (true) {                                            // build_levels (builder.jl:359-384)
    LevelB& lev = levels.back();
    std::vector<int> which;
    for (int i = 0; i < lev.n(); ++i) if (lev.hi[i] - lev.lo[i] + 1 > ppl) which.push_back(i);
    if (which.empty()) break;
    if ((int)levels.size() >= max_levels)
      throw Error(1, "tree reached max_levels = " + std::to_string(max_levels) + "; more than ppl = " + std::to_string(ppl) + " coincident points?");
    levels.emplace_back();
    split_nodes(levels[levels.size() - 2], which, (int)levels.size() - 2, levels.back(), pts, perm, spts, sperm, origin, W0, false);
  }
  int L = (int)levels.size();
  tag_root(levels[0]);
  for (int l = 1; l < L; ++l) tag_colleagues(levels[l], levels[l - 1]);
  // level_restrict! (builder.jl:289-316)
  compute_depths(levels);
  while (true) {
    int nsplit = 0;
    for (int l = 1; l <= L - 3; ++l) {
      LevelB& lev = levels[l];
      std::vector<int> which;
      for (int i = 0; i < lev.n(); ++i) {
        if (!lev.leaf[i]) continue;
        for (int k = 0; k < NCOL; ++k) {
          int j = lev.col[(size_t)NCOL * i + k];
          if (j >= 0 && std::abs(lev.depth[i] - lev.depth[j]) > 1) { which.push_back(i); break; }
        }
      }
      if (which.empty()) continue;
      split_nodes(lev, which, l, levels[l + 1], pts, perm, spts, sperm, origin, W0, false);
      tag_colleagues(levels[l + 1], levels[l]);
      compute_depths(levels);
      nsplit += (int)which.size();
    }
    if (nsplit == 0) break;
  }
  // add_ghosts! (builder.jl:328-351)
  for (int l = 1; l <= L - 2; ++l) {
    LevelB& lev = levels[l];
    for (int i = 0; i < lev.n(); ++i) {
      if (!lev.leaf[i]) continue;
      for (int k = 0; k < NCOL; ++k) {
        int j = lev.col[(size_t)NCOL * i + k];
        if (j >= 0 && lev.cf[j] >= 0) { lev.xlist[i] = 1; break; }
      }
    }
  }
  for (int l = 1; l <= L - 2; ++l) {
    LevelB& lev = levels[l];
    std::vector<int> which;
    for (int i = 0; i < lev.n(); ++i) if (lev.xlist[i]) which.push_back(i);
    if (which.empty()) continue;
    split_nodes(lev, which, l, levels[l + 1], pts, perm, spts, sperm, origin, W0, true);
    tag_colleagues(levels[l + 1], levels[l]);
  }
  // flatten (builder.jl:392-473)
  Tree t;
  std::copy(origin, origin + 3, t.origin); t.W0 = W0; t.L = L; t.N = N;
  t.level_start.assign(L + 1, 0);
  for (int l = 0; l < L; ++l) t.level_start[l + 1] = t.level_start[l] + levels[l].n();
  int n = t.level_start[L]; t.n = n;
  t.cell.resize(3 * (size_t)n); t.level.resize(n); t.parent.resize(n); t.cf.resize(n); t.plo.resize(n); t.phi.resize(n);
  t.leaf.resize(n); t.ghost.resize(n); t.xlist.resize(n); t.has_source.resize(n); t.col.assign((size_t)NCOL * n, -1);
  t.point_node.assign(N, -1);
  for (int l = 0; l < L; ++l) {
    LevelB& lev = levels[l];
    int off = t.level_start[l];
    for (int i = 0; i < lev.n(); ++i) {
      int g = off + i;
      for (int d = 0; d < 3; ++d) t.cell[3 * g + d] = lev.cell[3 * i + d];
      t.level[g] = l;
      t.parent[g] = l == 0 ? -1 : t.level_start[l - 1] + lev.parent[i];
      t.cf[g] = lev.cf[i] < 0 ? -1 : t.level_start[l + 1] + lev.cf[i];
      t.plo[g] = lev.lo[i]; t.phi[g] = lev.hi[i];
      t.leaf[g] = lev.leaf[i]; t.ghost[g] = lev.ghost[i]; t.xlist[g] = lev.xlist[i];
      t.has_source[g] = lev.hi[i] >= lev.lo[i];
      for (int k = 0; k < NCOL; ++k) { int j = lev.col[(size_t)NCOL * i + k]; t.col[(size_t)NCOL * g + k] = j < 0 ? -1 : off + j; }
      if (lev.leaf[i]) for (int j = lev.lo[i]; j <= lev.hi[i]; ++j) t.point_node[j] = g;
    }
  }
  for (int j = 0; j < N; ++j) if (t.point_node[j] < 0) throw Error(4, "point not assigned to a leaf");
  t.perm = perm;
  // interaction lists by target in fill order (lists.jl:15-124)
  std::vector<int> fidx = far_index_table();
  t.ptr.resize(L); t.src.resize(L); t.far.resize(L);
  for (int l = 0; l < L; ++l) {
    int lo = t.level_start[l], nl = t.level_start[l + 1] - lo;
    std::vector<int>& ptr = t.ptr[l]; ptr.assign(nl + 1, 0);
    if (l < 2) continue;
    for (int q = 0; q < nl; ++q) {
      int i = lo + q;
      if (t.ghost[i]) { ptr[q + 1] = ptr[q]; continue; }
      int p = t.parent[i];
      const int* ci = &t.cell[3 * i];
      for (int k = 0; k < NCOL; ++k) {
        int cc = t.col[(size_t)NCOL * p + k];
        if (cc < 0) continue;
        int f0 = t.cf[cc];
        if (f0 < 0) continue;
        for (int s = f0; s < f0 + NCH; ++s) {
          if (!t.has_source[s]) continue;
          int o[3] = {t.cell[3 * s] - ci[0], t.cell[3 * s + 1] - ci[1], t.cell[3 * s + 2] - ci[2]};
          if (!is_far(o)) continue;
          t.src[l].push_back(s); t.far[l].push_back(fidx[table_index(o)]);
        }
      }
      ptr[q + 1] = (int)t.src[l].size();
    }
  }
  return t;
}

// ---------------------------------------------------------------- harmonics (src/operators/harmonics.jl)
// regular_hobson, irregular_hobson (harmonics.jl:37-76)
static std::vector<cplx> regular_hobson(const double* x, int p) {
  std::vector<cplx> Y((p + 1) * (p + 1));
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2], z = x[2];
  cplx xy(x[0], x[1]), s(1.0, 0.0);
  for (int m = 0; m <= p; ++m) {
    Y[cidx(m, m)] = s;
    cplx prev(0, 0), cur = s;
    for (int n = m + 1; n <= p; ++n) {
      cplx nxt = (((double)(2 * n - 1) * z) * cur - r2 * prev) / (double)((n - m) * (n + m));
      Y[cidx(n, m)] = nxt; prev = cur; cur = nxt;
    }
    s = (-xy / (double)(2 * (m + 1))) * s;
  }
  for (int n = 1; n <= p; ++n)
    for (int m = 1; m <= n; ++m) Y[cidx(n, -m)] = (m % 2 ? -1.0 : 1.0) * std::conj(Y[cidx(n, m)]);
  return Y;
}
static std::vector<cplx> irregular_hobson(const double* x, int p) {
  std::vector<cplx> Y((p + 1) * (p + 1));
  double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2], ir2 = 1.0 / r2, z = x[2];
  cplx xy(x[0], x[1]), s(1.0 / std::sqrt(r2), 0.0);
  for (int m = 0; m <= p; ++m) {
    Y[cidx(m, m)] = s;
    cplx prev(0, 0), cur = s;
    for (int n = m + 1; n <= p; ++n) {
      cplx nxt = (((double)(2 * n - 1) * z) * cur - (double)((n - 1) * (n - 1) - m * m) * prev) * ir2;
      Y[cidx(n, m)] = nxt; prev = cur; cur = nxt;
    }
    s = ((-(double)(2 * m + 1)) * xy * ir2) * s;
  }
  for (int n = 1; n <= p; ++n)
    for (int m = 1; m <= n; ++m) Y[cidx(n, -m)] = (m % 2 ? -1.0 : 1.0) * std::conj(Y[cidx(n, m)]);
  return Y;
}
static std::vector<double> scaling_factors(int p) {   // harmonics.jl:83-92
  std::vector<double> s((p + 1) * (p + 1));
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      double a = 1.0; int am = std::abs(m);
      for (int k = 2; k <= n - am; ++k) a *= k;
      for (int k = 2; k <= n + am; ++k) a *= k;
      s[cidx(n, m)] = std::sqrt(a);
    }
  return s;
}
// real_operator (harmonics.jl:124-148): column-major N × N output
static std::vector<double> real_operator(const std::vector<cplx>& A, int p) {
  int N = (p + 1) * (p + 1);
  std::vector<double> R((size_t)N * N, 0.0);
  std::vector<cplx> v(N);
  auto Acol = [&](int j) { return &A[(size_t)j * N]; };
  for (int n1 = 0; n1 <= p; ++n1)
    for (int m1 = 0; m1 <= n1; ++m1)
      for (int part = 0; part <= (m1 == 0 ? 0 : 1); ++part) {
        int j = m1 == 0 ? n1 * n1 : n1 * n1 + 2 * m1 - 1 + part;
        if (m1 == 0) { for (int i = 0; i < N; ++i) v[i] = Acol(cidx(n1, 0))[i]; }
        else {
          double sg = (m1 % 2) ? -1.0 : 1.0;
          const cplx* a = Acol(cidx(n1, m1)); const cplx* b = Acol(cidx(n1, -m1));
          if (part == 0) for (int i = 0; i < N; ++i) v[i] = a[i] + sg * b[i];
          else for (int i = 0; i < N; ++i) v[i] = cplx(0, 1) * (a[i] - sg * b[i]);
        }
        double* col = &R[(size_t)j * N];
        for (int n = 0; n <= p; ++n) {
          col[n * n] = v[cidx(n, 0)].real();
          for (int m = 1; m <= n; ++m) { col[rre(n, m)] = v[cidx(n, m)].real(); col[rim(n, m)] = v[cidx(n, m)].imag(); }
        }
      }
  return R;
}
// _harmonic_m2l (harmonics.jl:365-374)
static std::vector<double> harmonic_m2l(const int* o, int p, double c, const std::vector<double>& s) {
  int N = (p + 1) * (p + 1);
  double od[3] = {(double)o[0], (double)o[1], (double)o[2]};
  std::vector<cplx> Th = irregular_hobson(od, 2 * p);
  std::vector<cplx> A((size_t)N * N);
  for (int k = 0; k <= p; ++k)
    for (int l = -k; l <= k; ++l) {
      double sk = (k % 2 ? -1.0 : 1.0) * c / s[cidx(k, l)];
      for (int n = 0; n <= p; ++n)
        for (int mm = -n; mm <= n; ++mm)
          A[(size_t)cidx(k, l) * N + cidx(n, mm)] = sk * Th[cidx(n + k, mm + l)] / s[cidx(n, mm)];
    }
  return real_operator(A, p);
}

// symmetry classes of the harmonic basis (src/operators/symmetry.jl:14-34,252-319)
struct SignedPerm { int perm[3]; int sign[3]; };
static std::vector<SignedPerm> hyperoctahedral() {
  // permutations in the recursive order of `_permutations`, signs with coordinate 1 fastest
  int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  std::vector<SignedPerm> G;
  for (auto& pp : perms)
    for (int sidx = 0; sidx < 8; ++sidx) {
      SignedPerm R;
      for (int d = 0; d < 3; ++d) { R.perm[d] = pp[d]; R.sign[d] = ((sidx >> d) & 1) ? -1 : 1; }
      G.push_back(R);
    }
  return G;
}
struct Classes {
  std::vector<I3> reps;
  std::vector<int> cls;                         // per far offset
  std::vector<std::vector<int>> idx, idx_t;     // per far offset, source / target side
  std::vector<std::vector<int8_t>> sgn, sgn_t;
};
static void harmonic_permutation(int p, int k, bool ey, bool ez, bool target, std::vector<int>& idx, std::vector<int8_t>& sgn) {
  int N = (p + 1) * (p + 1);
  idx.assign(N, 0); sgn.assign(N, 1);
  for (int n = 0; n <= p; ++n) {
    int i0 = n * n;
    idx[i0] = i0; sgn[i0] = (ez && (n % 2)) ? -1 : 1;
    for (int m = 1; m <= n; ++m) {
      int ir = rre(n, m), ii = ir + 1;
      int q = (((target ? m * k : -m * k) % 4) + 4) % 4;
      int s = (ez && ((n + m) % 2)) ? -1 : 1;
      int sig = ey ? -1 : 1;
      if (q == 0) { idx[ir] = ir; sgn[ir] = s; idx[ii] = ii; sgn[ii] = s * sig; }
      else if (q == 1) { idx[ir] = ii; sgn[ir] = s; idx[ii] = ir; sgn[ii] = -s * sig; }
      else if (q == 2) { idx[ir] = ir; sgn[ir] = -s; idx[ii] = ii; sgn[ii] = -s * sig; }
      else { idx[ir] = ii; sgn[ir] = -s; idx[ii] = ir; sgn[ii] = s * sig; }
    }
  }
}
static Classes harmonic_symmetry_classes(int p) {
  std::vector<I3> offs = far_offsets();
  std::vector<SignedPerm> G;
  for (auto& R : hyperoctahedral()) if (R.perm[2] == 2) G.push_back(R);   // d4h_group
  Classes sc;
  for (auto& o : offs) {
    int a = std::abs(o.v[0]), b = std::abs(o.v[1]);
    I3 r; r.v[0] = std::max(a, b); r.v[1] = std::min(a, b); r.v[2] = std::abs(o.v[2]);
    int c = -1;
    for (size_t q = 0; q < sc.reps.size(); ++q)
      if (sc.reps[q].v[0] == r.v[0] && sc.reps[q].v[1] == r.v[1] && sc.reps[q].v[2] == r.v[2]) { c = (int)q; break; }
    if (c < 0) { sc.reps.push_back(r); c = (int)sc.reps.size() - 1; }
    sc.cls.push_back(c);
    const SignedPerm* g = nullptr;
    for (auto& R : G) {
      bool ok = true;
      for (int k = 0; k < 3; ++k) if (R.sign[k] * r.v[R.perm[k]] != o.v[k]) ok = false;
      if (ok) { g = &R; break; }
    }
    // _d4h_factors (symmetry.jl:256-267)
    bool ez = g->sign[2] == -1;
    int A[2][2] = {{0, 0}, {0, 0}};
    A[0][g->perm[0]] = g->sign[0]; A[1][g->perm[1]] = g->sign[1];
    bool ey = A[0][0] * A[1][1] - A[0][1] * A[1][0] == -1;
    if (ey) { A[0][1] = -A[0][1]; A[1][1] = -A[1][1]; }
    int rots[4][2][2] = {{{1, 0}, {0, 1}}, {{0, -1}, {1, 0}}, {{-1, 0}, {0, -1}}, {{0, 1}, {-1, 0}}};
    int k = -1;
    for (int q = 0; q < 4; ++q)
      if (rots[q][0][0] == A[0][0] && rots[q][0][1] == A[0][1] && rots[q][1][0] == A[1][0] && rots[q][1][1] == A[1][1]) k = q;
    if (k < 0) throw Error(4, "not a rotation");
    std::vector<int> is, it; std::vector<int8_t> ss, st;
    harmonic_permutation(p, k, ey, ez, false, is, ss);
    harmonic_permutation(p, k, ey, ez, true, it, st);
    sc.idx.push_back(is); sc.sgn.push_back(ss); sc.idx_t.push_back(it); sc.sgn_t.push_back(st);
  }
  return sc;
}

// the recurrence tables (harmonics.jl:172-188)
struct Tables { int p; std::vector<double> a, b, e, cz, cm, cp; };
static Tables harmonic_tables(int p) {
  Tables tb; tb.p = p;
  int nt = tidx(p, p) + 1;
  tb.a.assign(nt, 0); tb.b.assign(nt, 0); tb.cz.assign(nt, 0); tb.cm.assign(nt, 0); tb.cp.assign(nt, 0);
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      int t = tidx(n, m);
      double c = std::sqrt((double)((n - m) * (n + m)));
      tb.cz[t] = c;
      if (n > m) { tb.a[t] = (double)(2 * n - 1) / c; tb.b[t] = std::sqrt((double)((n - m - 1) * (n + m - 1))) / c; }
      tb.cm[t] = n + m >= 2 ? std::sqrt((double)((n + m) * (n + m - 1))) : 0.0;
      tb.cp[t] = n - m >= 2 ? std::sqrt((double)((n - m) * (n - m - 1))) : 0.0;
    }
  for (int m = 1; m <= p; ++m) tb.e.push_back(std::sqrt((double)(2 * m - 1) / (double)(2 * m)));
  return tb;
}
// _fold_regular (harmonics.jl:196-216)
template <class F>
static inline void fold_regular(F&& f, const double* xh, int nmax, const Tables& tb) {
  double x = xh[0], y = xh[1], z = xh[2];
  double r2 = x * x + y * y + z * z;
  double sr = 1.0, si = 0.0;
  for (int m = 0; m <= nmax; ++m) {
    f(m, m, sr, si);
    double pr = 0, pi = 0, cr = sr, ci = si;
    for (int n = m + 1; n <= nmax; ++n) {
      int t = tidx(n, m);
      double az = tb.a[t] * z, br = tb.b[t] * r2;
      double nr = az * cr - br * pr, ni = az * ci - br * pi;
      f(n, m, nr, ni);
      pr = cr; pi = ci; cr = nr; ci = ni;
    }
    if (m < nmax) {
      double e = tb.e[m];
      double nsr = -e * (x * sr - y * si), nsi = -e * (x * si + y * sr);
      sr = nsr; si = nsi;
    }
  }
}
static inline void get_coef(const double* L, int n, int m, double& re, double& im) {
  if (m > n) { re = 0; im = 0; }
  else if (m == 0) { re = L[n * n]; im = 0; }
  else { re = L[rre(n, m)]; im = L[rim(n, m)]; }
}

// ---------------------------------------------------------------- BLAS (optional OpenBLAS through dlopen)
typedef void (*cblas_dgemm_t)(int, int, int, i64, i64, i64, double, const double*, i64, const double*, i64, double, double*, i64);
static cblas_dgemm_t g_dgemm = nullptr;
static void (*g_blas_threads)(i64) = nullptr;
// C = alpha A B (column-major, A m×k, B k×n), beta = 0
static void dgemm(int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb, double* C, int ldc) {
  if (g_dgemm) { g_dgemm(102, 111, 111, m, n, k, alpha, A, lda, B, ldb, 0.0, C, ldc); return; }
  for (int j = 0; j < n; ++j) {
    double* c = C + (size_t)j * ldc;
    for (int i = 0; i < m; ++i) c[i] = 0;
    for (int q = 0; q < k; ++q) {
      double b = alpha * B[(size_t)j * ldb + q];
      const double* a = A + (size_t)q * lda;
      for (int i = 0; i < m; ++i) c[i] += a[i] * b;
    }
  }
}

// ---------------------------------------------------------------- the FMM (src/fmm.jl, src/evaluate.jl)
static const double KC = 1.0 / (4.0 * M_PI);   // Laplace3D c (src/kernels.jl:182)

// the operators of one box width (Yukawa3D: src/operators/harmonics_yukawa.jl:164-218)
struct LevelOps { std::vector<double> M2M, L2L; std::vector<std::vector<double>> reps; };

// the kernel of the harmonic method: Laplace3D (harmonics.jl), Yukawa3D (harmonics_yukawa.jl),
// Stokeslet3D through four Laplace expansions (harmonics_stokes.jl)
enum Kind { LAPLACE = 0, YUKAWA = 1, STOKES = 2 };

struct FMM {
  int p, NP;
  int kind = LAPLACE;
  int nb = 1;                                   // scalar expansions per node (4 for Stokes)
  double kappa = 0;                             // Yukawa3D's κ
  std::vector<LevelOps> yk;                     // Yukawa3D: the operators of each level's width
  Tree t;
  double W0ref;                                 // the operator cache's reference width
  std::vector<double> M2M, L2L;                 // NP × 8NP and 8NP × NP, column-major
  std::vector<std::vector<double>> reps;        // 34 × (NP × NP), column-major, c_K/W0ref folded in
  Classes sc;
  Tables tb;
  std::vector<double> scale, m2l_scale;         // per level: 1/w and the M2L factor
  std::vector<std::vector<int>> s2m_nodes, leaf_nodes;
  // per level: Morton target order (level-local) and the class lists
  std::vector<std::vector<int>> torder;
  // expansions, column-major NP × nnodes
  std::vector<double> Mp, Pl, Lc, xs, tau;
};

static void level_operators(FMM& f) {
  int p = f.p, N = f.NP;
  std::vector<double> s = scaling_factors(2 * p);
  f.M2M.assign((size_t)N * 8 * N, 0.0); f.L2L.assign((size_t)8 * N * N, 0.0);
  for (int k = 0; k < NCH; ++k) {
    I3 d = child_off(k);
    double dh[3] = {(d.v[0] - 0.5) / 2, (d.v[1] - 0.5) / 2, (d.v[2] - 0.5) / 2};
    std::vector<cplx> Y = regular_hobson(dh, p);
    std::vector<cplx> A((size_t)N * N), B((size_t)N * N);
    for (int n1 = 0; n1 <= p; ++n1)
      for (int m1 = -n1; m1 <= n1; ++m1)
        for (int n = n1; n <= p; ++n) {
          int dd = n - n1;
          for (int mm = std::max(-n, m1 - dd); mm <= std::min(n, m1 + dd); ++mm) {
            cplx v = std::conj(Y[cidx(dd, mm - m1)]) * (s[cidx(n, mm)] / s[cidx(n1, m1)]);
            A[(size_t)cidx(n1, m1) * N + cidx(n, mm)] = v * std::ldexp(1.0, -n1);
            B[(size_t)cidx(n, mm) * N + cidx(n1, m1)] = v * std::ldexp(1.0, -n1);
          }
        }
    std::vector<double> RA = real_operator(A, p), RB = real_operator(B, p);
    // M2M = [blocks...] (N × 8N): block k occupies columns kN..(k+1)N-1
    for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) f.M2M[(size_t)(k * N + j) * N + i] = RA[(size_t)j * N + i];
    // L2L = [blocks; ...] (8N × N): block k occupies rows kN..(k+1)N-1
    for (int j = 0; j < N; ++j) for (int i = 0; i < N; ++i) f.L2L[(size_t)j * 8 * N + k * N + i] = RB[(size_t)j * N + i];
  }
  double c = KC / f.W0ref;
  f.sc = harmonic_symmetry_classes(p);
  f.reps.clear();
  for (auto& r : f.sc.reps) f.reps.push_back(harmonic_m2l(r.v, p, c, s));
  f.tb = harmonic_tables(p);
}

// ---------------------------------------------------------------- Yukawa3D (src/operators/harmonics_yukawa.jl)
// u_n(z) from z², n = 0..nmax: Miller's backward recurrence u_n = u_{n+1} + z² u_{n+2}/((2n+3)(2n+5))
// from above max(nmax, z), normalised with u_0 = sinh z / z; two series terms for z² < 1e-8
// (harmonics_yukawa.jl:44-59; _radial_weights, :232-253, is the same recurrence)
static void yukawa_u(double z2, int nmax, double* u) {
  if (z2 < 1e-8) {
    for (int n = 0; n <= nmax; ++n) u[n] = 1 + z2 / (2 * (2 * n + 3));
    return;
  }
  double z = std::sqrt(z2);
  int N = std::max(nmax, (int)std::ceil(z)) + 25;
  double a = 0, b = 1;
  for (int n = N - 1; n >= 0; --n) {
    double c = b + z2 * a / (double)((2 * n + 3) * (2 * n + 5));
    if (n <= nmax) u[n] = c;
    a = b; b = c;
  }
  double s = (std::sinh(z) / z) / b;
  for (int n = 0; n <= nmax; ++n) u[n] *= s;
}
// v_n(z): v_0 = e^{−z}, v_1 = e^{−z}(1 + z), v_{n+1} = v_n + z² v_{n−1}/((2n−1)(2n+1)) (:61-73)
static void yukawa_v(double z, int nmax, double* v) {
  double e = std::exp(-z), z2 = z * z;
  v[0] = e;
  if (nmax >= 1) v[1] = e * (1 + z);
  for (int n = 1; n <= nmax - 1; ++n) v[n + 1] = v[n] + z2 * v[n - 1] / (double)((2 * n - 1) * (2 * n + 1));
}
static double norm3(const double* y) { return std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]); }

// the product rule on the unit sphere (:94-110): Gauss–Legendre nodes t (ascending) × 4p+20
// equispaced angles; the nodes and weights come from the caller (the Golub–Welsch eigenvalues)
struct SphereRule { std::vector<double> x, w; int nq; };
static SphereRule sphere_quadrature(int p, const double* gt, const double* gw, int nt) {
  SphereRule S;
  int nphi = 4 * p + 20;
  for (int i = 0; i < nt; ++i)
    for (int k = 0; k < nphi; ++k) {
      double phi = 2 * M_PI * k / nphi, s = std::sqrt(std::max(0.0, 1 - gt[i] * gt[i]));
      S.x.push_back(s * std::cos(phi)); S.x.push_back(s * std::sin(phi)); S.x.push_back(gt[i]);
      S.w.push_back(gw[i] * 2 * M_PI / nphi);
    }
  S.nq = nt * nphi;
  return S;
}
// u_n(κ̂|y|) [Υ̃_n^0 | 2 Re Υ̃ | 2 Im Υ̃](y) (:111-125) into b[0..N)
static void yukawa_regular(double* b, const double* y, double kh, int p, const Tables& tb) {
  std::vector<double> u(p + 1);
  double r = norm3(y);
  yukawa_u((kh * r) * (kh * r), p, u.data());
  fold_regular([&](int n, int m, double vr, double vi) {
    double w = u[n];
    if (m == 0) b[n * n] = w * vr;
    else { b[rre(n, m)] = 2 * w * vr; b[rim(n, m)] = 2 * w * vi; }
  }, y, p, tb);
}
// v_n(κ̂|y|) |y|^{−(2n+1)} [Υ̃_n^0 | 2 Re Υ̃ | −2 Im Υ̃](y) (:126-142)
static void yukawa_irregular(double* b, const double* y, double kh, int p, const Tables& tb) {
  std::vector<double> v(p + 1);
  double r = norm3(y);
  yukawa_v(kh * r, p, v.data());
  double ir = 1 / r;
  fold_regular([&](int n, int m, double vr, double vi) {
    double w = v[n] * std::pow(ir, 2 * n + 1);
    if (m == 0) b[n * n] = w * vr;
    else { b[rre(n, m)] = 2 * w * vr; b[rim(n, m)] = -2 * w * vi; }
  }, y, p, tb);
}
// the projection onto the regular or irregular basis on the sphere of radius ρ (:143-163):
// N × nq column-major
static std::vector<double> yukawa_projection(int p, double kh, double rho, bool irregular, const SphereRule& S, const Tables& tb) {
  int N = (p + 1) * (p + 1);
  std::vector<double> B((size_t)N * S.nq);
  for (int q = 0; q < S.nq; ++q) {
    double* col = &B[(size_t)q * N];
    fold_regular([&](int n, int m, double vr, double vi) {
      if (m == 0) col[n * n] = vr;
      else { col[rre(n, m)] = 2 * vr; col[rim(n, m)] = 2 * vi; }
    }, &S.x[3 * q], p, tb);
    for (int i = 0; i < N; ++i) col[i] *= S.w[q];
  }
  std::vector<double> rad(p + 1);
  if (irregular) yukawa_v(kh * rho, p, rad.data());
  else yukawa_u((kh * rho) * (kh * rho), p, rad.data());
  for (int n = 0; n <= p; ++n) {
    double f = irregular ? rad[n] * std::pow(rho, -n - 1) : rad[n] * std::pow(rho, n);
    double g0 = 4 * M_PI / (2 * n + 1);
    for (int i = n * n; i < (n + 1) * (n + 1); ++i) {
      int k = i - n * n + 1;                    // 1-based position in the degree's block
      double g = k == 1 ? g0 : 2 * g0;
      double sg = (irregular && k > 1 && (k & 1)) ? -1.0 : 1.0;
      double fac = sg / (g * f);
      for (int q = 0; q < S.nq; ++q) B[(size_t)q * N + i] *= fac;
    }
  }
  return B;
}
// the operators of one width in box coordinates, κ̂ = κ w, the M2L carrying c/w (:164-207):
// projection spheres of radius ½ about the target, 2 about the parent, 1 about the child
static LevelOps yukawa_operators(int p, double kh, double cw, const Classes& sc, const Tables& tb, const SphereRule& S) {
  int N = (p + 1) * (p + 1), nq = S.nq;
  std::vector<double> Preg = yukawa_projection(p, kh, 0.5, false, S, tb);
  std::vector<double> Pirr = yukawa_projection(p, kh, 2.0, true, S, tb);
  std::vector<double> Pregc = yukawa_projection(p, kh / 2, 1.0, false, S, tb);
  for (double& x : Preg) x *= cw;                // (cw * Preg) * transpose(F)
  std::vector<double> FT((size_t)nq * N), col(N);   // FT[i·nq + q] = F[i, q]
  auto fill = [&](auto&& body) {
    for (int q = 0; q < nq; ++q) {
      body(&S.x[3 * q], col.data());
      for (int i = 0; i < N; ++i) FT[(size_t)i * nq + q] = col[i];
    }
  };
  LevelOps ops;
  for (const I3& o : sc.reps) {
    fill([&](const double* x, double* c) {
      double y[3] = {0.5 * x[0] - o.v[0], 0.5 * x[1] - o.v[1], 0.5 * x[2] - o.v[2]};
      yukawa_irregular(c, y, kh, p, tb);
    });
    std::vector<double> R((size_t)N * N);
    dgemm(N, N, nq, 1.0, Preg.data(), N, FT.data(), nq, R.data(), N);
    ops.reps.push_back(R);
  }
  ops.M2M.assign((size_t)N * 8 * N, 0.0);
  ops.L2L.assign((size_t)8 * N * N, 0.0);
  for (int k = 0; k < NCH; ++k) {
    I3 d = child_off(k);
    double dh[3] = {(d.v[0] - 0.5) / 2, (d.v[1] - 0.5) / 2, (d.v[2] - 0.5) / 2};
    fill([&](const double* x, double* c) {
      double y[3] = {2 * (2.0 * x[0] - dh[0]), 2 * (2.0 * x[1] - dh[1]), 2 * (2.0 * x[2] - dh[2])};
      yukawa_irregular(c, y, kh / 2, p, tb);
      for (int i = 0; i < N; ++i) c[i] *= 2;
    });
    dgemm(N, N, nq, 1.0, Pirr.data(), N, FT.data(), nq, &ops.M2M[(size_t)k * N * N], N);
    fill([&](const double* x, double* c) {
      double y[3] = {dh[0] + 1.0 * x[0] / 2, dh[1] + 1.0 * x[1] / 2, dh[2] + 1.0 * x[2] / 2};
      yukawa_regular(c, y, kh, p, tb);
    });
    dgemm(N, N, nq, 1.0, Pregc.data(), N, FT.data(), nq, &ops.L2L[(size_t)k * N], 8 * N);
  }
  return ops;
}

// S2M of one childless node (harmonics.jl:425-434, 242-250)
static void s2m_node(FMM& f, int node, double* col) {
  const Tree& t = f.t;
  int l = t.level[node];
  double w = std::ldexp(t.W0, -l), c[3];
  cell_center(t.origin, &t.cell[3 * node], w, c);
  double s = f.scale[l];
  const int N = f.NP;
  for (int i = 0; i < f.nb * N; ++i) col[i] = 0;
  // M_n^m += w(n) τ conj Υ̃_n^m(x̂) (harmonics.jl:243-252); the weight is 1, or u_n(κ̂|x̂|) for Yukawa
  auto charge = [&](double* b, const double* xh, double tau, const double* wt) {
    fold_regular([&](int n, int m, double vr, double vi) {
      double tw = wt ? tau * wt[n] : tau;
      if (m == 0) b[n * n] += tw * vr;
      else { b[rre(n, m)] += tw * vr; b[rim(n, m)] += -tw * vi; }
    }, xh, f.p, f.tb);
  };
  std::vector<double> u(f.p + 2);
  double kh = f.kappa * w;
  for (int j = t.plo[node]; j <= t.phi[node]; ++j) {
    double xh[3] = {(f.xs[3 * j] - c[0]) * s, (f.xs[3 * j + 1] - c[1]) * s, (f.xs[3 * j + 2] - c[2]) * s};
    if (f.kind == LAPLACE) {
      charge(col, xh, f.tau[j], nullptr);
    } else if (f.kind == YUKAWA) {                 // harmonics_yukawa.jl:290-302
      yukawa_u(kh * kh * ((xh[0] * xh[0] + xh[1] * xh[1]) + xh[2] * xh[2]), f.p + 1, u.data());
      charge(col, xh, f.tau[j], u.data());
    } else {                                       // the four blocks of a Stokeslet (harmonics_stokes.jl:197-204)
      const double* fk = &f.tau[3 * j];
      for (int k = 0; k < 3; ++k) charge(col + k * N, xh, fk[k], nullptr);
      charge(col + 3 * N, xh, (xh[0] * fk[0] + xh[1] * fk[1]) + xh[2] * fk[2], nullptr);
    }
  }
}

static void upward(FMM& f) {   // fmm.jl:170-205
  const Tree& t = f.t;
  int N = f.NP, L = t.L, NB = f.nb * N;
  std::fill(f.Mp.begin(), f.Mp.end(), 0.0);
  for (int l = L - 1; l >= 2; --l) {
    const std::vector<int>& nodes = f.s2m_nodes[l];
#pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < (int)nodes.size(); ++q) s2m_node(f, nodes[q], &f.Mp[(size_t)nodes[q] * NB]);
    if (l < L - 1) {
      int c0 = t.level_start[l + 1], ng = (t.level_start[l + 2] - c0) / NCH;
      std::vector<double> tmp((size_t)NB * ng);
      // the parent level's operator (Yukawa: its width's; harmonics_yukawa.jl:209-218)
      const double* M2M = f.kind == YUKAWA ? f.yk[l].M2M.data() : f.M2M.data();
      int nth = omp_get_max_threads();
#pragma omp parallel for schedule(static)
      for (int ch = 0; ch < nth; ++ch) {
        int g0 = (int)((i64)ch * ng / nth), g1 = (int)((i64)(ch + 1) * ng / nth);
        if (g1 <= g0) continue;
        if (f.kind != STOKES) {
          dgemm(N, g1 - g0, 8 * N, 1.0, M2M, N, &f.Mp[(size_t)(c0 + NCH * g0) * N], 8 * N, &tmp[(size_t)g0 * N], N);
          continue;
        }
        // Stokes (harmonics_stokes.jl:157-179): block a of the parent is M2M on the children's
        // block a stacked; the fourth with the coupling folded in, ½Ψ̂ + δ̂·Φ
        int nc = g1 - g0;
        std::vector<double> X((size_t)8 * N * nc), R((size_t)N * nc);
        for (int a = 0; a < 4; ++a) {
          for (int g = 0; g < nc; ++g)
            for (int j = 0; j < NCH; ++j) {
              const double* B = &f.Mp[(size_t)(c0 + NCH * (g0 + g) + j) * NB];
              double* x = &X[(size_t)g * 8 * N + (size_t)j * N];
              I3 d = child_off(j);
              double dh[3] = {(d.v[0] - 0.5) / 2, (d.v[1] - 0.5) / 2, (d.v[2] - 0.5) / 2};
              for (int i = 0; i < N; ++i)
                x[i] = a < 3 ? B[a * N + i] : B[3 * N + i] / 2 + dh[0] * B[i] + dh[1] * B[N + i] + dh[2] * B[2 * N + i];
            }
          dgemm(N, nc, 8 * N, 1.0, M2M, N, X.data(), 8 * N, R.data(), N);
          for (int g = 0; g < nc; ++g) std::copy(&R[(size_t)g * N], &R[(size_t)(g + 1) * N], &tmp[(size_t)(g0 + g) * NB + a * N]);
        }
      }
      for (int g = 0; g < ng; ++g) {
        int par = t.parent[c0 + NCH * g];
        std::copy(&tmp[(size_t)g * NB], &tmp[(size_t)(g + 1) * NB], &f.Mp[(size_t)par * NB]);
      }
    }
  }
}

static void m2l_level(FMM& f, int l) {   // harmonics.jl:531-645, symmetry.jl:207-240
  const Tree& t = f.t;
  int N = f.NP, lo = t.level_start[l], nb = f.nb, NB = nb * N;
  const std::vector<int>& ptr = t.ptr[l]; const std::vector<int>& src = t.src[l]; const std::vector<int>& far = t.far[l];
  const std::vector<int>& ord = f.torder[l];
  int nt = (int)ord.size();
  if (nt == 0) return;
  // Laplace and Stokes: the reference width's representatives and the level's factor;
  // Yukawa: the level width's representatives (harmonics_yukawa.jl:209-218)
  const std::vector<std::vector<double>>& reps = f.kind == YUKAWA ? f.yk[l].reps : f.reps;
  int nclass = (int)reps.size();
  const int TB = 32;                              // _TARGET_BLOCK
  int nblocks = (nt + TB - 1) / TB;
  double alpha = f.kind == YUKAWA ? 1.0 : f.m2l_scale[l];
  static const std::vector<I3> offs = far_offsets();
#pragma omp parallel
  {
    std::vector<double> G((size_t)N * 512 * nb), R((size_t)N * 512 * nb);
    std::vector<int> qs; qs.reserve(512);
    std::vector<int> qt; qt.reserve(512);
#pragma omp for schedule(dynamic, 1)
    for (int b = 0; b < nblocks; ++b) {
      int g1 = b * TB, g2 = std::min(nt, g1 + TB);
      for (int c = 0; c < nclass; ++c) {
        qs.clear(); qt.clear();
        for (int g = g1; g < g2; ++g) {
          int q = ord[g];
          for (int e = ptr[q]; e < ptr[q + 1]; ++e) if (f.sc.cls[far[e]] == c) { qs.push_back(e); qt.push_back(lo + q); }
        }
        int nc = (int)qs.size();
        if (nc == 0) continue;
        if ((size_t)nc * nb * N > G.size()) { G.resize((size_t)nc * nb * N); R.resize((size_t)nc * nb * N); }
        // one column per pair and scalar expansion, the blocks of a pair consecutive (_gather_column!)
        for (int j = 0; j < nc; ++j) {
          int e = qs[j], fo = far[e];
          const int* idx = f.sc.idx[fo].data(); const int8_t* sg = f.sc.sgn[fo].data();
          for (int a = 0; a < nb; ++a) {
            const double* m = &f.Mp[(size_t)src[e] * NB + (size_t)a * N];
            double* gcol = &G[(size_t)(j * nb + a) * N];
            for (int i = 0; i < N; ++i) gcol[i] = sg[i] * m[idx[i]];
          }
        }
        dgemm(N, nc * nb, N, alpha, reps[c].data(), N, G.data(), N, R.data(), N);
        // _scatter_target!: the target permutation, and for Stokes Ψ̂ += o·Φ with the pair's offset
        for (int j = 0; j < nc; ++j) {
          int fo = far[qs[j]];
          const int* it = f.sc.idx_t[fo].data(); const int8_t* st = f.sc.sgn_t[fo].data();
          for (int a = 0; a < nb; ++a) {
            double* pl = &f.Pl[(size_t)qt[j] * NB + (size_t)a * N];
            const double* r = &R[(size_t)(j * nb + a) * N];
            if (nb == 4 && a == 3) {
              const double *r1 = &R[(size_t)(j * nb) * N], *r2 = r1 + N, *r3 = r2 + N;
              const I3& o = offs[fo];
              for (int i = 0; i < N; ++i) pl[it[i]] += st[i] * (r[i] + o.v[0] * r1[i] + o.v[1] * r2[i] + o.v[2] * r3[i]);
            } else {
              for (int i = 0; i < N; ++i) pl[it[i]] += st[i] * r[i];
            }
          }
        }
      }
    }
  }
}

static void downward(FMM& f) {   // fmm.jl:207-262
  const Tree& t = f.t;
  int N = f.NP, L = t.L, NB = f.nb * N;
  std::fill(f.Pl.begin(), f.Pl.end(), 0.0);
  std::fill(f.Lc.begin(), f.Lc.end(), 0.0);
  for (int l = 2; l < L; ++l) {
    int lo = t.level_start[l], nl = t.level_start[l + 1] - lo;
    if (l > 2) {
      int ng = nl / NCH;
      std::vector<double> G((size_t)NB * ng);
      for (int g = 0; g < ng; ++g) {
        int par = t.parent[lo + NCH * g];
        std::copy(&f.Pl[(size_t)par * NB], &f.Pl[(size_t)(par + 1) * NB], &G[(size_t)g * NB]);
      }
      // the parent level's operator (Yukawa: its width's)
      const double* L2L = f.kind == YUKAWA ? f.yk[l - 1].L2L.data() : f.L2L.data();
      int nth = omp_get_max_threads();
#pragma omp parallel for schedule(static)
      for (int ch = 0; ch < nth; ++ch) {
        int g0 = (int)((i64)ch * ng / nth), g1 = (int)((i64)(ch + 1) * ng / nth);
        if (g1 <= g0) continue;
        if (f.kind != STOKES) {
          dgemm(8 * N, g1 - g0, N, 1.0, L2L, 8 * N, &G[(size_t)g0 * N], N, &f.Pl[(size_t)(lo + NCH * g0) * N], 8 * N);
          continue;
        }
        // Stokes (harmonics_stokes.jl:180-203): R_a = L2L · G_a per block; child blocks 1-3 are
        // R_a, the fourth 2·R_4 − 2 δ̂·(R_1, R_2, R_3)
        int nc = g1 - g0;
        std::vector<double> X((size_t)N * nc), R((size_t)4 * 8 * N * nc);
        for (int a = 0; a < 4; ++a) {
          for (int g = 0; g < nc; ++g) std::copy(&G[(size_t)(g0 + g) * NB + a * N], &G[(size_t)(g0 + g) * NB + (a + 1) * N], &X[(size_t)g * N]);
          dgemm(8 * N, nc, N, 1.0, L2L, 8 * N, X.data(), N, &R[(size_t)a * 8 * N * nc], 8 * N);
        }
        for (int g = 0; g < nc; ++g)
          for (int j = 0; j < NCH; ++j) {
            I3 d = child_off(j);
            double dh[3] = {(d.v[0] - 0.5) / 2, (d.v[1] - 0.5) / 2, (d.v[2] - 0.5) / 2};
            double* out = &f.Pl[(size_t)(lo + NCH * (g0 + g) + j) * NB];
            for (int i = 0; i < N; ++i) {
              size_t x0 = (size_t)g * 8 * N + (size_t)j * N + i, bs = (size_t)8 * N * nc;
              double r1 = R[x0], r2 = R[bs + x0], r3 = R[2 * bs + x0];
              out[i] = r1; out[N + i] = r2; out[2 * N + i] = r3;
              out[3 * N + i] = 2 * R[3 * bs + x0] - 2 * (dh[0] * r1 + dh[1] * r2 + dh[2] * r3);
            }
          }
      }
    }
    m2l_level(f, l);
    for (int i : f.leaf_nodes[l]) std::copy(&f.Pl[(size_t)i * NB], &f.Pl[(size_t)(i + 1) * NB], &f.Lc[(size_t)i * NB]);
  }
}

// evaluate_target (evaluate.jl:33-48) for potential and gradient at once; skip = tree index or -1.
// Laplace3D (harmonics.jl:447-486) and Yukawa3D, whose far field weighs degree n by u_n(κ̂|x̂|) and
// adds x̂ times the potential weighted by κ̂² u_{n+1}/(2n+3) to the gradient (harmonics_yukawa.jl:304-317)
static void evaluate_target(const FMM& f, const double* x, int i, int skip, double* pot, double* grad) {
  const Tree& t = f.t;
  int l = t.level[i];
  double w = std::ldexp(t.W0, -l), c[3];
  cell_center(t.origin, &t.cell[3 * i], w, c);
  double s = f.scale[l];
  double xh[3] = {(x[0] - c[0]) * s, (x[1] - c[1]) * s, (x[2] - c[2]) * s};
  const double* Lc = &f.Lc[(size_t)i * f.NP];
  const bool yk = f.kind == YUKAWA;
  double kh = f.kappa * w, kh2 = kh * kh, r2h = (xh[0] * xh[0] + xh[1] * xh[1]) + xh[2] * xh[2];
  std::vector<double> up(f.p + 2), ug(f.p + 2);
  if (yk) { yukawa_u(kh * kh * r2h, f.p, up.data()); yukawa_u(kh * kh * r2h, f.p + 1, ug.data()); }
  // Σ w(n) L conj Υ̃ (_harmonic_potential) with the weights wt (null: 1) or the radial ones
  auto potential = [&](const double* wt, bool radial) {
    double u = 0;
    fold_regular([&](int n, int m, double vr, double vi) {
      double lr, li; get_coef(Lc, n, m, lr, li);
      double wn = radial ? kh2 * wt[n + 1] / (2 * n + 3) : (wt ? wt[n] : 1.0);
      if (!wt) u = m == 0 ? u + lr * vr : u + 2 * (lr * vr + li * vi);
      else u = m == 0 ? u + wn * (lr * vr) : u + wn * (2 * (lr * vr + li * vi));
    }, xh, f.p, f.tb);
    return u;
  };
  double u = potential(yk ? up.data() : nullptr, false);
  double gx = 0, gy = 0, gz = 0;
  const Tables& tb = f.tb;
  fold_regular([&](int n1, int m1, double vr, double vi) {
    int n = n1 + 1;
    double wn = yk ? ug[n] : 1.0;
    if (m1 == 0) {
      double lr, li; get_coef(Lc, n, 1, lr, li);
      double cc = tb.cm[tidx(n, 1)];
      double ax = -cc * lr, ay = -cc * li, az = tb.cz[tidx(n, 0)] * Lc[n * n];
      if (yk) { gx += wn * (ax * vr); gy += wn * (ay * vr); gz += wn * (az * vr); }
      else { gx += ax * vr; gy += ay * vr; gz += az * vr; }
    } else {
      double ur, ui, dr, di, zr, zi;
      get_coef(Lc, n, m1 + 1, ur, ui); get_coef(Lc, n, m1 - 1, dr, di);
      double cu = tb.cm[tidx(n, m1 + 1)] / 2, cd = tb.cp[tidx(n, m1 - 1)] / 2;
      double axr = -cu * ur + cd * dr, axi = -cu * ui + cd * di;
      double ayr = -(cu * ui + cd * di), ayi = cu * ur + cd * dr;
      double czv = tb.cz[tidx(n, m1)];
      get_coef(Lc, n, m1, zr, zi);
      double w2 = 2 * wn;
      gx += w2 * (axr * vr + axi * vi); gy += w2 * (ayr * vr + ayi * vi); gz += w2 * (czv * (zr * vr + zi * vi));
    }
  }, xh, f.p - 1, tb);
  if (yk) {
    double pr = potential(ug.data(), true);
    gx += xh[0] * pr; gy += xh[1] * pr; gz += xh[2] * pr;
  }
  gx *= s; gy *= s; gz *= s;
  // near field over the 27 colleagues, the excluded source masked (evaluate.jl:12-25, kernels.jl:179-193;
  // Yukawa: the radial kernel c e^{−κr}/r and its gradient (c f′/r) d, kernels.jl:33-41,228-242)
  for (int k = 0; k < NCOL; ++k) {
    int cn = t.col[(size_t)NCOL * i + k];
    if (cn < 0) continue;
    for (int j = t.plo[cn]; j <= t.phi[cn]; ++j) {
      if (j == skip) continue;
      double d0 = x[0] - f.xs[3 * j], d1 = x[1] - f.xs[3 * j + 1], d2 = x[2] - f.xs[3 * j + 2];
      double r2 = std::fma(d2, d2, std::fma(d1, d1, d0 * d0));
      double tj = f.tau[j];
      if (yk) {
        double r = std::sqrt(r2), ir = 1 / r, e = std::exp(-f.kappa * r);
        u += (KC * (e * ir)) * tj;
        double fp = -e * (f.kappa * ir + ir * ir);
        double a = KC * fp / r;
        gx += (a * d0) * tj; gy += (a * d1) * tj; gz += (a * d2) * tj;
        continue;
      }
      double ir = 1.0 / std::sqrt(r2);
      u += (KC * ir) * tj;
      double a = -KC * ir * ir * ir;
      gx += (a * d0) * tj; gy += (a * d1) * tj; gz += (a * d2) * tj;
    }
  }
  *pot = u; grad[0] = gx; grad[1] = gy; grad[2] = gz;
}

// ---------------------------------------------------------------- Stokes outputs (harmonics_stokes.jl:236-343)
// the (n, m) coefficient of block `o` as a complex number, zero outside the triangle; negative m
// by conjugate symmetry (_cget)
static cplx cget(const double* L, int p, int n, int m) {
  if (n > p || std::abs(m) > n) return cplx(0, 0);
  if (m == 0) return cplx(L[n * n], 0);
  if (m > 0) return cplx(L[rre(n, m)], L[rim(n, m)]);
  return (double)((-m) % 2 == 0 ? 1 : -1) * cplx(L[rre(n, -m)], -L[rim(n, -m)]);
}
static double tcz(const Tables& tb, int n, int m) { return std::abs(m) > n ? 0.0 : tb.cz[tidx(n, std::abs(m))]; }
static double tcm(const Tables& tb, int n, int m) { return std::abs(m) > n ? 0.0 : m >= 0 ? tb.cm[tidx(n, m)] : tb.cp[tidx(n, -m)]; }
static double tcp(const Tables& tb, int n, int m) { return std::abs(m) > n ? 0.0 : m >= 0 ? tb.cp[tidx(n, m)] : tb.cm[tidx(n, -m)]; }
// the (n′, m′) coefficients of the scaled gradient of one block (_dcoef)
static void dcoef(const double* L, int p, const Tables& tb, int n1, int m1, cplx* a) {
  int n = n1 + 1;
  cplx dm = -tcm(tb, n, m1 + 1) * cget(L, p, n, m1 + 1);
  cplx dp = tcp(tb, n, m1 - 1) * cget(L, p, n, m1 - 1);
  cplx dz = tcz(tb, n, m1) * cget(L, p, n, m1);
  a[0] = (dm + dp) / 2.0; a[1] = cplx(0, 1) * (dp - dm) / 2.0; a[2] = dz;
}
static double re_conj(cplx c, cplx v) { return (c * std::conj(v)).real(); }

// velocity ½[Φ − x̂·∇̂Φ + ∇̂Ψ̂] and pressure −s·tr ∇̂Φ of the leaf's four local expansions
// (_stokes_fold1, _stokes_output), plus the Stokeslet near field c[f/r + d(d·f)/r³] and its
// pressure 2c(d·f)/r³ (kernels.jl:253-272); skip = tree index or -1
static void stokes_evaluate_target(const FMM& f, const double* x, int i, int skip, double* vel, double* pres) {
  const Tree& t = f.t;
  int l = t.level[i], N = f.NP, p = f.p;
  double w = std::ldexp(t.W0, -l), c[3];
  cell_center(t.origin, &t.cell[3 * i], w, c);
  double s = f.scale[l];
  double xh[3] = {(x[0] - c[0]) * s, (x[1] - c[1]) * s, (x[2] - c[2]) * s};
  const double* Lc = &f.Lc[(size_t)i * 4 * N];
  double Phi[3] = {0, 0, 0}, G[3][3] = {{0}}, gP[3] = {0, 0, 0};   // G[i][k] = ∂̂_iΦ_k
  fold_regular([&](int n, int m, double vr, double vi) {
    cplx v(vr, vi);
    double wt = m == 0 ? 1 : 2;
    for (int k = 0; k < 3; ++k) Phi[k] += wt * re_conj(cget(Lc + k * N, p, n, m), v);
    if (n < p) {
      cplx a[3];
      for (int k = 0; k < 3; ++k) {
        dcoef(Lc + k * N, p, f.tb, n, m, a);
        for (int d = 0; d < 3; ++d) G[d][k] += wt * re_conj(a[d], v);
      }
      dcoef(Lc + 3 * N, p, f.tb, n, m, a);
      for (int d = 0; d < 3; ++d) gP[d] += wt * re_conj(a[d], v);
    }
  }, xh, p, f.tb);
  double u[3], pr = -s * ((G[0][0] + G[1][1]) + G[2][2]);
  for (int d = 0; d < 3; ++d) u[d] = (Phi[d] - ((G[d][0] * xh[0] + G[d][1] * xh[1]) + G[d][2] * xh[2]) + gP[d]) / 2;
  const double KS = 1.0 / (8.0 * M_PI);
  for (int k = 0; k < NCOL; ++k) {
    int cn = t.col[(size_t)NCOL * i + k];
    if (cn < 0) continue;
    for (int j = t.plo[cn]; j <= t.phi[cn]; ++j) {
      if (j == skip) continue;
      double d[3] = {x[0] - f.xs[3 * j], x[1] - f.xs[3 * j + 1], x[2] - f.xs[3 * j + 2]};
      double r2 = std::fma(d[2], d[2], std::fma(d[1], d[1], d[0] * d[0]));
      double ir = 1.0 / std::sqrt(r2);
      double a = KS * ir, b = a * ir * ir;
      const double* fj = &f.tau[3 * j];
      double df = (d[0] * fj[0] + d[1] * fj[1]) + d[2] * fj[2];
      for (int e = 0; e < 3; ++e) u[e] += a * fj[e] + b * d[e] * df;
      pr += (2 * KS * ir * ir * ir) * df;
    }
  }
  if (vel) { vel[0] = u[0]; vel[1] = u[1]; vel[2] = u[2]; }
  if (pres) *pres = pr;
}

static int locate(const Tree& t, const double* x) {   // locate.jl:10-22
  for (int d = 0; d < 3; ++d) if (!(t.origin[d] <= x[d] && x[d] <= t.origin[d] + t.W0)) throw Error(1, "point lies outside the tree's box");
  int i = 0;
  while (!t.leaf[i]) {
    double c[3]; cell_center(t.origin, &t.cell[3 * i], std::ldexp(t.W0, -t.level[i]), c);
    i = t.cf[i] + child_slot(x, c);
  }
  return i;
}

// kind: LAPLACE, YUKAWA (κ = kappa; gt/gw: the Gauss–Legendre rule of 2p+10 points) or STOKES
static FMM* make_fmm(int p, const double* xyz, int N, int ppl, const double* origin, double W0, int max_levels, double W0ref,
                     int kind = LAPLACE, double kappa = 0, const double* gt = nullptr, const double* gw = nullptr, int ngl = 0) {
  FMM* f = new FMM();
  try {
    f->p = p; f->NP = (p + 1) * (p + 1);
    f->kind = kind; f->kappa = kappa; f->nb = kind == STOKES ? 4 : 1;
    f->t = build_tree(xyz, N, ppl, origin, W0, max_levels);
    f->W0ref = W0ref > 0 ? W0ref : W0;
    level_operators(*f);
    const Tree& t = f->t;
    int L = t.L;
    if (kind == YUKAWA) {
      if (ngl != 2 * p + 10) throw Error(1, "the Yukawa sphere rule needs 2p+10 Gauss-Legendre nodes");
      SphereRule S = sphere_quadrature(p, gt, gw, ngl);
      f->yk.resize(L);
      for (int l = 2; l < L; ++l) {
        double w = std::ldexp(t.W0, -l);
        f->yk[l] = yukawa_operators(p, kappa * w, KC / w, f->sc, f->tb, S);
      }
    }
    f->scale.resize(L); f->m2l_scale.resize(L);
    for (int l = 0; l < L; ++l) {
      double w = std::ldexp(t.W0, -l), lam = w / f->W0ref;
      f->scale[l] = (1.0 / f->W0ref) / lam;       // _rescaled (harmonics.jl:362)
      if (kind == YUKAWA) f->scale[l] = 1 / w;      // built per width (harmonics_yukawa.jl:209-218)
      f->m2l_scale[l] = 1.0 / lam;                 // rescale (harmonics.jl:414-418)
    }
    f->s2m_nodes.resize(L); f->leaf_nodes.resize(L); f->torder.resize(L);
    for (int l = 0; l < L; ++l) {
      for (int i = t.level_start[l]; i < t.level_start[l + 1]; ++i) {
        if (t.cf[i] < 0 && t.has_source[i]) f->s2m_nodes[l].push_back(i);
        if (t.leaf[i]) f->leaf_nodes[l].push_back(i);
      }
      // targets with pairs in Morton order of their cells (lists.jl:50-66)
      int lo = t.level_start[l], nl = t.level_start[l + 1] - lo;
      std::vector<std::pair<uint64_t, int>> ks;
      int nbits = std::min(l, 21);
      for (int q = 0; q < nl; ++q) if (t.ptr[l][q + 1] > t.ptr[l][q]) ks.push_back({morton_key(&t.cell[3 * (lo + q)], nbits), q});
      std::stable_sort(ks.begin(), ks.end(), [](const std::pair<uint64_t, int>& a, const std::pair<uint64_t, int>& b) { return a.first < b.first; });
      for (auto& kq : ks) f->torder[l].push_back(kq.second);
    }
    size_t ne = (size_t)f->nb * f->NP * t.n;
    f->Mp.assign(ne, 0.0); f->Pl.assign(ne, 0.0); f->Lc.assign(ne, 0.0);
    f->xs.resize(3 * (size_t)N); f->tau.resize((kind == STOKES ? 3 : 1) * (size_t)N);
  } catch (...) { delete f; throw; }
  return f;
}

}  // namespace orc

// ---------------------------------------------------------------- C API (for ctypes)
using namespace orc;
static thread_local std::string g_err;
#define GUARD(...) try { __VA_ARGS__ } catch (Error & e) { g_err = e.what(); return e.code; } catch (std::exception & e) { g_err = e.what(); return 4; }

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_set_blas(const char* path, int threads) {
  if (path && *path) {
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) { g_err = dlerror(); return 1; }
    g_dgemm = (cblas_dgemm_t)dlsym(h, "scipy_cblas_dgemm64_");
    g_blas_threads = (void (*)(i64))dlsym(h, "scipy_openblas_set_num_threads64_");
    if (!g_dgemm) { g_err = "no scipy_cblas_dgemm64_ in the BLAS library"; return 1; }
    if (g_blas_threads) g_blas_threads(1);       // one BLAS thread per task (harmonics.jl:543-545)
  } else { g_dgemm = nullptr; }
  if (threads > 0) omp_set_num_threads(threads);
  return 0;
}
int orc_num_threads() { return omp_get_max_threads(); }

// ---- tree
int orc_tree_build(const double* xyz, i64 n, int ppl, const double* origin, double W0, int max_levels, void** out) {
  GUARD({ *out = new Tree(build_tree(xyz, (int)n, ppl, origin, W0, max_levels)); return 0; })
}
void orc_tree_free(void* h) { delete (Tree*)h; }
// info: [L, nnodes, N, level_start[0..L]]
void orc_tree_info(void* h, i64* info) {
  Tree* t = (Tree*)h; info[0] = t->L; info[1] = t->n; info[2] = t->N;
  for (int l = 0; l <= t->L; ++l) info[3 + l] = t->level_start[l];
}
void orc_tree_get(void* h, int32_t* cell, int32_t* level, int32_t* parent, int32_t* cf, int32_t* plo, int32_t* phi,
                  uint8_t* leaf, uint8_t* ghost, uint8_t* xlist, uint8_t* has_source, int32_t* col, int32_t* perm, int32_t* point_node) {
  Tree* t = (Tree*)h;
  std::copy(t->cell.begin(), t->cell.end(), cell); std::copy(t->level.begin(), t->level.end(), level);
  std::copy(t->parent.begin(), t->parent.end(), parent); std::copy(t->cf.begin(), t->cf.end(), cf);
  std::copy(t->plo.begin(), t->plo.end(), plo); std::copy(t->phi.begin(), t->phi.end(), phi);
  std::copy(t->leaf.begin(), t->leaf.end(), leaf); std::copy(t->ghost.begin(), t->ghost.end(), ghost);
  std::copy(t->xlist.begin(), t->xlist.end(), xlist); std::copy(t->has_source.begin(), t->has_source.end(), has_source);
  std::copy(t->col.begin(), t->col.end(), col); std::copy(t->perm.begin(), t->perm.end(), perm);
  std::copy(t->point_node.begin(), t->point_node.end(), point_node);
}
i64 orc_tree_npairs(void* h, int l) { Tree* t = (Tree*)h; return (i64)t->src[l].size(); }
// pairs of a level as (target node, source node, far index), in fill order
void orc_tree_pairs(void* h, int l, int32_t* tgt, int32_t* src, int32_t* far) {
  Tree* t = (Tree*)h;
  int lo = t->level_start[l], nl = t->level_start[l + 1] - lo;
  for (int q = 0; q < nl; ++q)
    for (int e = t->ptr[l][q]; e < t->ptr[l][q + 1]; ++e) { tgt[e] = lo + q; src[e] = t->src[l][e]; far[e] = t->far[l][e]; }
}

// ---- the FMM
int orc_fmm_create(int p, const double* xyz, i64 n, int ppl, const double* origin, double W0, int max_levels, double W0ref, void** out) {
  GUARD({ *out = make_fmm(p, xyz, (int)n, ppl, origin, W0, max_levels, W0ref); return 0; })
}
// the harmonic method of another kernel: kind 1 Yukawa3D(κ) (gt/gw: the Gauss–Legendre rule of
// 2p+10 points on [−1, 1], ascending), kind 2 Stokeslet3D (four expansions per node)
int orc_fmm_create_kind(int kind, int p, double kappa, const double* gt, const double* gw, int ngl, const double* xyz, i64 n,
                        int ppl, const double* origin, double W0, int max_levels, double W0ref, void** out) {
  GUARD({ *out = make_fmm(p, xyz, (int)n, ppl, origin, W0, max_levels, W0ref, kind, kappa, gt, gw, ngl); return 0; })
}
void orc_fmm_free(void* h) { delete (FMM*)h; }
void* orc_fmm_tree(void* h) { return &((FMM*)h)->t; }
// build_expansions! (fmm.jl:271-298): inputs in the original order
int orc_fmm_build(void* h, const double* xyz, const double* tau) {
  FMM& f = *(FMM*)h;
  GUARD({
    for (int k = 0; k < f.t.N; ++k) {
      int j = f.t.perm[k];
      f.xs[3 * k] = xyz[3 * j]; f.xs[3 * k + 1] = xyz[3 * j + 1]; f.xs[3 * k + 2] = xyz[3 * j + 2];
      if (f.kind == STOKES) for (int d = 0; d < 3; ++d) f.tau[3 * k + d] = tau[3 * j + d];
      else f.tau[k] = tau[j];
    }
    upward(f); downward(f); return 0;
  })
}
int orc_fmm_upward(void* h) { FMM& f = *(FMM*)h; upward(f); return 0; }
// evaluate_at_sources! (evaluate.jl:111-127): outputs in the original order
int orc_fmm_eval_sources(void* h, double* pot, double* grad) {
  FMM& f = *(FMM*)h;
  if (f.kind == STOKES) { g_err = "a Stokes FMM: use the Stokes outputs"; return 1; }
  int N = f.t.N;
#pragma omp parallel for schedule(dynamic, 256)
  for (int k = 0; k < N; ++k) {
    double u, g[3];
    evaluate_target(f, &f.xs[3 * k], f.t.point_node[k], k, &u, g);
    int j = f.t.perm[k];
    if (pot) pot[j] = u;
    if (grad) { grad[3 * j] = g[0]; grad[3 * j + 1] = g[1]; grad[3 * j + 2] = g[2]; }
  }
  return 0;
}
// evaluate! (evaluate.jl:81-96)
int orc_fmm_eval_targets(void* h, const double* tg, i64 nt, double* pot, double* grad) {
  FMM& f = *(FMM*)h;
  if (f.kind == STOKES) { g_err = "a Stokes FMM: use the Stokes outputs"; return 1; }
  std::vector<int> node(nt);
  GUARD({ for (i64 q = 0; q < nt; ++q) node[q] = locate(f.t, &tg[3 * q]); })
#pragma omp parallel for schedule(dynamic, 256)
  for (i64 q = 0; q < nt; ++q) {
    double u, g[3];
    evaluate_target(f, &tg[3 * q], node[q], -1, &u, g);
    if (pot) pot[q] = u;
    if (grad) { grad[3 * q] = g[0]; grad[3 * q + 1] = g[1]; grad[3 * q + 2] = g[2]; }
  }
  return 0;
}
// the Stokes outputs (velocity N × 3, pressure N) at the sources, self excluded, original order
int orc_fmm_eval_sources_stokes(void* h, double* vel, double* pres) {
  FMM& f = *(FMM*)h;
  if (f.kind != STOKES) { g_err = "not a Stokes FMM"; return 1; }
  int N = f.t.N;
#pragma omp parallel for schedule(dynamic, 256)
  for (int k = 0; k < N; ++k) {
    double u[3], pr;
    stokes_evaluate_target(f, &f.xs[3 * k], f.t.point_node[k], k, u, &pr);
    int j = f.t.perm[k];
    if (vel) { vel[3 * j] = u[0]; vel[3 * j + 1] = u[1]; vel[3 * j + 2] = u[2]; }
    if (pres) pres[j] = pr;
  }
  return 0;
}
int orc_fmm_eval_targets_stokes(void* h, const double* tg, i64 nt, double* vel, double* pres) {
  FMM& f = *(FMM*)h;
  if (f.kind != STOKES) { g_err = "not a Stokes FMM"; return 1; }
  std::vector<int> node(nt);
  GUARD({ for (i64 q = 0; q < nt; ++q) node[q] = locate(f.t, &tg[3 * q]); })
#pragma omp parallel for schedule(dynamic, 256)
  for (i64 q = 0; q < nt; ++q) {
    double u[3], pr;
    stokes_evaluate_target(f, &tg[3 * q], node[q], -1, u, &pr);
    if (vel) { vel[3 * q] = u[0]; vel[3 * q + 1] = u[1]; vel[3 * q + 2] = u[2]; }
    if (pres) pres[q] = pr;
  }
  return 0;
}
int orc_fmm_nblocks(void* h) { return ((FMM*)h)->nb; }
int orc_fmm_locate(void* h, const double* tg, i64 nt, int32_t* node) {
  FMM& f = *(FMM*)h;
  GUARD({ for (i64 q = 0; q < nt; ++q) node[q] = locate(f.t, &tg[3 * q]); return 0; })
}
int orc_fmm_np(void* h) { return ((FMM*)h)->NP; }
// multipoles / locals, column-major NP × nnodes (node order)
void orc_fmm_expansions(void* h, double* M, double* L) {
  FMM& f = *(FMM*)h;
  if (M) std::copy(f.Mp.begin(), f.Mp.end(), M);
  if (L) std::copy(f.Lc.begin(), f.Lc.end(), L);
}
// the operators of the FMM's reference width: M2M (NP × 8NP), L2L (8NP × NP), reps (34 × NP × NP), column-major
void orc_fmm_operators(void* h, double* M2M, double* L2L, double* reps) {
  FMM& f = *(FMM*)h;
  if (M2M) std::copy(f.M2M.begin(), f.M2M.end(), M2M);
  if (L2L) std::copy(f.L2L.begin(), f.L2L.end(), L2L);
  if (reps) for (size_t c = 0; c < f.reps.size(); ++c) std::copy(f.reps[c].begin(), f.reps[c].end(), reps + c * f.reps[c].size());
}

// ---- operator pieces (for the known-answer tests)
void orc_regular_hobson(const double* x, int p, double* out) {
  std::vector<cplx> Y = regular_hobson(x, p);
  for (size_t i = 0; i < Y.size(); ++i) { out[2 * i] = Y[i].real(); out[2 * i + 1] = Y[i].imag(); }
}
void orc_irregular_hobson(const double* x, int p, double* out) {
  std::vector<cplx> Y = irregular_hobson(x, p);
  for (size_t i = 0; i < Y.size(); ++i) { out[2 * i] = Y[i].real(); out[2 * i + 1] = Y[i].imag(); }
}
void orc_scaling_factors(int p, double* out) { std::vector<double> s = scaling_factors(p); std::copy(s.begin(), s.end(), out); }
// Υ̃ values of the Schmidt recurrence at complex indices (2 doubles each, zero for m < 0)
void orc_fold_regular(const double* x, int p, double* out) {
  Tables tb = harmonic_tables(p);
  std::fill(out, out + 2 * (p + 1) * (p + 1), 0.0);
  fold_regular([&](int n, int m, double vr, double vi) { out[2 * cidx(n, m)] = vr; out[2 * cidx(n, m) + 1] = vi; }, x, p, tb);
}
void orc_harmonic_m2l(const int* o, int p, double c, double* out) {
  std::vector<double> s = scaling_factors(2 * p);
  std::vector<double> R = harmonic_m2l(o, p, c, s);
  std::copy(R.begin(), R.end(), out);
}
// the classes: cls[316], reps[34*3], idx/idx_t[316*NP], sgn/sgn_t[316*NP]
int orc_harmonic_classes(int p, int32_t* cls, int32_t* reps, int32_t* idx, int8_t* sgn, int32_t* idx_t, int8_t* sgn_t) {
  Classes sc = harmonic_symmetry_classes(p);
  int N = (p + 1) * (p + 1);
  for (int f = 0; f < NFAR; ++f) {
    cls[f] = sc.cls[f];
    for (int i = 0; i < N; ++i) {
      idx[f * N + i] = sc.idx[f][i]; sgn[f * N + i] = sc.sgn[f][i]; idx_t[f * N + i] = sc.idx_t[f][i]; sgn_t[f * N + i] = sc.sgn_t[f][i];
    }
  }
  for (size_t c = 0; c < sc.reps.size(); ++c) for (int d = 0; d < 3; ++d) reps[3 * c + d] = sc.reps[c].v[d];
  return (int)sc.reps.size();
}
void orc_far_offsets(int32_t* out) { std::vector<I3> o = far_offsets(); for (int f = 0; f < NFAR; ++f) for (int d = 0; d < 3; ++d) out[3 * f + d] = o[f].v[d]; }

// ---- Yukawa pieces (for the known-answer tests of harmonics_yukawa.jl)
void orc_yukawa_uv(double z, int nmax, double* u, double* v) { yukawa_u(z * z, nmax, u); yukawa_v(z, nmax, v); }
void orc_yukawa_bases(const double* y, const double* x, double kappa, int p, double* br, double* bi) {
  Tables tb = harmonic_tables(p);
  yukawa_regular(br, y, kappa, p, tb);
  yukawa_irregular(bi, x, kappa, p, tb);
}

// ---- direct sums (kernels.jl:442-487): self excludes the target's own index
void orc_direct(const double* src, const double* tau, i64 ns, const double* tg, i64 nt, int self, double* pot, double* grad) {
#pragma omp parallel for schedule(dynamic, 16)
  for (i64 q = 0; q < nt; ++q) {
    const double* x = &tg[3 * q];
    double u = 0, gx = 0, gy = 0, gz = 0;
    for (i64 j = 0; j < ns; ++j) {
      if (self && j == q) continue;
      double d0 = x[0] - src[3 * j], d1 = x[1] - src[3 * j + 1], d2 = x[2] - src[3 * j + 2];
      double r2 = std::fma(d2, d2, std::fma(d1, d1, d0 * d0));
      double ir = 1.0 / std::sqrt(r2);
      u += (KC * ir) * tau[j];
      double a = -KC * ir * ir * ir;
      gx += (a * d0) * tau[j]; gy += (a * d1) * tau[j]; gz += (a * d2) * tau[j];
    }
    if (pot) pot[q] = u;
    if (grad) { grad[3 * q] = gx; grad[3 * q + 1] = gy; grad[3 * q + 2] = gz; }
  }
}
// direct sum at a sample of the sources (indices `sel`), excluding each target itself
void orc_direct_sample(const double* src, const double* tau, i64 ns, const int64_t* sel, i64 nsel, double* pot, double* grad) {
#pragma omp parallel for schedule(dynamic, 4)
  for (i64 q = 0; q < nsel; ++q) {
    i64 t = sel[q];
    const double* x = &src[3 * t];
    double u = 0, gx = 0, gy = 0, gz = 0;
    for (i64 j = 0; j < ns; ++j) {
      if (j == t) continue;
      double d0 = x[0] - src[3 * j], d1 = x[1] - src[3 * j + 1], d2 = x[2] - src[3 * j + 2];
      double r2 = std::fma(d2, d2, std::fma(d1, d1, d0 * d0));
      double ir = 1.0 / std::sqrt(r2);
      u += (KC * ir) * tau[j];
      double a = -KC * ir * ir * ir;
      gx += (a * d0) * tau[j]; gy += (a * d1) * tau[j]; gz += (a * d2) * tau[j];
    }
    if (pot) pot[q] = u;
    if (grad) { grad[3 * q] = gx; grad[3 * q + 1] = gy; grad[3 * q + 2] = gz; }
  }
}

}  // extern "C"
