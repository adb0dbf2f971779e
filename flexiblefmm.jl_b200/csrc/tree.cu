// The ghost-cell adaptive octree, built on the device from the points there, with the same
// structure as the reference's host builder (src/tree/builder.jl:45-473) and its device
// builder (src/tree/device_builder.jl:398-501):
//   1. a 63-bit key per point: its child slot at levels 0..KL-1 by the exact comparison
//      against the box centres (src/util.jl:39-45, src/tree/tree.jl:81-83; the centres are
//      formed with explicit round-to-nearest operations so that no contraction changes them)
//   2. a stable radix sort of the keys
//   3. per level (host loop, one count read back per pass): split the nodes with more than
//      ppl points, each child's point range found by two binary searches of its key prefix;
//      colleagues by the parent rule; the 2:1 restriction; the xlist flags of all levels,
//      then the ghost children
//   4. flattening to global node numbers, and the points of every childless node put in
//      their original order (a stable counting sort does that on the host), so that `perm`
//      equals the host tree's too
#include <algorithm>

#include "plan.cuh"
#include "scan_sort.cuh"

namespace fmmb {
namespace {

__device__ __forceinline__ double center_coord(double origin, int c, double w) {
  return __dadd_rn(origin, __dmul_rn(__dadd_rn((double)c, 0.5), w));
}

__device__ __forceinline__ uint64_t morton3(int x, int y, int z, int nbits) {
  uint64_t key = 0;
  for (int b = 0; b < nbits; ++b)
    key |= ((uint64_t)((x >> b) & 1) << (3 * b)) | ((uint64_t)((y >> b) & 1) << (3 * b + 1)) |
           ((uint64_t)((z >> b) & 1) << (3 * b + 2));
  return key;
}

__global__ void k_keys(const double* __restrict__ xyz, int64_t n, double ox, double oy, double oz, double W0, int KL,
                       uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double x = xyz[3 * j], y = xyz[3 * j + 1], z = xyz[3 * j + 2];
  int cx = 0, cy = 0, cz = 0;
  double w = W0;
  uint64_t key = 0;
  for (int b = 0; b < KL; ++b) {
    int k = (x > center_coord(ox, cx, w)) | ((y > center_coord(oy, cy, w)) << 1) | ((z > center_coord(oz, cz, w)) << 2);
    key |= (uint64_t)k << (3 * (KL - 1 - b));
    cx = 2 * cx + (k & 1);
    cy = 2 * cy + ((k >> 1) & 1);
    cz = 2 * cz + ((k >> 2) & 1);
    w = __dmul_rn(w, 0.5);
  }
  keys[j] = key;
  idx[j] = (uint32_t)j;
}

__global__ void k_flag_split(const int* __restrict__ lo, const int* __restrict__ hi, int n, int ppl, int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = hi[i] - lo[i] + 1 > ppl;
}

__global__ void k_compact(const int* __restrict__ flag, const int* __restrict__ pos, int n, int* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) out[pos[i]] = i;
}

// first j in [lo, hi] with keys[j] >= x, hi + 1 if none
__device__ __forceinline__ int lower_bound(const uint64_t* __restrict__ keys, int lo, int hi, uint64_t x) {
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (keys[mid] < x) lo = mid + 1;
    else hi = mid - 1;
  }
  return lo;
}

// children of the split nodes `which` of level l, appended from n0 on level l+1
__global__ void k_children(const int4* __restrict__ pcell, const int* __restrict__ plo, const int* __restrict__ phi,
                           int* __restrict__ pcf, uint8_t* __restrict__ pflags, const int* __restrict__ which, int nw,
                           int4* __restrict__ ccell, int* __restrict__ cparent, int* __restrict__ ccf, int* __restrict__ clo,
                           int* __restrict__ chi, uint8_t* __restrict__ cflags, int* __restrict__ cdepth, int n0,
                           const uint64_t* __restrict__ keys, int l, int KL, int ghost) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= NCH * nw) return;
  int q = g >> 3, k = g & 7;
  int i = which[q];
  int4 pc = pcell[i];
  int x = 2 * pc.x + (k & 1), y = 2 * pc.y + ((k >> 1) & 1), z = 2 * pc.z + ((k >> 2) & 1);
  uint64_t pk = morton3(x, y, z, l + 1);
  int shift = 3 * (KL - 1 - l);
  int lo = plo[i], hi = phi[i];
  int first = lower_bound(keys, lo, hi, pk << shift);
  int last = lower_bound(keys, first, hi, (pk + 1) << shift) - 1;
  int c = n0 + NCH * q + k;
  ccell[c] = make_int4(x, y, z, l + 1);
  cparent[c] = i;
  ccf[c] = -1;
  clo[c] = first;
  chi[c] = last;
  cflags[c] = ghost ? F_GHOST : F_LEAF;
  cdepth[c] = 0;
  if (k == 0) {
    pcf[i] = n0 + NCH * q;
    if (!ghost) pflags[i] &= (uint8_t)~F_LEAF;
  }
}

// colleagues by the parent rule (src/tree/builder.jl:212-248)
__global__ void k_tag(const int4* __restrict__ cell, const int* __restrict__ parent, int n, const int* __restrict__ pcol,
                      const int* __restrict__ pcf, int* __restrict__ col) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int4 c = cell[i];
  int p = parent[i];
  int px = c.x >> 1, py = c.y >> 1, pz = c.z >> 1;
  for (int k = 0; k < NCOL; ++k) {
    int x = c.x + k % 3 - 1, y = c.y + (k / 3) % 3 - 1, z = c.z + k / 9 - 1;
    int oi = ((x >> 1) - px + 1) + 3 * ((y >> 1) - py + 1) + 9 * ((z >> 1) - pz + 1);
    int q = pcol[(int64_t)p * NCOL + oi];
    col[(int64_t)i * NCOL + k] = (q < 0 || pcf[q] < 0) ? -1 : pcf[q] + ((x & 1) | ((y & 1) << 1) | ((z & 1) << 2));
  }
}

__global__ void k_depth(const int* __restrict__ cf, int n, const int* __restrict__ cdepth, int* __restrict__ depth) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int f = cf[i];
  if (f < 0) { depth[i] = 0; return; }
  int m = 0;
  for (int k = 0; k < NCH; ++k) m = max(m, cdepth[f + k]);
  depth[i] = m + 1;
}

// a leaf is bad if a colleague's depth differs from its own by more than one
__global__ void k_flag_bad(const uint8_t* __restrict__ flags, const int* __restrict__ depth, const int* __restrict__ col, int n,
                           int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = 0;
  if (flags[i] & F_LEAF) {
    int di = depth[i];
    for (int k = 0; k < NCOL; ++k) {
      int j = col[(int64_t)i * NCOL + k];
      if (j >= 0 && abs(di - depth[j]) > 1) { b = 1; break; }
    }
  }
  flag[i] = b;
}

// a real leaf with a colleague that has children is an xlist leaf
__global__ void k_flag_xlist(uint8_t* __restrict__ flags, const int* __restrict__ cf, const int* __restrict__ col, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!(flags[i] & F_LEAF)) return;
  for (int k = 0; k < NCOL; ++k) {
    int j = col[(int64_t)i * NCOL + k];
    if (j >= 0 && cf[j] >= 0) { flags[i] |= F_XLIST; return; }
  }
}

__global__ void k_xlist_flag(const uint8_t* __restrict__ flags, int n, int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (flags[i] & F_XLIST) != 0;
}

__global__ void k_flatten(const int4* __restrict__ lcell, const int* __restrict__ lparent, const int* __restrict__ lcf,
                          const int* __restrict__ llo, const int* __restrict__ lhi, const uint8_t* __restrict__ lflags,
                          const int* __restrict__ lcol, int n, int l, int off, int poff, int noff, int4* __restrict__ cell,
                          int* __restrict__ parent, int* __restrict__ cf, int* __restrict__ plo, int* __restrict__ phi,
                          uint8_t* __restrict__ flags, int* __restrict__ col, int* __restrict__ point_node) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int g = off + i;
  int4 c = lcell[i];
  c.w = l;
  cell[g] = c;
  parent[g] = l == 0 ? -1 : poff + lparent[i];
  cf[g] = lcf[i] < 0 ? -1 : noff + lcf[i];
  int lo = llo[i], hi = lhi[i];
  plo[g] = lo;
  phi[g] = hi;
  uint8_t f = lflags[i] | (hi >= lo ? F_SOURCE : 0);
  flags[g] = f;
  for (int k = 0; k < NCOL; ++k) {
    int j = lcol[(int64_t)i * NCOL + k];
    col[(int64_t)g * NCOL + k] = j < 0 ? -1 : off + j;
  }
  if (f & F_LEAF)
    for (int j = lo; j <= hi; ++j) point_node[j] = g;
}

// key of each point for the order within childless nodes: (range start, original index)
__global__ void k_leaf_keys(const int* __restrict__ cf, const int* __restrict__ plo, const int* __restrict__ phi, int n,
                            const uint32_t* __restrict__ perm, uint64_t* __restrict__ keys) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n || cf[g] >= 0) return;
  int lo = plo[g], hi = phi[g];
  for (int j = lo; j <= hi; ++j) keys[j] = ((uint64_t)lo << 32) | perm[j];
}

__global__ void k_unpack_perm(const uint64_t* __restrict__ keys, int64_t n, int* __restrict__ perm) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) perm[j] = (int)(uint32_t)keys[j];
}

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// one level of the builder (src/tree/device_builder.jl:152-179), level-local indices
struct DLevel {
  int n = 0;
  DBuf<int4> cell;
  DBuf<int> parent, cf, lo, hi, depth, col;
  DBuf<uint8_t> flags;
  void grow(int nn, cudaStream_t s) {
    cell.grow(nn, n, s); parent.grow(nn, n, s); cf.grow(nn, n, s); lo.grow(nn, n, s); hi.grow(nn, n, s);
    depth.grow(nn, n, s); flags.grow(nn, n, s);
  }
};

// the set flags' indices, in order
int compact(const int* flag, int n, DBuf<int>& out, cudaStream_t s) {
  if (n == 0) return 0;
  DBuf<int> pos(n);
  int cnt = (int)scan_exclusive_total(flag, pos.p, n, s);
  out.alloc(std::max(cnt, 1));
  if (cnt) k_compact<<<nblk(n), 256, 0, s>>>(flag, pos.p, n, out.p);
  FMMB_LAUNCH_CHECK();
  return cnt;
}

void split(DLevel& par, const DBuf<int>& which, int nw, int l, DLevel& chi, const uint64_t* keys, int KL, bool ghost,
           cudaStream_t s) {
  if (nw == 0) return;
  int n0 = chi.n;
  chi.grow(n0 + NCH * nw, s);
  k_children<<<nblk((int64_t)NCH * nw), 256, 0, s>>>(par.cell.p, par.lo.p, par.hi.p, par.cf.p, par.flags.p, which.p, nw,
                                                     chi.cell.p, chi.parent.p, chi.cf.p, chi.lo.p, chi.hi.p, chi.flags.p,
                                                     chi.depth.p, n0, keys, l, KL, ghost ? 1 : 0);
  FMMB_LAUNCH_CHECK();
  chi.n = n0 + NCH * nw;
}

void tag(DLevel& lev, const DLevel& par, cudaStream_t s) {
  lev.col.alloc((size_t)NCOL * std::max(lev.n, 1));
  if (lev.n) k_tag<<<nblk(lev.n), 256, 0, s>>>(lev.cell.p, lev.parent.p, lev.n, par.col.p, par.cf.p, lev.col.p);
  FMMB_LAUNCH_CHECK();
}

void depths(std::vector<DLevel>& levels, cudaStream_t s) {
  int L = (int)levels.size();
  FMMB_CUDA(cudaMemsetAsync(levels[L - 1].depth.p, 0, sizeof(int) * levels[L - 1].n, s));
  for (int l = L - 2; l >= 0; --l)
    k_depth<<<nblk(levels[l].n), 256, 0, s>>>(levels[l].cf.p, levels[l].n, levels[l + 1].depth.p, levels[l].depth.p);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

void build_tree(Plan& P, const double* xyz_dev, int ppl, int max_levels) {
  cudaStream_t s = P.ctx->stream;
  const int64_t N = P.N;
  require(N > 0, FMMB_ERR_ARGUMENT, "no points");
  require(N < (1ll << 31) - 1, FMMB_ERR_ARGUMENT, "too many points for 32-bit indices");
  require(ppl >= 1, FMMB_ERR_ARGUMENT, "ppl must be positive");
  int KL = std::min(max_levels - 1, 21);   // key levels: 3 bits each (src/tree/device_builder.jl:407)
  require(KL >= 0, FMMB_ERR_ARGUMENT, "max_levels must be positive");
  int maxl = KL + 1;
  P.KL = KL;

  // keys and their stable sort
  DBuf<uint64_t> keys(N);
  DBuf<uint32_t> perm(N);
  if (KL > 0) {
    k_keys<<<nblk(N), 256, 0, s>>>(xyz_dev, N, P.origin[0], P.origin[1], P.origin[2], P.W0, KL, keys.p, perm.p);
    FMMB_LAUNCH_CHECK();
    radix_sort_pairs(keys.p, perm.p, N, 3 * KL, s);
  } else {
    FMMB_CUDA(cudaMemsetAsync(keys.p, 0, N * sizeof(uint64_t), s));
    k_keys<<<nblk(N), 256, 0, s>>>(xyz_dev, N, 0, 0, 0, 1, 0, keys.p, perm.p);
    FMMB_LAUNCH_CHECK();
  }

  // the root
  std::vector<DLevel> levels(1);
  {
    DLevel& r = levels[0];
    r.grow(1, s);
    int4 c0 = make_int4(0, 0, 0, 0);
    int m1 = -1, z = 0, hi = (int)N - 1;
    uint8_t lf = F_LEAF;
    FMMB_CUDA(cudaMemcpyAsync(r.cell.p, &c0, sizeof(int4), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.parent.p, &m1, sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.cf.p, &m1, sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.lo.p, &z, sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.hi.p, &hi, sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.flags.p, &lf, 1, cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(r.depth.p, &z, sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    r.n = 1;
  }
  // refinement (src/tree/device_builder.jl:427-438)
  DBuf<int> flag, which;
  while (true) {
    DLevel& lev = levels.back();
    flag.alloc(lev.n);
    k_flag_split<<<nblk(lev.n), 256, 0, s>>>(lev.lo.p, lev.hi.p, lev.n, ppl, flag.p);
    FMMB_LAUNCH_CHECK();
    int nsplit = compact(flag.p, lev.n, which, s);
    if (nsplit == 0) break;
    require((int)levels.size() < maxl, FMMB_ERR_ARGUMENT,
            "tree reached max_levels = " + std::to_string(maxl) + "; more than ppl = " + std::to_string(ppl) +
                " coincident points?");
    levels.emplace_back();
    int l = (int)levels.size() - 2;
    split(levels[l], which, nsplit, l, levels[l + 1], keys.p, KL, false, s);
  }
  const int L = (int)levels.size();
  // colleagues
  {
    DLevel& r = levels[0];
    r.col.alloc(NCOL);
    std::vector<int> rc(NCOL, -1);
    rc[13] = 0;
    FMMB_CUDA(cudaMemcpyAsync(r.col.p, rc.data(), NCOL * sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
  }
  for (int l = 1; l < L; ++l) tag(levels[l], levels[l - 1], s);
  // 2:1 restriction (src/tree/builder.jl:289-316)
  depths(levels, s);
  while (true) {
    int nsplit = 0;
    for (int l = 1; l <= L - 3; ++l) {
      DLevel& lev = levels[l];
      flag.alloc(lev.n);
      k_flag_bad<<<nblk(lev.n), 256, 0, s>>>(lev.flags.p, lev.depth.p, lev.col.p, lev.n, flag.p);
      FMMB_LAUNCH_CHECK();
      int nb = compact(flag.p, lev.n, which, s);
      if (nb == 0) continue;
      split(lev, which, nb, l, levels[l + 1], keys.p, KL, false, s);
      tag(levels[l + 1], lev, s);
      depths(levels, s);
      nsplit += nb;
    }
    if (nsplit == 0) break;
  }
  // ghosts: the xlist flags of all levels first, then the splits (src/tree/builder.jl:328-351)
  for (int l = 1; l <= L - 2; ++l)
    k_flag_xlist<<<nblk(levels[l].n), 256, 0, s>>>(levels[l].flags.p, levels[l].cf.p, levels[l].col.p, levels[l].n);
  FMMB_LAUNCH_CHECK();
  for (int l = 1; l <= L - 2; ++l) {
    DLevel& lev = levels[l];
    flag.alloc(lev.n);
    k_xlist_flag<<<nblk(lev.n), 256, 0, s>>>(lev.flags.p, lev.n, flag.p);
    FMMB_LAUNCH_CHECK();
    int nx = compact(flag.p, lev.n, which, s);
    if (nx == 0) continue;
    split(lev, which, nx, l, levels[l + 1], keys.p, KL, true, s);
    tag(levels[l + 1], lev, s);
  }

  // flatten (src/tree/builder.jl:392-436)
  P.L = L;
  P.level_start.assign(L + 1, 0);
  for (int l = 0; l < L; ++l) P.level_start[l + 1] = P.level_start[l] + levels[l].n;
  int n = P.level_start[L];
  P.nnodes = n;
  P.cell.alloc(n); P.parent.alloc(n); P.cf.alloc(n); P.plo.alloc(n); P.phi.alloc(n); P.flags.alloc(n);
  P.col.alloc((size_t)NCOL * n);
  P.point_node.alloc(N);
  for (int l = 0; l < L; ++l) {
    DLevel& lev = levels[l];
    k_flatten<<<nblk(lev.n), 256, 0, s>>>(lev.cell.p, lev.parent.p, lev.cf.p, lev.lo.p, lev.hi.p, lev.flags.p, lev.col.p,
                                          lev.n, l, P.level_start[l], l == 0 ? 0 : P.level_start[l - 1],
                                          l == L - 1 ? 0 : P.level_start[l + 1], P.cell.p, P.parent.p, P.cf.p, P.plo.p,
                                          P.phi.p, P.flags.p, P.col.p, P.point_node.p);
    FMMB_LAUNCH_CHECK();
  }
  // the points of every childless node in their original order
  k_leaf_keys<<<nblk(n), 256, 0, s>>>(P.cf.p, P.plo.p, P.phi.p, n, perm.p, keys.p);
  FMMB_LAUNCH_CHECK();
  int nbits = 1;
  while ((1ll << nbits) < N) ++nbits;
  radix_sort_pairs(keys.p, perm.p, N, 32 + nbits, s);
  P.perm.alloc(N);
  k_unpack_perm<<<nblk(N), 256, 0, s>>>(keys.p, N, P.perm.p);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb
