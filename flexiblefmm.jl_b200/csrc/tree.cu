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
// A batch plan is a forest: several independent point sets, each with its own root box of
// width ldexp(cache W0, e_i), built together. Levels are global: the nodes of a level share
// one width, so an instance's root sits on the level of its width (E − e_i below the widest
// root's). Each instance's keys are taken in its own box, and a second stable sort by the
// instance groups the points per instance; every kernel of the build works per node, and an
// instance's roots, splits, colleagues, 2:1 and ghost steps are those of its own build. At
// flattening, the sibling groups of every level are ordered by instance (stable), then the
// roots of the level follow: the nodes of one instance and level are contiguous and in the
// order of the instance's own tree.
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

// the instance of input point j: the last i with off[i] <= j
__device__ __forceinline__ int instance_of(const int64_t* __restrict__ off, int ninst, int64_t j) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= j) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// the keys of a batch: each point's in its instance's root box (box: origin x, y, z, width)
__global__ void k_keys_batch(const double* __restrict__ xyz, int64_t n, const int64_t* __restrict__ off, int ninst,
                             const double* __restrict__ box, int KL, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = instance_of(off, ninst, j);
  const double ox = box[4 * i], oy = box[4 * i + 1], oz = box[4 * i + 2];
  double x = xyz[3 * j], y = xyz[3 * j + 1], z = xyz[3 * j + 2];
  int cx = 0, cy = 0, cz = 0;
  double w = box[4 * i + 3];
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

// the second sort key of a batch: the instance of each sorted point, with its position
__global__ void k_instance_keys(const uint32_t* __restrict__ perm, int64_t n, const int64_t* __restrict__ off, int ninst,
                                uint64_t* __restrict__ k2, uint32_t* __restrict__ v2) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  k2[j] = (uint64_t)instance_of(off, ninst, perm[j]);
  v2[j] = (uint32_t)j;
}

__global__ void k_gather_sorted(const uint32_t* __restrict__ v2, int64_t n, const uint64_t* __restrict__ keys,
                                const uint32_t* __restrict__ perm, uint64_t* __restrict__ okeys, uint32_t* __restrict__ operm) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  okeys[j] = keys[v2[j]];
  operm[j] = perm[v2[j]];
}

// the nodes of level l with more than ppl points; a node that would split below its instance's
// max_levels sets *deep
__global__ void k_flag_split(const int* __restrict__ lo, const int* __restrict__ hi, const int* __restrict__ inst,
                             const int* __restrict__ root_level, int n, int ppl, int l, int maxl, int* __restrict__ flag,
                             int* __restrict__ deep) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = hi[i] - lo[i] + 1 > ppl;
  flag[i] = f;
  if (f && l - root_level[inst[i]] + 1 >= maxl) *deep = 1;
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
                           const uint64_t* __restrict__ keys, int l, int KL, int ghost, const int* __restrict__ pinst,
                           int* __restrict__ cinst, const int* __restrict__ root_level) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= NCH * nw) return;
  int q = g >> 3, k = g & 7;
  int i = which[q];
  int4 pc = pcell[i];
  const int in = pinst[i];
  const int lr = l - root_level[in];      // the parent's level in its own instance's tree
  int x = 2 * pc.x + (k & 1), y = 2 * pc.y + ((k >> 1) & 1), z = 2 * pc.z + ((k >> 2) & 1);
  uint64_t pk = morton3(x, y, z, lr + 1);
  int shift = 3 * (KL - 1 - lr);
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
  cinst[c] = in;
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
  if (p < 0) {                    // a root: its only colleague is itself
    for (int k = 0; k < NCOL; ++k) col[(int64_t)i * NCOL + k] = k == NCOL / 2 ? i : -1;
    return;
  }
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

// node i of the flat level takes level-local node ord[i]; pos maps level-local indices of this
// level (pos), of the one above (ppos) and below (npos) to flat positions in their levels
__global__ void k_flatten(const int4* __restrict__ lcell, const int* __restrict__ lparent, const int* __restrict__ lcf,
                          const int* __restrict__ llo, const int* __restrict__ lhi, const uint8_t* __restrict__ lflags,
                          const int* __restrict__ lcol, const int* __restrict__ linst, const int* __restrict__ ord,
                          const int* __restrict__ pos, const int* __restrict__ ppos, const int* __restrict__ npos, int n,
                          int l, int off, int poff, int noff, int4* __restrict__ cell, int* __restrict__ parent,
                          int* __restrict__ cf, int* __restrict__ plo, int* __restrict__ phi, uint8_t* __restrict__ flags,
                          int* __restrict__ col, int* __restrict__ inst, int* __restrict__ point_node) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = ord ? ord[i] : i;
  int g = off + i;
  int4 c = lcell[o];
  c.w = l;
  cell[g] = c;
  const int lp = l == 0 ? -1 : lparent[o];
  parent[g] = lp < 0 ? -1 : poff + (ppos ? ppos[lp] : lp);
  cf[g] = lcf[o] < 0 ? -1 : noff + (npos ? npos[lcf[o]] : lcf[o]);
  int lo = llo[o], hi = lhi[o];
  plo[g] = lo;
  phi[g] = hi;
  uint8_t f = lflags[o] | (hi >= lo ? F_SOURCE : 0);
  flags[g] = f;
  for (int k = 0; k < NCOL; ++k) {
    int j = lcol[(int64_t)o * NCOL + k];
    col[(int64_t)g * NCOL + k] = j < 0 ? -1 : off + (pos ? pos[j] : j);
  }
  inst[g] = linst[o];
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
  DBuf<int> parent, cf, lo, hi, depth, col, inst;
  DBuf<uint8_t> flags;
  void grow(int nn, cudaStream_t s) {
    cell.grow(nn, n, s); parent.grow(nn, n, s); cf.grow(nn, n, s); lo.grow(nn, n, s); hi.grow(nn, n, s);
    depth.grow(nn, n, s); flags.grow(nn, n, s); inst.grow(nn, n, s);
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
           const int* root_level, cudaStream_t s) {
  if (nw == 0) return;
  int n0 = chi.n;
  chi.grow(n0 + NCH * nw, s);
  k_children<<<nblk((int64_t)NCH * nw), 256, 0, s>>>(par.cell.p, par.lo.p, par.hi.p, par.cf.p, par.flags.p, which.p, nw,
                                                     chi.cell.p, chi.parent.p, chi.cf.p, chi.lo.p, chi.hi.p, chi.flags.p,
                                                     chi.depth.p, n0, keys, l, KL, ghost ? 1 : 0, par.inst.p, chi.inst.p,
                                                     root_level);
  FMMB_LAUNCH_CHECK();
  chi.n = n0 + NCH * nw;
}

// the colleagues of a level (par: the level above, null for level 0, whose nodes are roots)
void tag(DLevel& lev, const DLevel* par, cudaStream_t s) {
  lev.col.alloc((size_t)NCOL * std::max(lev.n, 1));
  if (lev.n)
    k_tag<<<nblk(lev.n), 256, 0, s>>>(lev.cell.p, lev.parent.p, lev.n, par ? par->col.p : nullptr,
                                      par ? par->cf.p : nullptr, lev.col.p);
  FMMB_LAUNCH_CHECK();
}

void depths(std::vector<DLevel>& levels, cudaStream_t s) {
  int L = (int)levels.size();
  FMMB_CUDA(cudaMemsetAsync(levels[L - 1].depth.p, 0, sizeof(int) * levels[L - 1].n, s));
  for (int l = L - 2; l >= 0; --l)
    if (levels[l].n)
      k_depth<<<nblk(levels[l].n), 256, 0, s>>>(levels[l].cf.p, levels[l].n, levels[l + 1].depth.p, levels[l].depth.p);
  FMMB_LAUNCH_CHECK();
}

// appends the roots of the instances whose root lies on level l (one node each, all their points)
void add_roots(DLevel& lev, int l, const Plan& P, cudaStream_t s) {
  std::vector<int> ids;
  for (int i = 0; i < P.ninst; ++i)
    if (P.inst_root[i] == l) ids.push_back(i);
  if (ids.empty()) return;
  const int r = (int)ids.size(), n0 = lev.n;
  lev.grow(n0 + r, s);
  std::vector<int4> cell(r, make_int4(0, 0, 0, 0));
  std::vector<int> m1(r, -1), zero(r, 0), lo(r), hi(r);
  std::vector<uint8_t> lf(r, F_LEAF);
  for (int k = 0; k < r; ++k) {
    lo[k] = (int)P.inst_off[ids[k]];
    hi[k] = (int)P.inst_off[ids[k] + 1] - 1;
  }
  FMMB_CUDA(cudaMemcpyAsync(lev.cell.p + n0, cell.data(), sizeof(int4) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.parent.p + n0, m1.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.cf.p + n0, m1.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.lo.p + n0, lo.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.hi.p + n0, hi.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.flags.p + n0, lf.data(), r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.depth.p + n0, zero.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaMemcpyAsync(lev.inst.p + n0, ids.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  lev.n = n0 + r;
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
  if (P.inst_off.empty()) {                 // one point set: the plan's box, its root on level 0
    P.ninst = 1;
    P.inst_off = {0, N};
    P.inst_box = {P.origin[0], P.origin[1], P.origin[2], P.W0};
    P.inst_e = {P.e0};
    P.inst_root = {0};
  }
  const bool batch = P.ninst > 1;
  DBuf<int> root_level;
  to_device(root_level, P.inst_root, s);
  const int maxroot = *std::max_element(P.inst_root.begin(), P.inst_root.end());

  // keys and their stable sort (a batch: then stably by instance)
  DBuf<uint64_t> keys(N);
  DBuf<uint32_t> perm(N);
  if (KL > 0) {
    if (batch) {
      to_device(P.d_inst_off, P.inst_off, s);
      to_device(P.d_inst_box, P.inst_box, s);
      k_keys_batch<<<nblk(N), 256, 0, s>>>(xyz_dev, N, P.d_inst_off.p, P.ninst, P.d_inst_box.p, KL, keys.p, perm.p);
    } else {
      k_keys<<<nblk(N), 256, 0, s>>>(xyz_dev, N, P.origin[0], P.origin[1], P.origin[2], P.W0, KL, keys.p, perm.p);
    }
    FMMB_LAUNCH_CHECK();
    radix_sort_pairs(keys.p, perm.p, N, 3 * KL, s);
  } else {
    FMMB_CUDA(cudaMemsetAsync(keys.p, 0, N * sizeof(uint64_t), s));
    k_keys<<<nblk(N), 256, 0, s>>>(xyz_dev, N, 0, 0, 0, 1, 0, keys.p, perm.p);
    FMMB_LAUNCH_CHECK();
  }
  if (batch) {
    if (P.d_inst_off.n == 0) to_device(P.d_inst_off, P.inst_off, s);
    DBuf<uint64_t> k2(N), k3(N);
    DBuf<uint32_t> v2(N), p3(N);
    k_instance_keys<<<nblk(N), 256, 0, s>>>(perm.p, N, P.d_inst_off.p, P.ninst, k2.p, v2.p);
    FMMB_LAUNCH_CHECK();
    int ib = 1;
    while ((1 << ib) < P.ninst) ++ib;
    radix_sort_pairs(k2.p, v2.p, N, ib, s);
    k_gather_sorted<<<nblk(N), 256, 0, s>>>(v2.p, N, keys.p, perm.p, k3.p, p3.p);
    FMMB_LAUNCH_CHECK();
    keys = std::move(k3);
    perm = std::move(p3);
  }

  // the roots, and the refinement (src/tree/device_builder.jl:427-438), level by level
  std::vector<DLevel> levels(1);
  add_roots(levels[0], 0, P, s);
  DBuf<int> flag, which, deep(1);
  while (true) {
    const int l = (int)levels.size() - 1;
    int nsplit = 0;
    if (levels[l].n) {
      DLevel& lev = levels[l];
      flag.alloc(lev.n);
      FMMB_CUDA(cudaMemsetAsync(deep.p, 0, sizeof(int), s));
      k_flag_split<<<nblk(lev.n), 256, 0, s>>>(lev.lo.p, lev.hi.p, lev.inst.p, root_level.p, lev.n, ppl, l, maxl, flag.p,
                                               deep.p);
      FMMB_LAUNCH_CHECK();
      nsplit = compact(flag.p, lev.n, which, s);
      require(nsplit == 0 || read_one(deep.p, s) == 0, FMMB_ERR_ARGUMENT,
              "tree reached max_levels = " + std::to_string(maxl) + "; more than ppl = " + std::to_string(ppl) +
                  " coincident points?");
    }
    if (nsplit == 0 && l >= maxroot) break;
    levels.emplace_back();
    add_roots(levels[l + 1], l + 1, P, s);
    split(levels[l], which, nsplit, l, levels[l + 1], keys.p, KL, false, root_level.p, s);
  }
  const int L = (int)levels.size();
  // colleagues
  for (int l = 0; l < L; ++l) tag(levels[l], l ? &levels[l - 1] : nullptr, s);
  // 2:1 restriction (src/tree/builder.jl:289-316)
  depths(levels, s);
  while (true) {
    int nsplit = 0;
    for (int l = 1; l <= L - 3; ++l) {
      DLevel& lev = levels[l];
      if (lev.n == 0) continue;
      flag.alloc(lev.n);
      k_flag_bad<<<nblk(lev.n), 256, 0, s>>>(lev.flags.p, lev.depth.p, lev.col.p, lev.n, flag.p);
      FMMB_LAUNCH_CHECK();
      int nb = compact(flag.p, lev.n, which, s);
      if (nb == 0) continue;
      split(lev, which, nb, l, levels[l + 1], keys.p, KL, false, root_level.p, s);
      tag(levels[l + 1], &lev, s);
      depths(levels, s);
      nsplit += nb;
    }
    if (nsplit == 0) break;
  }
  // ghosts: the xlist flags of all levels first, then the splits (src/tree/builder.jl:328-351)
  for (int l = 1; l <= L - 2; ++l)
    if (levels[l].n)
      k_flag_xlist<<<nblk(levels[l].n), 256, 0, s>>>(levels[l].flags.p, levels[l].cf.p, levels[l].col.p, levels[l].n);
  FMMB_LAUNCH_CHECK();
  for (int l = 1; l <= L - 2; ++l) {
    DLevel& lev = levels[l];
    if (lev.n == 0) continue;
    flag.alloc(lev.n);
    k_xlist_flag<<<nblk(lev.n), 256, 0, s>>>(lev.flags.p, lev.n, flag.p);
    FMMB_LAUNCH_CHECK();
    int nx = compact(flag.p, lev.n, which, s);
    if (nx == 0) continue;
    split(lev, which, nx, l, levels[l + 1], keys.p, KL, true, root_level.p, s);
    tag(levels[l + 1], &lev, s);
  }

  // flatten (src/tree/builder.jl:392-436); a batch's levels ordered: the sibling groups by
  // instance (stable), then the roots
  P.L = L;
  P.level_start.assign(L + 1, 0);
  for (int l = 0; l < L; ++l) P.level_start[l + 1] = P.level_start[l] + levels[l].n;
  int n = P.level_start[L];
  P.nnodes = n;
  P.level_groups.assign(L, 0);
  std::vector<DBuf<int>> ord(L), pos(L);
  for (int l = 0; l < L; ++l) {
    const int nl = levels[l].n;
    if (!batch) {
      P.level_groups[l] = l == 0 ? 0 : nl / NCH;
      continue;
    }
    std::vector<int> par = to_host(levels[l].parent.p, nl, s), ins = to_host(levels[l].inst.p, nl, s);
    std::vector<int> groups, roots;   // first node of each sibling group; the roots
    for (int i = 0; i < nl;) {
      if (par[i] < 0) { roots.push_back(i); ++i; }
      else { groups.push_back(i); i += NCH; }
    }
    std::stable_sort(groups.begin(), groups.end(), [&](int a, int b) { return ins[a] < ins[b]; });
    std::vector<int> o, q(nl);
    o.reserve(nl);
    for (int g : groups)
      for (int k = 0; k < NCH; ++k) o.push_back(g + k);
    for (int r : roots) o.push_back(r);
    for (int i = 0; i < nl; ++i) q[o[i]] = i;
    P.level_groups[l] = (int)groups.size();
    to_device(ord[l], o, s);
    to_device(pos[l], q, s);
  }
  P.cell.alloc(n); P.parent.alloc(n); P.cf.alloc(n); P.plo.alloc(n); P.phi.alloc(n); P.flags.alloc(n);
  P.col.alloc((size_t)NCOL * n);
  P.node_inst.alloc(n);
  P.point_node.alloc(N);
  for (int l = 0; l < L; ++l) {
    DLevel& lev = levels[l];
    if (lev.n == 0) continue;
    k_flatten<<<nblk(lev.n), 256, 0, s>>>(lev.cell.p, lev.parent.p, lev.cf.p, lev.lo.p, lev.hi.p, lev.flags.p, lev.col.p,
                                          lev.inst.p, ord[l].p, pos[l].p, l ? pos[l - 1].p : nullptr,
                                          l + 1 < L ? pos[l + 1].p : nullptr, lev.n, l, P.level_start[l],
                                          l == 0 ? 0 : P.level_start[l - 1], l == L - 1 ? 0 : P.level_start[l + 1],
                                          P.cell.p, P.parent.p, P.cf.p, P.plo.p, P.phi.p, P.flags.p, P.col.p,
                                          P.node_inst.p, P.point_node.p);
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
  if (batch) P.h_inst = to_host(P.node_inst.p, n, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb
