// The node lists and the M2L interaction lists of a plan.
//
// Far pairs (src/tree/lists.jl:71-124, src/device_lists.jl:261-312): a non-ghost target on
// level ≥ 2 (0-based) pairs with every sourced child of its parent's colleagues at a far
// offset (Chebyshev norm ≥ 2). The reference lists them class-major per level and cuts
// chunks for one GEMM each (src/device_lists.jl:219-278). Here the targets of every level
// ≥ 2 are cut into blocks of TB consecutive nodes, each block owning the pairs of its
// targets grouped by symmetry class, and inside a class by target, then by the enumeration
// order. A block is the unit of the M2L kernels: it owns its targets' partial locals, so
// the scatter is deterministic and needs no atomics, and one launch covers all levels.
#include <algorithm>
#include <numeric>

#include "plan.cuh"
#include "scan_sort.cuh"

namespace fmmb {
namespace {

__constant__ int c_far_index[343];   // m2l table slot → far offset index, -1 for a near offset
__constant__ int c_class[NFAR];      // far offset → symmetry class

__device__ __forceinline__ int far_of(int4 t, int4 s) {
  int ox = s.x - t.x, oy = s.y - t.y, oz = s.z - t.z;
  if (max(abs(ox), max(abs(oy), abs(oz))) < 2) return -1;
  return c_far_index[(ox + 3) + 7 * (oy + 3) + 49 * (oz + 3)];
}

// visits the far pairs (source node, far index) of target t in the reference's order
template <class F>
__device__ __forceinline__ void for_far_pairs(int t, const int4* __restrict__ cell, const int* __restrict__ parent,
                                              const int* __restrict__ cf, const int* __restrict__ col,
                                              const uint8_t* __restrict__ flags, F&& fn) {
  if (flags[t] & F_GHOST) return;
  int p = parent[t];
  if (p < 0) return;               // a root (a batch's roots sit on any level)
  int4 ct = cell[t];
  for (int k = 0; k < NCOL; ++k) {
    int pc = col[(int64_t)p * NCOL + k];
    if (pc < 0) continue;
    int s0 = cf[pc];
    if (s0 < 0) continue;
    for (int s = s0; s < s0 + NCH; ++s) {
      if (!(flags[s] & F_SOURCE)) continue;
      int f = far_of(ct, cell[s]);
      if (f >= 0) fn(s, f);
    }
  }
}

__global__ void k_pair_count(const int4* __restrict__ cell, const int* __restrict__ parent, const int* __restrict__ cf,
                             const int* __restrict__ col, const uint8_t* __restrict__ flags, int first, int n,
                             int* __restrict__ cnt) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int c = 0;
  for_far_pairs(first + q, cell, parent, cf, col, flags, [&](int, int) { ++c; });
  cnt[first + q] = c;
}

// the target-major list of the kernel-independent M2L: target g's pairs (source, far index)
// at tp[ptr[g]..], in the enumeration order
__global__ void k_target_fill(const int4* __restrict__ cell, const int* __restrict__ parent, const int* __restrict__ cf,
                              const int* __restrict__ col, const uint8_t* __restrict__ flags, int first, int n,
                              const int* __restrict__ ptr, int2* __restrict__ tp) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int k = ptr[first + q];
  for_far_pairs(first + q, cell, parent, cf, col, flags, [&](int s, int f) { tp[k++] = make_int2(s, f); });
}

// one CTA per block, one thread per target: counts per (target, class), the class-major
// offsets, and the fill; for the tensor-core M2L the round table: per class and target its
// pair count << 16 | its first pair's offset in the class, and per class the largest count
// (the class's rounds: round r gathers every target's r-th pair of the class)
__global__ void k_block_fill(const int4* __restrict__ blocks, const int4* __restrict__ cell, const int* __restrict__ parent,
                             const int* __restrict__ cf, const int* __restrict__ col, const uint8_t* __restrict__ flags,
                             int* __restrict__ cls_off, int2* __restrict__ pairs, int TB, int* __restrict__ rtab,
                             int* __restrict__ rounds) {
  // blockDim.x = max(TB, 64) threads: the class scans below take one thread per class
  extern __shared__ int sm[];
  int* cnt = sm;                 // [NCLASS][TB]
  int* tot = sm + NCLASS * TB;   // [NCLASS + 1]
  int4 b = blocks[blockIdx.x];
  int t = threadIdx.x;
  if (t < TB)
    for (int c = 0; c < NCLASS; ++c) cnt[c * TB + t] = 0;
  if (t < b.z)
    for_far_pairs(b.y + t, cell, parent, cf, col, flags, [&](int, int f) { cnt[c_class[f] * TB + t]++; });
  __syncthreads();
  if (t < TB)
    for (int c = 0; c < NCLASS; ++c) rtab[((int64_t)blockIdx.x * NCLASS + c) * TB + t] = cnt[c * TB + t] << 16;
  __syncthreads();         // the counts are read above before the scans below overwrite them
  if (t < NCLASS) {        // exclusive scan down each class column, and the class's largest count
    int run = 0, mx = 0;
    for (int q = 0; q < TB; ++q) { int v = cnt[t * TB + q]; cnt[t * TB + q] = run; run += v; mx = max(mx, v); }
    tot[t] = run;
    rounds[(int64_t)blockIdx.x * NCLASS + t] = mx;
  }
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int c = 0; c < NCLASS; ++c) { int v = tot[c]; tot[c] = run; run += v; }
    tot[NCLASS] = run;
  }
  __syncthreads();
  if (t <= NCLASS) cls_off[(int64_t)blockIdx.x * (NCLASS + 1) + t] = tot[t];
  if (t < TB)
    for (int c = 0; c < NCLASS; ++c) rtab[((int64_t)blockIdx.x * NCLASS + c) * TB + t] |= cnt[c * TB + t];
  if (t < b.z) {
    int cur[NCLASS];
#pragma unroll
    for (int c = 0; c < NCLASS; ++c) cur[c] = tot[c] + cnt[c * TB + t];
    int2* out = pairs + b.w;
    for_far_pairs(b.y + t, cell, parent, cf, col, flags, [&](int s, int f) {
      int c = c_class[f];
      int pos = 0;
#pragma unroll
      for (int k = 0; k < NCLASS; ++k)
        if (k == c) pos = cur[k]++;
      out[pos] = make_int2(s, (f << 8) | t);
    });
  }
}

}  // namespace

// the M2L blocks of TB targets each, from the pairs per target (P.h_pair_count): per block its
// class offsets, pairs and round table, launched heaviest first
void build_blocks(Plan& P, int TB) {
  cudaStream_t s = P.ctx->stream;
  const int L = P.L;
  require(TB >= 1 && TB <= 128, FMMB_ERR_ARGUMENT, "targets per M2L block must be in 1..128");
  P.TB = TB;
  P.h_blocks.clear();
  P.level_pairs.assign(L, 0);
  int64_t base = 0;
  require(L < 256, FMMB_ERR_ARGUMENT, "too many levels");
  for (int q = 0; q < P.nseg; ++q) {
    const int l = P.seg_level[q], end = P.seg_start[q + 1];
    if (l < 2) continue;
    for (int b0 = P.seg_start[q]; b0 < end; b0 += P.TB) {
      int c = std::min(P.TB, end - b0);
      int64_t np = 0;
      for (int g = b0; g < b0 + c; ++g) np += P.h_pair_count[g];
      if (np == 0) continue;
      P.h_blocks.push_back({l, q, b0, c, (int)base});
      base += np;
      P.level_pairs[l] += np;
    }
  }
  require(base < (1ll << 31), FMMB_ERR_ARGUMENT, "too many far pairs for 32-bit offsets");
  P.npairs = base;
  int nb = (int)P.h_blocks.size();
  // the M2L kernels take the blocks in launch order heaviest first (most far pairs): the CTA
  // scheduler hands out blocks in index order, so the light ones fill the last wave (longest
  // processing time first); every block owns its targets, so the order changes no sum
  std::vector<int64_t> bp(nb);
  for (int b = 0; b < nb; ++b) bp[b] = (b + 1 < nb ? P.h_blocks[b + 1].pair_base : base) - P.h_blocks[b].pair_base;
  std::vector<int> order(nb);
  for (int b = 0; b < nb; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return bp[a] > bp[b]; });
  std::vector<int4> hb(nb);
  for (int i = 0; i < nb; ++i) {
    const M2LBlock& B = P.h_blocks[order[i]];
    hb[i] = make_int4(B.level | B.seg << 8, B.first, B.count, B.pair_base);
  }
  to_device(P.blocks, hb, s);
  P.cls_off.alloc((size_t)std::max(nb, 1) * (NCLASS + 1));
  P.pairs.alloc(std::max<int64_t>(base, 1));
  P.rtab.alloc((size_t)std::max(nb, 1) * NCLASS * P.TB);
  P.rounds.alloc((size_t)std::max(nb, 1) * NCLASS);
  if (nb) {
    size_t smem = sizeof(int) * (NCLASS * P.TB + NCLASS + 1);
    k_block_fill<<<nb, std::max(P.TB, 64), smem, s>>>(P.blocks.p, P.cell.p, P.parent.p, P.cf.p, P.col.p, P.flags.p,
                                                    P.cls_off.p, P.pairs.p, P.TB, P.rtab.p, P.rounds.p);
    FMMB_LAUNCH_CHECK();
  }
  FMMB_CUDA(cudaStreamSynchronize(s));
}

void build_lists(Plan& P) {
  cudaStream_t s = P.ctx->stream;
  const int n = P.nnodes, L = P.L;
  P.h_parent = to_host(P.parent.p, n, s);
  P.h_cf = to_host(P.cf.p, n, s);
  P.h_plo = to_host(P.plo.p, n, s);
  P.h_phi = to_host(P.phi.p, n, s);
  P.h_flags = to_host(P.flags.p, n, s);

  // childless nodes with sources on levels ≥ 2 of their own tree (src/fmm.jl:45-46), real
  // leaves with points
  const bool batch = P.ninst > 1;
  std::vector<int> s2m, leaves, lstart, lcount;
  for (int l = 0; l < L; ++l)
    for (int g = P.level_start[l]; g < P.level_start[l + 1]; ++g) {
      bool src = (P.h_flags[g] & F_SOURCE) != 0;
      const int lr = batch ? l - P.inst_root[P.h_inst[g]] : l;
      if (lr >= 2 && P.h_cf[g] < 0 && src) s2m.push_back(g);
      if ((P.h_flags[g] & F_LEAF) && src) {
        leaves.push_back(g);
        lstart.push_back(P.h_plo[g]);
        lcount.push_back(P.h_phi[g] - P.h_plo[g] + 1);
      }
    }
  P.n_s2m = (int)s2m.size();
  P.n_leaves = (int)leaves.size();
  to_device(P.s2m_nodes, s2m, s);
  to_device(P.leaves, leaves, s);
  to_device(P.leaf_start, lstart, s);
  to_device(P.leaf_count, lcount, s);
  P.group_parent.clear();
  P.group_parent.resize(L);
  for (int l = 1; l < L; ++l) {
    const int ng = P.level_groups[l];
    std::vector<int> gp(ng);
    for (int g = 0; g < ng; ++g) gp[g] = P.h_parent[P.level_start[l] + NCH * g];
    to_device(P.group_parent[l], gp, s);
  }
  // the segments: per level, the runs of one instance's nodes (one per level for one point set)
  P.seg_start.clear(); P.seg_level.clear(); P.seg_inst.clear();
  for (int l = 0; l < L; ++l)
    for (int g = P.level_start[l]; g < P.level_start[l + 1]; ++g)
      if (g == P.level_start[l] || (batch && P.h_inst[g] != P.h_inst[g - 1])) {
        P.seg_start.push_back(g);
        P.seg_level.push_back(l);
        P.seg_inst.push_back(batch ? P.h_inst[g] : 0);
      }
  P.nseg = (int)P.seg_level.size();
  P.seg_start.push_back(n);
  if (batch) {
    std::vector<int> ns(n);
    for (int q = 0; q < P.nseg; ++q)
      for (int g = P.seg_start[q]; g < P.seg_start[q + 1]; ++g) ns[g] = q;
    to_device(P.node_seg, ns, s);
  } else {
    require(P.nseg == L, FMMB_ERR_DEVICE, "a level without nodes");
  }

  // the offset tables
  {
    std::vector<int> fidx(343, -1);
    int k = 0;
    for (int t = 0; t < 343; ++t) {
      int o[3] = {t % 7 - 3, (t / 7) % 7 - 3, (t / 49) % 7 - 3};
      if (std::max(std::abs(o[0]), std::max(std::abs(o[1]), std::abs(o[2]))) >= 2) fidx[t] = k++;
    }
    FMMB_CUDA(cudaMemcpyToSymbolAsync(c_far_index, fidx.data(), sizeof(int) * 343, 0, cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyToSymbolAsync(c_class, P.cache->host.cls.data(), sizeof(int) * NFAR, 0, cudaMemcpyHostToDevice, s));
  }

  // pairs per target, then the blocks and their bases
  DBuf<int> cnt(std::max(n, 1));
  FMMB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * n, s));
  for (int l = 2; l < L; ++l) {
    int first = P.level_start[l], nl = P.level_start[l + 1] - first;
    k_pair_count<<<(nl + 127) / 128, 128, 0, s>>>(P.cell.p, P.parent.p, P.cf.p, P.col.p, P.flags.p, first, nl, cnt.p);
    FMMB_LAUNCH_CHECK();
  }
  P.h_pair_count = to_host(cnt.p, n, s);
  // targets per block: a tuned size for plans of this kind (tune.cu), else 128, halved (down to
  // 16) while the targets with far pairs fill fewer blocks than the device has SMs, so that small
  // trees still spread over the whole GPU
  int TB = tuned_block_size(P);
  if (TB <= 0) {
    int64_t nt = 0;
    for (int g = P.level_start[std::min(2, L)]; g < P.level_start[L]; ++g) nt += P.h_pair_count[g] > 0;
    TB = 128;
    while (TB > 16 && nt / TB < P.ctx->num_sms) TB /= 2;
  }
  build_blocks(P, TB);
  // per level factors
  std::vector<double> sc(L), ms(L);
  for (int l = 0; l < L; ++l) { sc[l] = P.scale[l]; ms[l] = P.m2l_scale[l]; }
  to_device(P.d_scale, sc, s);
  to_device(P.d_m2l_scale, ms, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// the far pairs of every target as one target-major list (the kernel-independent method's
// spectral M2L pulls each target's sources; ptr has nnodes + 1 entries)
void build_target_pairs(Plan& P) {
  cudaStream_t s = P.ctx->stream;
  const int n = P.nnodes, L = P.L;
  DBuf<int> cnt(n + 1);
  FMMB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (n + 1), s));
  for (int l = 2; l < L; ++l) {
    int first = P.level_start[l], nl = P.level_start[l + 1] - first;
    if (nl) k_pair_count<<<(nl + 127) / 128, 128, 0, s>>>(P.cell.p, P.parent.p, P.cf.p, P.col.p, P.flags.p, first, nl, cnt.p);
    FMMB_LAUNCH_CHECK();
  }
  P.tp_ptr.alloc(n + 1);
  const int64_t total = scan_exclusive_total(cnt.p, P.tp_ptr.p, n + 1, s);
  require(total < (1ll << 31), FMMB_ERR_ARGUMENT, "too many far pairs for 32-bit offsets");
  P.tp.alloc(std::max<int64_t>(total, 1));
  for (int l = 2; l < L; ++l) {
    int first = P.level_start[l], nl = P.level_start[l + 1] - first;
    if (nl) k_target_fill<<<(nl + 127) / 128, 128, 0, s>>>(P.cell.p, P.parent.p, P.cf.p, P.col.p, P.flags.p, first, nl,
                                                        P.tp_ptr.p, P.tp.p);
    FMMB_LAUNCH_CHECK();
  }
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb
