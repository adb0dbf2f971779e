// The mixed path's M2L on the 5th-generation tensor cores (tcgen05, kind::f16).
//
// Same work decomposition as the FP64 kernel (one CTA per block of targets, the block's far
// pairs grouped by symmetry class; src/device_passes.jl:565-580, harmonics.jl:589-645), with
// the class product on the tensor cores in three-term split precision over FP16:
//   - every multipole column is scaled by a power of two (per node, so that its largest entry
//     lies in [2^13, 2^14)) and split into an FP16 head and tail, x·2^e ≈ hi + lo (22
//     significant bits over FP16's range; the scale keeps every column inside it);
//   - every row of a class operator is scaled the same way (per class and (n, m) pair of rows);
//   - A·B ≈ hi(A)·hi(B) + hi(A)·lo(B) + lo(A)·hi(B), accumulated in FP32 in tensor memory;
//     FP16 products are exact in FP32. The read-back removes both scales (exact powers of two).
// Orders with (p+1)² ≤ 128 use one 128-row tile of outputs; up to (p+1)² = 144 (p = 11) a
// second tile covers rows 128..(p+1)²-1.
//
// Per CTA, three roles connected by mbarriers over a ring of STAGES (warp specialisation):
//   - one gather warp per stage builds chunk i (≤ 64 pairs of one class) in B stage i mod
//     STAGES, so STAGES chunks are gathered at once; in the UMMA K-major canonical layout
//     (8-row × 16-byte core matrices, no swizzle): 8 consecutive lanes write the 8 pairs of one
//     core matrix (one 128-byte row of banks), 4 lanes read 64 contiguous bytes of one source
//     column, and the loads of two groups of 8 pairs are in flight together. The source-side
//     signed permutation P_sᵀ costs one XOR per word: odd quarter-turn rotations read a second
//     copy of the multipoles in which the two entries of every odd-order pair are swapped;
//   - one thread loads the class operator (head and tail, laid out on the host) with one bulk
//     copy (cp.async.bulk, no tensor map, no multicast) when the class changes, after the
//     previous class's MMAs completed; then per chunk issues (p+1)²/16 K-steps × tiles × 3 MMAs
//     (M = 128, N = chunk rounded to 16, K = 16) into accumulator stage s and commits them;
//   - the read-back warps (thread = output row) load the stage from tensor memory, apply the
//     target-side permutation P_t (one shuffle), sum the consecutive pairs of each target in
//     FP32 and add the sum, with both scales and the level factor W_ref/w applied, to the FP64
//     partial local with a reduction (the block owns its targets and each entry has one
//     writing thread, so the additions apply in program order: deterministic).
// Every wait on an mbarrier is bounded and also gives up when another role has given up; the
// CTA then waits (bounded) for the copies and MMAs it issued, records an error in a device
// flag, frees its tensor memory and returns; the host turns the flag into FMMB_ERR_TIMEOUT.
#include <cstring>

#include <cuda_fp16.h>

#include "d4h.cuh"
#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int NCHK = 64;          // pairs per MMA chunk (the N of the MMA)
constexpr int CORE = 128;         // bytes of one 8 × 16 B core matrix
constexpr int NPMAX = 144;        // (p+1)² supported: p ≤ 11
constexpr int GROUP = 32;         // entries one gather lane octet covers per instruction (4 core columns)
constexpr unsigned long long SPIN_LIMIT = 1ull << 26;
constexpr uint64_t WAIT_NS = 1000000000ull;  // one second: a wait in a working pipeline takes microseconds
constexpr int TMEM_COLS = 512;

__host__ __device__ constexpr int kp_of(int np) { return (np + 15) / 16 * 16; }          // K, padded to the MMA's K
__host__ __device__ constexpr int rows_of(int np) { return np > 128 ? 128 + (np - 128 + 7) / 8 * 8 : 128; }  // rows stored

// canonical K-major offset (bytes) of FP16 element (row, k) in a tile with kp columns
__host__ __device__ __forceinline__ uint32_t canon16(int row, int k, int kp) {
  return (uint32_t)((row >> 3) * (kp / 8) * CORE + (k >> 3) * CORE + (row & 7) * 16 + (k & 7) * 2);
}

// bit i of x moved to bit 2i
__device__ __forceinline__ uint64_t spread_bits(uint32_t x32) {
  uint64_t x = x32;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fff);               // start address
  d |= (uint64_t)((CORE >> 4) & 0x3fff) << 16;          // leading byte offset: next core matrix along K
  d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;           // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                               // descriptor version (sm_100)
  return d;                                             // base offset 0, no swizzle
}

// instruction descriptor: D f32, A/B f16, both K-major, M = m (128 or 64), N = n
__device__ __forceinline__ uint32_t instr_desc(int n, int m = 128) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}

// a wait bounded in time (WAIT_NS of the global timer) and in polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (unsigned long long it = 0; it < SPIN_LIMIT; ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 63) == 63) {
      const uint64_t t = global_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 > WAIT_NS) return false;
    }
  }
  return false;
}

// a bounded wait that also gives up when another role aborted
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (unsigned long long it = 0; it < SPIN_LIMIT; ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 63) == 63) {
      if (*abort_flag) return false;
      const uint64_t t = global_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 > WAIT_NS) break;
    }
  }
  *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
      : "memory");
}

__device__ __forceinline__ void tmem_st1(uint32_t taddr, float v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v)) : "memory");
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// the 16 D4h elements' (swap, negate) codes for one entry, 2 bits per element; the source
// side (gather, phase conjugated) or the target side (scatter, sign of the partner when swapped)
__host__ __device__ __forceinline__ uint32_t perm_mask(int k, bool target) {
  int n, m, part;
  coef_nmp(k, n, m, part);
  uint32_t mask = 0;
  for (int fac = 0; fac < 16; ++fac) {
    const int q = ((target ? m : -m) * (fac & 3)) & 3;
    const bool sw = part != 0 && (q & 1);
    const int sp = target && sw ? 3 - part : part;
    const bool neg = perm_sign(sp, q, n + m, fac) < 0;
    mask |= (uint32_t)((sw ? 1 : 0) | (neg ? 2 : 0)) << (2 * fac);
  }
  return mask;
}

// per chunk: the source scale, D4h element and target of every column; the target runs (bit q
// of `starts` set where column q begins a run; per run its last column and its target)
struct __align__(16) PairInfo {
  float cs[NCHK];
  float keep[NCHK];  // 0 where the column starts a target run, else 1 (the running sum's factor)
  int fac[NCHK];     // twice the D4h element (the shift of its code in a row's mask)
  int tgt[NCHK];
  int rend[NCHK];
  int rtgt[NCHK];
  unsigned long long starts;
  int n, nruns, split;      // split: the first run start at or after column n/2 (n if none)
};

template <int KP, int MT>
struct TcCfg {
  static constexpr int KC = KP / 8;                        // 16-byte core columns along K
  static constexpr int SBO = KC * CORE;                    // bytes between 8-row groups
  static constexpr int U = (KC + 3) / 4;                   // gather instructions per column and half
  static constexpr int A_BYTES = 2 * (MT == 1 ? 128 : NPMAX) * KP * 2;   // head + tail of one class
  static constexpr int B_HALF = NCHK * KP * 2;
  static constexpr int STAGE_BYTES = 2 * B_HALF;
  static constexpr int STAGES = MT == 1 ? 4 : 3;
  // warp roles (a warp reads the tensor-memory lane quadrant warp % 4): read-back warps 0-7 for the
  // first tile (two per quadrant), for a second tile (p = 11) warps 8 and 12 (its rows lie in
  // quadrant 0); the issuing warp IW = 16; the other warps gather, GPS per stage
  static constexpr int NEPI = 8 + 2 * (MT - 1);            // read-back warps
  static constexpr int GPS = 2;                            // gather warps per stage
  static constexpr int IW = 16;
  static constexpr int THREADS = 32 * (IW + 1);
  static_assert(NEPI + STAGES * GPS + 1 == IW + 1, "warp roles");
  // the gather index of warp w (not a read-back or the issuing warp)
  __device__ static int gather_index(int w) { return MT == 1 ? w - 8 : (w < 12 ? w - 9 : w - 10); }
  static constexpr int B_OFF = (A_BYTES + 1023) / 1024 * 1024;
  static constexpr int PI_OFF = B_OFF + STAGES * STAGE_BYTES;
  static constexpr int SGN_OFF = PI_OFF + STAGES * (int)sizeof(PairInfo);
  static constexpr int D4H_OFF = SGN_OFF + 16 * KC * 16;
  static constexpr int BAR_OFF = D4H_OFF + NFAR * 4;
  static constexpr int SMEM = BAR_OFF + (1 + 3 * STAGES) * 8 + 16;
  static_assert(STAGES * MT * NCHK <= TMEM_COLS, "tensor memory");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// perm16 (global): KC × 16 × 4 sign words of the source-side permutation (0x8000 in each FP16
// half that is negated); Mh/Ml: two copies of the split multipoles vstride apart, the second
// with the two entries of every odd-order pair swapped (what odd quarter-turns read)
template <int KP, int MT>
__global__ void __launch_bounds__(TcCfg<KP, MT>::THREADS, 1)
k_m2l_tc(const int4* __restrict__ blocks, const int* __restrict__ cls_off, const int2* __restrict__ pairs,
         const uint16_t* __restrict__ reps16, const float* __restrict__ row_scale, const uint32_t* __restrict__ perm16,
         const double* __restrict__ m2l_scale, int NP, int LD, int lo_off, int64_t vstride, const uint16_t* __restrict__ Mh,
         const uint16_t* __restrict__ Ml, const float* __restrict__ Msc, double* __restrict__ Pl, int* __restrict__ err) {
  using G = TcCfg<KP, MT>;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sA = sm;                                         // head rows, then the tail at lo_off
  unsigned char* sB = sm + G::B_OFF;                              // stage s: head at s·STAGE_BYTES, tail after it
  PairInfo* pinfo = (PairInfo*)(sm + G::PI_OFF);                  // per stage
  uint4* s_sgn = (uint4*)(sm + G::SGN_OFF);                       // [KC][16]
  int* s_d4h = (int*)(sm + G::D4H_OFF);
  uint64_t* bars = (uint64_t*)(sm + G::BAR_OFF);
  uint64_t* bar_a = bars;                                         // operator load
  uint64_t* full = bars + 1;                                      // [STAGES] gathered (32·GPS arrivals)
  uint64_t* done = bars + 1 + G::STAGES;                          // [STAGES] MMAs complete (commit)
  uint64_t* tempty = bars + 1 + 2 * G::STAGES;                    // [STAGES] read back (NEPI·32 arrivals)
  uint32_t* tmem_slot = (uint32_t*)(bars + 1 + 3 * G::STAGES);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);

  for (int f = tid; f < NFAR; f += G::THREADS) s_d4h[f] = c_d4h[f];
  for (int e = tid; e < 16 * G::KC; e += G::THREADS) s_sgn[e] = reinterpret_cast<const uint4*>(perm16)[e];
  if (tid == 0) {
    mbar_init(bar_a, 1);
    for (int s = 0; s < G::STAGES; ++s) {
      mbar_init(&full[s], 32 * G::GPS);
      mbar_init(&done[s], 1);
      mbar_init(&tempty[s], 32 * G::NEPI);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  const bool reader = warp < 8 || (MT == 2 && (warp == 8 || warp == 12));
  if (reader) {
    // ---------------- read back and scatter: thread = output row of tile `tile`
    // two warps per lane quadrant and tile: one takes the columns before the chunk's split, the
    // other the rest; the split is a run start, so every entry still has one writer per chunk
    const int tile = warp < 8 ? 0 : 1;
    const int half = warp < 8 ? warp >> 2 : (warp == 8 ? 0 : 1), quad = warp & 3;
    const int row = 128 * tile + 32 * quad + lane;
    const bool live = row < NP;
    const double alpha = m2l_scale[b.x];
    uint32_t emask = 0;
    int src_lane = lane;
    if (live) {
      int en, em, epart;
      coef_nmp(row, en, em, epart);
      emask = perm_mask(row, true);
      const int partner = epart == 0 ? row : (epart == 1 ? row + 1 : row - 1);
      src_lane = partner & 31;                       // pairs never straddle a 32-row boundary (p ≤ 11)
    }
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int a0 = co[c], a1 = co[c + 1];
      if (a0 == a1) continue;
      const double rs = live ? alpha * (double)row_scale[c * NP + row] : 0.0;
      for (int q0 = a0; q0 < a1; q0 += NCHK, ++i) {
        const int s = i % G::STAGES;
        const uint32_t ph = (uint32_t)(i / G::STAGES) & 1;
        const bool w = mbar_wait_abortable(&full[s], ph, abort_flag) && mbar_wait_abortable(&done[s], ph, abort_flag);
        if (!__all_sync(0xffffffffu, w)) { ok = false; break; }   // the warp leaves together (tcgen05.ld is warp-wide)
        tc_fence_after();
        const PairInfo& pi = pinfo[s];
        const int nc = pi.n;
        const uint64_t starts = pi.starts;
        const int lo = half ? pi.split : 0, hi = half ? nc : pi.split;
        const uint32_t ta = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)((s * MT + tile) * NCHK);
        // phase 1 (branch-free): per column the permuted, unscaled value, and the running sum of
        // the column's target run (reset where a run starts), written back in place of the
        // accumulator columns just read (only this warp's columns: the other half owns the rest)
        float acc = 0.f;
#pragma unroll
        for (int c16 = 0; c16 < NCHK / 16; ++c16) {
          if (16 * c16 >= hi) break;                      // uniform across the warp
          if (16 * c16 + 16 <= lo) continue;
          float d[16], a[16];
          tmem_ld16(ta + 16 * c16, d);
          tmem_wait_ld();
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4) {
            const int4 f4 = reinterpret_cast<const int4*>(pi.fac)[4 * c16 + e4];
            const float4 c4 = reinterpret_cast<const float4*>(pi.cs)[4 * c16 + e4];
            const float4 k4 = reinterpret_cast<const float4*>(pi.keep)[4 * c16 + e4];
            const float kk[4] = {k4.x, k4.y, k4.z, k4.w};
            const int ff[4] = {f4.x, f4.y, f4.z, f4.w};
            const float cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float v = d[4 * e4 + e];
              const float other = __shfl_sync(0xffffffffu, v, src_lane);
              const uint32_t code = emask >> ff[e];   // ff = 2·(D4h element): its 2-bit code
              float y = ((code & 1) ? other : v) * cc[e];
              y = (code & 2) ? -y : y;
              acc = fmaf(acc, kk[e], y);   // y where a run starts (0·acc + y), else acc + y
              a[4 * e4 + e] = acc;
            }
          }
          if (16 * c16 >= lo && (16 * c16 + 16 <= hi || hi == nc)) {
            tmem_st16(ta + 16 * c16, a);
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (16 * c16 + e >= lo && 16 * c16 + e < hi) tmem_st1(ta + 16 * c16 + e, a[e]);   // uniform
          }
        }
        tmem_wait_st();
        // phase 2: the sum of each run is the scan at its last column; one reduction per run
        // (the only writer of these entries: the reductions apply in program order)
        const int k_lo = lo >= 64 ? __popcll(starts) : __popcll(starts & ((1ull << lo) - 1));
        const int k_hi = hi >= 64 ? __popcll(starts) : __popcll(starts & ((1ull << hi) - 1));
        for (int k0 = k_lo; k0 < k_hi; k0 += 4) {
          float v[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) v[k] = tmem_ld1(ta + (uint32_t)pi.rend[min(k0 + k, k_hi - 1)]);
          tmem_wait_ld();
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (live && k0 + k < k_hi) atomicAdd(&Pl[(int64_t)(b.y + pi.rtgt[k0 + k]) * LD + row], rs * (double)v[k]);
        }
        tc_fence_before();
        mbar_arrive(&tempty[s]);
      }
    }
  } else if (warp != G::IW) {
    // ---------------- gather: the GPS warps of stage s build the chunks i ≡ s (mod STAGES), warp h
    // of them every GPS-th pair of groups; lane octet o = lane & 7 the pairs of a group of 8,
    // cq = lane >> 3 the core column
    const int gw = G::gather_index(warp), o = lane & 7, cq = lane >> 3;
    const int s = gw / G::GPS, h = gw % G::GPS;
    unsigned char* bh = sB + s * G::STAGE_BYTES;
    PairInfo& pi = pinfo[s];
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int a0 = co[c], a1 = co[c + 1];
      for (int q0 = a0; q0 < a1; q0 += NCHK, ++i) {
        if (i % G::STAGES != s) continue;
        if (i >= G::STAGES) {
          const bool w = mbar_wait_abortable(&tempty[s], (uint32_t)(i / G::STAGES - 1) & 1, abort_flag);
          if (!__all_sync(0xffffffffu, w)) { ok = false; break; }   // the warp leaves together (shuffles below)
        }
        const int nc = min(NCHK, a1 - q0), ng = (nc + 15) / 16 * 2;   // groups of 8 up to N = nc rounded to 16
        // the chunk's pairs: lane l holds columns 2l and 2l + 1
        int srcA = -1, srcB = -1, facA = 0, facB = 0, tA = -1, tB = -1;
        const bool vA = 2 * lane < nc, vB = 2 * lane + 1 < nc;
        if (vA) {
          const int2 pr = pairs[b.w + q0 + 2 * lane];
          srcA = pr.x;
          facA = s_d4h[pr.y >> 8];
          tA = pr.y & 0xff;
        }
        if (vB) {
          const int2 pr = pairs[b.w + q0 + 2 * lane + 1];
          srcB = pr.x;
          facB = s_d4h[pr.y >> 8];
          tB = pr.y & 0xff;
        }
        if (h == 0) {                                   // the first warp of the stage records the chunk
          if (vA) { pi.fac[2 * lane] = 2 * facA; pi.tgt[2 * lane] = tA; }
          if (vB) { pi.fac[2 * lane + 1] = 2 * facB; pi.tgt[2 * lane + 1] = tB; }
          // the target runs of the chunk (pairs are sorted by target within a class)
          const int tprev = __shfl_up_sync(0xffffffffu, tB, 1);
          const bool stA = vA && (lane == 0 || tA != tprev), stB = vB && tB != tA;
          if (vA) pi.keep[2 * lane] = stA ? 0.f : 1.f;
          if (vB) pi.keep[2 * lane + 1] = stB ? 0.f : 1.f;
          const uint64_t starts = spread_bits(__ballot_sync(0xffffffffu, stA)) | (spread_bits(__ballot_sync(0xffffffffu, stB)) << 1);
          const bool endA = vA && (2 * lane + 1 == nc || stB);
          const bool endB = vB && (2 * lane + 2 == nc || ((starts >> (2 * lane + 2)) & 1));
          if (endA) {
            const int k = __popcll(starts & ((2ull << (2 * lane)) - 1)) - 1;
            pi.rend[k] = 2 * lane;
            pi.rtgt[k] = tA;
          }
          if (endB) {
            const int k = __popcll(starts & ((2ull << (2 * lane + 1)) - 1)) - 1;
            pi.rend[k] = 2 * lane + 1;
            pi.rtgt[k] = tB;
          }
          if (lane == 0) {
            const int h = (nc + 1) / 2;
            const uint64_t later = h >= 64 ? 0ull : starts & (~0ull << h);
            pi.starts = starts;
            pi.nruns = __popcll(starts);
            pi.split = later ? __ffsll((long long)later) - 1 : nc;
          }
        }
        const float csA = srcA >= 0 ? Msc[srcA] : 0.f, csB = srcB >= 0 ? Msc[srcB] : 0.f;
        for (int g0 = 2 * h; g0 < ng; g0 += 2 * G::GPS) {
          uint4 vh[2][G::U], vl[2][G::U];
          int facg[2];
#pragma unroll
          for (int gg = 0; gg < 2; ++gg) {
            const int j = 8 * (g0 + gg) + o;
            const int s1 = __shfl_sync(0xffffffffu, srcA, j >> 1), s2 = __shfl_sync(0xffffffffu, srcB, j >> 1);
            const int f1 = __shfl_sync(0xffffffffu, facA, j >> 1), f2 = __shfl_sync(0xffffffffu, facB, j >> 1);
            const int src = (j & 1) ? s2 : s1;
            facg[gg] = (j & 1) ? f2 : f1;
            // odd quarter-turns read the copy with the odd-order pairs swapped
            const int64_t base = src >= 0 ? (int64_t)(facg[gg] & 1) * vstride + (int64_t)src * KP : 0;
#pragma unroll
            for (int u = 0; u < G::U; ++u) {
              const int kc = 4 * u + cq;
              vh[gg][u] = vl[gg][u] = make_uint4(0, 0, 0, 0);
              if (src >= 0 && kc < G::KC) {
                vh[gg][u] = __ldg(reinterpret_cast<const uint4*>(Mh + base) + kc);
                vl[gg][u] = __ldg(reinterpret_cast<const uint4*>(Ml + base) + kc);
              }
            }
          }
#pragma unroll
          for (int gg = 0; gg < 2; ++gg) {
            const int j = 8 * (g0 + gg) + o;
#pragma unroll
            for (int u = 0; u < G::U; ++u) {
              const int kc = 4 * u + cq;
              if (kc >= G::KC) continue;
              const uint4 sg = s_sgn[kc * 16 + facg[gg]];
              const uint32_t off = canon16(j, 8 * kc, KP);
              *(uint4*)(bh + off) = make_uint4(vh[gg][u].x ^ sg.x, vh[gg][u].y ^ sg.y, vh[gg][u].z ^ sg.z, vh[gg][u].w ^ sg.w);
              *(uint4*)(bh + G::B_HALF + off) = make_uint4(vl[gg][u].x ^ sg.x, vl[gg][u].y ^ sg.y, vl[gg][u].z ^ sg.z, vl[gg][u].w ^ sg.w);
            }
          }
        }
        if (h == 0) {
          if (2 * lane < nc) pi.cs[2 * lane] = csA;
          if (2 * lane + 1 < nc) pi.cs[2 * lane + 1] = csB;
          if (lane == 0) pi.n = nc;
        }
        fence_async_smem();
        __syncwarp();
        mbar_arrive(&full[s]);
      }
    }
  } else if (lane == 0) {
    // ---------------- issue: the class operator when the class changes, then the chunk's MMAs
    int i = 0, ncls = 0;
    bool a_pending = false;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int a0 = co[c], a1 = co[c + 1];
      if (a0 == a1) continue;
      // the previous class's MMAs must have completed before its operator is replaced
      if (i > 0 && !mbar_wait_abortable(&done[(i - 1) % G::STAGES], (uint32_t)((i - 1) / G::STAGES) & 1, abort_flag)) {
        ok = false;
        break;
      }
      bulk_load(sA, reps16 + (size_t)c * lo_off, 2u * (uint32_t)lo_off, bar_a);   // lo_off bytes = lo_off/2 elements per half
      a_pending = true;
      if (!mbar_wait_abortable(bar_a, (uint32_t)ncls & 1, abort_flag)) { ok = false; break; }
      a_pending = false;
      ++ncls;
      for (int q0 = a0; q0 < a1; q0 += NCHK, ++i) {
        const int s = i % G::STAGES;
        const uint32_t ph = (uint32_t)(i / G::STAGES) & 1;
        if (!mbar_wait_abortable(&full[s], ph, abort_flag)) { ok = false; break; }
        if (i >= G::STAGES && !mbar_wait_abortable(&tempty[s], ph ^ 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const int nn = (pinfo[s].n + 15) & ~15;
        // the second tile holds rows 128..(p+1)²-1 (16 at p = 11): M = 64 halves its tensor time;
        // its rows 0-15 sit in lanes 0-15 of the first lane quadrant, as with M = 128
        const uint32_t id = instr_desc(nn), id1 = instr_desc(nn, 64);
        const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB + s * G::STAGE_BYTES);
#pragma unroll 2
        for (int ks = 0; ks < KP / 16; ++ks) {
          const uint32_t ko = (uint32_t)ks * 2 * CORE;   // 16 FP16 along K: two core matrices
          const uint64_t dbh = umma_desc(b_base + ko, G::SBO), dbl = umma_desc(b_base + G::B_HALF + ko, G::SBO);
#pragma unroll
          for (int t = 0; t < MT; ++t) {
            const uint32_t ah = a_base + (uint32_t)(t * 16 * G::SBO) + ko;
            const uint64_t dah = umma_desc(ah, G::SBO), dal = umma_desc(ah + (uint32_t)lo_off, G::SBO);
            const uint32_t td = tmem + (uint32_t)((s * MT + t) * NCHK);
            const uint32_t it = t == 0 ? id : id1;
            mma_f16(td, dah, dbh, it, ks > 0 ? 1u : 0u);
            mma_f16(td, dah, dbl, it, 1u);
            mma_f16(td, dal, dbh, it, 1u);
          }
        }
        mma_commit(&done[s]);
      }
    }
    if (!ok) {
      // give the work already issued a bounded time to finish before the memory is released
      if (a_pending) mbar_wait(bar_a, (uint32_t)ncls & 1);
      if (i > 0) mbar_wait(&done[(i - 1) % G::STAGES], (uint32_t)((i - 1) / G::STAGES) & 1);
    }
  }
  if (!ok) *abort_flag = 1;
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// the multipoles of every node, scaled by a power of two so that the largest entry of the
// column lies in [2^13, 2^14), as FP16 head and tail (one warp per node), twice: as they are and
// with the two entries of every odd-order pair swapped (vstride further); Msc = the inverse scale
__global__ void k_split16(const double* __restrict__ M, int nnodes, int NP, int LD, int KP, int64_t vstride,
                          uint16_t* __restrict__ Mh, uint16_t* __restrict__ Ml, float* __restrict__ Msc) {
  const int node = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (node >= nnodes) return;
  const double* m = M + (int64_t)node * LD;
  double mx = 0.0;
  for (int k = lane; k < NP; k += 32) mx = fmax(mx, fabs(m[k]));
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int e = 0;
  if (mx > 0.0 && mx <= 1.7e308) {                 // finite and nonzero; otherwise unscaled (0 or non-finite)
    int ex;
    frexp(mx, &ex);                                // mx = f·2^ex, f ∈ [0.5, 1)
    e = 14 - ex;                                   // mx·2^e ∈ [2^13, 2^14)
    e = max(-100, min(100, e));                    // keeps the inverse scale inside FP32's range
  }
  for (int k = lane; k < KP; k += 32) {
    int n, mm, part;
    coef_nmp(k, n, mm, part);
    const int ks = (part != 0 && (mm & 1)) ? (part == 1 ? k + 1 : k - 1) : k;
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      const int kk = v ? ks : k;
      const double x = k < NP ? ldexp(m[kk], e) : 0.0;
      const __half h = __double2half(x);
      const __half l = __double2half(x - (double)__half2float(h));
      Mh[v * vstride + (int64_t)node * KP + k] = __half_as_ushort(h);
      Ml[v * vstride + (int64_t)node * KP + k] = __half_as_ushort(l);
    }
  }
  if (lane == 0) Msc[node] = (float)ldexp(1.0, -e);
}

}  // namespace

// the signs of the source-side permutation for (p+1)² = np: per 16-byte core column kc, D4h
// element g and 32-bit word, 0x8000 in each FP16 half that is negated (the swaps of odd
// quarter-turns are in the multipole copy the gather reads)
std::vector<uint32_t> build_sign16(int np) {
  const int KC = kp_of(np) / 8;
  std::vector<uint32_t> sg((size_t)KC * 16 * 4, 0);
  for (int k = 0; k < np; ++k) {
    const uint32_t mask = perm_mask(k, false);
    for (int g = 0; g < 16; ++g)
      if ((mask >> (2 * g)) & 2) sg[((size_t)(k / 8) * 16 + g) * 4 + (k & 7) / 2] |= (k & 1) ? 0x80000000u : 0x8000u;
  }
  return sg;
}

// the class operators of the mixed path: per class, every row scaled by a power of two (its
// largest entry in [2^13, 2^14)) and split into FP16 head then tail, in the canonical K-major
// layout of the tensor-core M2L; rsc = the inverse row scales [class][row]
void build_reps16(const HostOperators& op, std::vector<uint16_t>& h, std::vector<float>& rsc) {
  const int np = op.np, LD = op.ld;
  const int KP = kp_of(np), rows = rows_of(np);
  const size_t half = (size_t)rows * KP;             // elements of one half (head or tail) of a class
  // per class: row-scaled head then tail in the canonical K-major layout; inverse row scales
  h.assign((size_t)NCLASS * 2 * half, 0);
  rsc.assign((size_t)NCLASS * np, 1.0f);
  for (int c = 0; c < NCLASS; ++c) {
    uint16_t* hi = &h[(size_t)c * 2 * half];
    uint16_t* lo = hi + half;
    const double* A = &op.reps[(size_t)c * LD * LD];   // column-major: A[r, k] at k·LD + r
    for (int r = 0; r < np; ++r) {
      // the two rows of an (n, m) pair share their scale: the read-back swaps them
      int n, m, part;
      coef_nmp(r, n, m, part);
      const int r2 = part == 0 ? r : (part == 1 ? r + 1 : r - 1);
      double mx = 0.0;
      for (int k = 0; k < np; ++k) mx = std::max(mx, std::max(std::fabs(A[(size_t)k * LD + r]), std::fabs(A[(size_t)k * LD + r2])));
      int e = 0;
      if (mx > 0.0) {
        int ex;
        std::frexp(mx, &ex);
        e = 14 - ex;
      }
      rsc[(size_t)c * np + r] = (float)std::ldexp(1.0, -e);
      for (int k = 0; k < np; ++k) {
        const double a = std::ldexp(A[(size_t)k * LD + r], e);
        const __half ah = __double2half(a);
        const __half al = __double2half(a - (double)__half2float(ah));
        const uint32_t off = canon16(r, k, KP) / 2;
        hi[off] = __half_as_ushort(ah);
        lo[off] = __half_as_ushort(al);
      }
    }
  }
}

void prepare_mixed_operators(Cache& C) {
  if (C.split_ready) return;
  const int np = C.np;
  require(np <= NPMAX, FMMB_ERR_UNSUPPORTED, "the mixed path is built for p ≤ 11");
  // the gather's lane octets and the read-back warps exchange partners inside 32 entries
  for (int k = GROUP; k < np; k += GROUP) {
    int n, m, part;
    coef_nmp(k, n, m, part);
    require(part != 2, FMMB_ERR_UNSUPPORTED, "the mixed path does not support this order");
  }
  std::vector<uint16_t> h;
  std::vector<float> rsc;
  build_reps16(C.host, h, rsc);
  std::vector<uint32_t> perm = build_sign16(np);
  to_device(C.reps16, h, C.ctx->stream);
  to_device(C.row_scale, rsc, C.ctx->stream);
  to_device(C.perm16, perm, C.ctx->stream);
  FMMB_CUDA(cudaStreamSynchronize(C.ctx->stream));
  C.split_ready = true;
}

namespace {
template <int KP, int MT>
void launch_tc(State& S, int nb) {
  using G = TcCfg<KP, MT>;
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  const int lo_off = rows_of(C.np) * KP * 2;
  FMMB_CUDA(cudaFuncSetAttribute(k_m2l_tc<KP, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  k_m2l_tc<KP, MT><<<nb, G::THREADS, G::SMEM, P.ctx->stream>>>(P.blocks.p, P.cls_off.p, P.pairs.p, C.reps16.p, C.row_scale.p,
                                                               C.perm16.p, P.d_m2l_scale.p, C.np, C.ld, lo_off, (int64_t)P.nnodes * KP, S.Mh.p,
                                                               S.Ml.p, S.Msc.p, S.Pl.p, S.err.p);
  FMMB_LAUNCH_CHECK();
}
}  // namespace

void m2l_mixed(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  const int nb = (int)P.h_blocks.size();
  if (nb == 0) return;
  const int KP = kp_of(C.np);
  const size_t ne = (size_t)P.nnodes * KP;
  if (S.Mh.n < 2 * ne) { S.Mh.alloc(2 * ne); S.Ml.alloc(2 * ne); }
  if (S.Msc.n < (size_t)P.nnodes) S.Msc.alloc(P.nnodes);
  if (!S.err.p) S.err.alloc(1);
  k_split16<<<(unsigned)(((int64_t)P.nnodes * 32 + 255) / 256), 256, 0, s>>>(S.M.p, P.nnodes, C.np, C.ld, KP, (int64_t)ne, S.Mh.p, S.Ml.p,
                                                                              S.Msc.p);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), s));
  switch (KP) {
    case 16: launch_tc<16, 1>(S, nb); break;
    case 32: launch_tc<32, 1>(S, nb); break;
    case 48: launch_tc<48, 1>(S, nb); break;
    case 64: launch_tc<64, 1>(S, nb); break;
    case 96: launch_tc<96, 1>(S, nb); break;
    case 112: launch_tc<112, 1>(S, nb); break;
    case 128: launch_tc<128, 1>(S, nb); break;
    case 144: launch_tc<144, 2>(S, nb); break;
    default: throw Error(FMMB_ERR_UNSUPPORTED, "the mixed path does not support this order");
  }
}

int mixed_error_flag(State& S) {
  if (!S.err.p) return 0;
  return read_one(S.err.p, S.plan->ctx->stream);
}

}  // namespace fmmb
