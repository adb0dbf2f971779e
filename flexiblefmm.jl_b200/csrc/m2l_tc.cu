// The mixed path's M2L on the 5th-generation tensor cores (tcgen05, kind::f16).
//
// The block decomposition of the FP64 kernel (one CTA per block of ≤ 128 targets, the block's far
// pairs grouped by symmetry class; src/device_passes.jl:565-580, harmonics.jl:589-645), with the
// class product on the tensor cores in three-term split precision over FP16:
//   - the multipoles of each level are scaled by a power of two (so that the level's largest
//     entry lies in [2^13, 2^14)) and split into an FP16 head and tail, x·2^e ≈ hi + lo (22
//     significant bits over FP16's range);
//   - every row of a class operator is scaled the same way (per class and (n, m) pair of rows);
//   - A·B ≈ hi(A)·hi(B) + hi(A)·lo(B) + lo(A)·hi(B), accumulated in FP32 in tensor memory;
//     FP16 products are exact in FP32. The read-back removes both scales (exact powers of two).
//
// The product is oriented so that one MMA serves every target of the block: M = 128 is the
// block's targets (one TMEM lane each), N = (p+1)² rounded to 16 is the output rows, K likewise.
// A class runs in rounds; round r gathers each target's r-th pair of the class (a zero row where
// it has fewer), so a target's pairs all land in its own lane and its class sum is a running sum
// in one thread: D = A·Bᵀ with A = the gathered source multipoles (source-side signed
// permutation applied) and B = the class operator, resident in shared memory for the class.
//
// Per CTA, four roles connected by mbarriers (warp specialisation):
//   - two setup warps write, per round (alternately), each target's pair (source node, D4h
//     element, source scale) into a ring of round records;
//   - gather warps build K-step slabs of A (128 rows × 16 FP16, head and tail, in the UMMA
//     K-major canonical layout) into a ring: 8 lanes write the 8 rows of one 128-byte core
//     matrix; odd quarter-turn rotations read a second copy of the multipoles in which the two
//     entries of every odd-order pair are swapped, and the source-side signs cost one XOR;
//   - one thread loads the class operator (head and tail, laid out on the host) with one bulk
//     copy (cp.async.bulk, no tensor map, no multicast) when the class changes, after the
//     previous class's MMAs completed; then per K-step issues three MMAs (M = 128, N, K = 16)
//     into one of two accumulator stages in tensor memory;
//   - read-back warps (thread = target; two warps per TMEM lane quadrant, each half of the
//     columns) apply the target-side permutation of the pair's element (odd-m entries take their
//     partner's value for odd rotations, signs by XOR) and the source scale, and add the row into
//     the target's class sums, kept in tensor memory; at the class's last round they add the sums,
//     with the row scales and the level factor W_ref/w, to the FP64 partial locals with
//     reductions, transposed through shared memory so that each covers consecutive rows.
// Every wait on an mbarrier is bounded and also gives up when another role has given up; the
// CTA then waits (bounded) for the copies and MMAs it issued, records an error in a device
// flag, frees its tensor memory and returns; the host turns the flag into FMMB_ERR_TIMEOUT.
#include <atomic>
#include <cstring>

#include <cuda_fp16.h>

#include "d4h.cuh"
#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int CORE = 128;         // bytes of one 8 × 16 B core matrix
constexpr int NPMAX = 144;        // (p+1)² supported: p ≤ 11
constexpr unsigned long long SPIN_LIMIT = 1ull << 26;
constexpr uint64_t WAIT_NS = 1000000000ull;  // one second: a wait in a working pipeline takes microseconds
constexpr int TMEM_COLS = 512;

__host__ __device__ constexpr int kp_of(int np) { return (np + 15) / 16 * 16; }          // K, padded to the MMA's K
__host__ __device__ constexpr int rows_of(int np) { return np > 128 ? 128 + (np - 128 + 7) / 8 * 8 : 128; }  // rows stored

// canonical K-major offset (bytes) of FP16 element (row, k) in a tile with kp columns
__host__ __device__ __forceinline__ uint32_t canon16(int row, int k, int kp) {
  return (uint32_t)((row >> 3) * (kp / 8) * CORE + (k >> 3) * CORE + (row & 7) * 16 + (k & 7) * 2);
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

// a wait bounded in time (wait_ns of the global timer) and in polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t wait_ns) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (unsigned long long it = 0; it < SPIN_LIMIT; ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 63) == 63) {
      const uint64_t t = global_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 > wait_ns) return false;
    }
  }
  return false;
}

// a bounded wait that also gives up when another role aborted
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t* bar, uint32_t parity, volatile int* abort_flag, uint64_t wait_ns) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (unsigned long long it = 0; it < SPIN_LIMIT; ++it) {
    if (mbar_try(a, parity)) return true;
    if ((it & 63) == 63) {
      if (*abort_flag) return false;
      const uint64_t t = global_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 > wait_ns) break;
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

// 16 bytes from global memory into shared memory, asynchronously (L2 only); the bytes past
// src_bytes (0 or 16) are zero-filled
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// a reduction without a returned value (an atomicAdd whose result is unused may still wait for one)
__device__ __forceinline__ void red_add_f64(double* p, double v) {
  asm volatile("red.global.add.f64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "d"(v) : "memory");
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

// ---------------------------------------------------------------- the kernel
// One CTA per block of ≤ 128 targets, one TMEM lane (one row of the MMA's M = 128) per target.
// The block's far pairs are taken class by class; a class runs in rounds, round r gathering every
// target's r-th pair of the class (a zero row where a target has fewer), so that each target's
// pairs land in its own lane and its sum over the class is a per-thread running sum: no sums
// across lanes, no runs. Per round the product is D = A·Bᵀ with A = the gathered multipoles
// (128 × K, the pairs' source-side permutation applied) and B = the class operator (N = (p+1)²
// rounded to 16 rows × K, resident in shared memory for the whole class): one MMA per K-step
// and split term covers all 128 targets and every output row.
constexpr int LANES = 128;                 // targets per block tile: the MMA's M
constexpr int RING_KSTEPS = 12;            // K-steps of A staged in the ring (12 × 8 KB)
constexpr int GW = 8;                      // gather warps
constexpr int RBQ = 4;                     // read-back warps per TMEM lane quadrant
constexpr int RBW = 4 * RBQ;               // read-back warps 0..15 (warp w reads lanes 32·(w % 4)..)
constexpr int W_GATHER = RBW;              // gather warps 16..23
constexpr int SW = 2;                      // round setup warps (alternate rounds)
constexpr int W_SETUP = RBW + GW;          // round setup warps 24, 25
constexpr int W_ISSUE = RBW + GW + SW;     // MMA issuing warp 26
constexpr int THREADS = 32 * (W_ISSUE + 1);

// one round: per target (lane) the source node of its pair (-1: none) and the pair's D4h element
struct __align__(16) RoundRec {
  int src[LANES];
  int fac[LANES];
};

// per 16-row group g of the real storage: the rows whose target-side permutation may swap them
// with their partner (Re/Im entries of odd order m), and of those the Re rows (partner below them
// at +1; Im rows take theirs at −1). Odd-m pairs never straddle a multiple of 4, so a row and
// its partner always share a group.
__host__ __device__ constexpr int row_n(int k) {
  int n = 0;
  while ((n + 1) * (n + 1) <= k) ++n;
  return n;
}
__host__ __device__ constexpr uint32_t swap16(int g) {
  uint32_t m = 0;
  for (int e = 0; e < 16; ++e) {
    const int k = 16 * g + e, r = k - row_n(k) * row_n(k), mm = (r + 1) >> 1;
    if (r != 0 && (mm & 1)) m |= 1u << e;
  }
  return m;
}
__host__ __device__ constexpr uint32_t re16(int g) {
  uint32_t m = 0;
  for (int e = 0; e < 16; ++e) {
    const int k = 16 * g + e, r = k - row_n(k) * row_n(k);
    if (r != 0 && (r & 1)) m |= 1u << e;
  }
  return m;
}

template <int KP>
struct Cfg {
  static constexpr int KC = KP / 8;                        // 16-byte core columns along K
  static constexpr int KS = KP / 16;                       // K-steps of 16
  // a slab holds SK K-steps of A (a barrier wait, a fence and a commit per slab cost about as
  // much as three MMAs, so slabs span up to three K-steps); KS / SK slabs per round
  static constexpr int SK = KS % 3 == 0 ? 3 : (KS % 2 == 0 ? 2 : 1);
  static constexpr int SPR = KS / SK;
  static constexpr int NSLAB = RING_KSTEPS / SK;
  // gather warps in use: a warp that waits for slab k's buffer (consumed fill k − NSLAB) must
  // already have seen fill k − 2·NSLAB consumed, or the wait on that barrier's phase parity could
  // pass a phase early; its previous slab k − NGW waited for k − NGW − NSLAB, so NGW ≤ NSLAB
  static constexpr int NGW = GW < NSLAB ? GW : NSLAB;
  // round records in the ring. A gather warp may work up to (RING_KSTEPS + KS − 2) / KS rounds ahead
  // of the oldest unconsumed slab's round; the ring must be longer than that, or a wait on a
  // record's phase parity could see the record's previous-but-one phase as complete
  static constexpr int NREC_MIN = (RING_KSTEPS + KS - 2) / KS + 2;
  static constexpr int NREC = NREC_MIN > 6 ? NREC_MIN : 6;
  static constexpr int NG = KP / 16;                       // 16-column groups of an accumulator
  static constexpr int NW = (KP + 31) / 32;                // 32-row words of the sign masks
  static constexpr int OPR = KP > 128 ? KP : 128;          // operator rows stored (rows_of)
  static constexpr int OP_BYTES = 2 * OPR * KP * 2;        // head and tail of one class
  static constexpr int SLAB_HALF = LANES * 16 * 2 * SK;    // SK K-steps of 128 rows, FP16
  static constexpr int SLAB = 2 * SLAB_HALF;
  static constexpr int SBO_A = 2 * SK * CORE;                // bytes between 8-row groups of a slab
  // TMEM columns: accumulator stage 0 at 0, the class sums at SCOL, stage 1 at D1 (64-aligned)
  static constexpr int SCOL = (KP + 31) / 32 * 32;
  static constexpr int D1 = (SCOL + KP + 63) / 64 * 64;
  static_assert(D1 + KP <= TMEM_COLS, "tensor memory");
  static constexpr int SLAB_OFF = (OP_BYTES + 1023) / 1024 * 1024;
  static constexpr int REC_OFF = SLAB_OFF + NSLAB * SLAB;
  static constexpr int XP_OFF = REC_OFF + NREC * (int)sizeof(RoundRec);   // per read-back warp 32 × 17 floats
  static constexpr int SGN_OFF = XP_OFF + RBW * 32 * 17 * 4;
  static constexpr int D4H_OFF = SGN_OFF + 16 * KC * 16;
  static constexpr int NEG_OFF = D4H_OFF + NFAR * 4;
  static constexpr int MSK_OFF = NEG_OFF + NW * 16 * 4;      // swap16, re16 per group
  static constexpr int BAR_OFF = (MSK_OFF + 2 * NG * 4 + 7) / 8 * 8;
  // slab full/empty, record full/empty, accumulator full/empty, operator loaded/free
  static constexpr int NBAR = 2 * NSLAB + 2 * NREC + 4 + 2;
  static constexpr int SMEM = BAR_OFF + NBAR * 8 + 16;
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// the read-back of one round for column groups [g0, g1) of lane quadrant q: the accumulator row
// of this lane's pair, the target-side permutation of its D4h element (rot: odd-m entries take
// their partner's value; s_neg: the negated rows per element), times the source scale, into the
// class sums;
// sw/re: per group the swappable rows and the Re rows among them (swap16, re16)
// the read-back of one round for column groups [g0, g1) of lane quadrant q: the accumulator row
// of this lane's pair, the target-side permutation of its D4h element (rot: odd-m entries take
// their partner's value; s_neg: the negated rows per element), into the class sums; sw/re: per
// group the swappable rows and the Re rows among them (swap16, re16)
template <int KP>
__device__ __forceinline__ void rb_round(uint32_t tq, int g0, int g1, int d, bool first, bool rot, const uint32_t* s_neg, int fac,
                                         const uint32_t* sw, const uint32_t* re) {
  using G = Cfg<KP>;
#pragma unroll 1
  for (int g = g0; g < g1; ++g) {
    const uint32_t SW = rot ? sw[g] : 0u, RE = re[g];
    float dv[16], sv[16];
    tmem_ld16(tq + (uint32_t)((d ? G::D1 : 0) + 16 * g), dv);
    if (!first) tmem_ld16(tq + (uint32_t)(G::SCOL + 16 * g), sv);
    tmem_wait_ld();
    const uint32_t nw = s_neg[(g >> 1) * 16 + fac] >> (16 * (g & 1));   // this group's 16 negation bits
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const float yp = ((RE >> e) & 1u) ? dv[e < 15 ? e + 1 : e] : dv[e > 0 ? e - 1 : e];
      float y = ((SW >> e) & 1u) ? yp : dv[e];
      y = __uint_as_float(__float_as_uint(y) ^ ((nw << (31 - e)) & 0x80000000u));
      sv[e] = first ? y : sv[e] + y;
    }
    tmem_st16(tq + (uint32_t)(G::SCOL + 16 * g), sv);
  }
}

// the class sums of lane quadrant q, column groups [g0, g1): times the row scales and the level
// factor, added to the targets' FP64 partial locals, transposed through xp so that each
// reduction covers 16 consecutive rows of two targets
template <int KP>
__device__ __forceinline__ void rb_write(uint32_t tq, int g0, int g1, float* xp, int lane, int q, unsigned anymask, int nodes0,
                                         int count, int NP, int LD, const float* __restrict__ rsc, double alpha,
                                         double* __restrict__ Pl) {
  using G = Cfg<KP>;
#pragma unroll 1
  for (int g = g0; g < g1; ++g) {
    float sv[16];
    tmem_ld16(tq + (uint32_t)(G::SCOL + 16 * g), sv);
    tmem_wait_ld();
#pragma unroll
    for (int e = 0; e < 16; ++e) xp[lane * 17 + e] = sv[e];
    __syncwarp();
    const int e = lane & 15, r = 16 * g + e;
    const double rs = r < NP ? alpha * (double)rsc[r] : 0.0;
#pragma unroll 4
    for (int it = 0; it < 16; ++it) {
      const int t = 2 * it + (lane >> 4), tgt = 32 * q + t;
      if (!((anymask >> (2 * it)) & 3u)) continue;                 // uniform: neither target had a pair
      if (((anymask >> t) & 1u) && tgt < count && r < NP)
        red_add_f64(&Pl[(int64_t)(nodes0 + tgt) * LD + r], rs * (double)xp[t * 17 + e]);
    }
    __syncwarp();
  }
}

// The launch's control: the bounded waits' time limit, and (tests only) one K-step slab whose
// gather never reports it full, so that the waits run out and the kernel reports the abort
struct TcCtl {
  uint64_t wait_ns;
  long long stall_slab;     // -1: none
};

// blocks: (level, first node, count, pair base); cls_off: per block the class offsets of its
// pairs; rtab/rounds: the round table (per class and target count << 16 | offset; per class the
// rounds); reps16_lv/rsc_lv: per level the class operators (head, tail) and their inverse row
// scales;
// perm16: the source-side sign words; Mh/Ml/lsc: the split multipoles (two copies vstride
// apart) and the inverse scale of each level
template <int KP>
__global__ void __launch_bounds__(THREADS, 1)
k_m2l_tc(const int4* __restrict__ blocks, const int* __restrict__ cls_off, const int2* __restrict__ pairs,
         const int* __restrict__ rtab, const int* __restrict__ rounds, int TB, const uint64_t* __restrict__ reps16_lv,
         const uint64_t* __restrict__ rsc_lv, const uint32_t* __restrict__ perm16, const double* __restrict__ m2l_scale,
         int NP, int LD, int lo_off, int64_t vstride, const uint16_t* __restrict__ Mh, const uint16_t* __restrict__ Ml,
         const float* __restrict__ lsc, double* __restrict__ Pl, int* __restrict__ err, TcCtl ctl) {
  using G = Cfg<KP>;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sOp = sm;                                     // class operator: head rows, then the tail at lo_off
  unsigned char* sSlab = sm + G::SLAB_OFF;                     // slab s: head at s·SLAB, tail after it
  RoundRec* recs = (RoundRec*)(sm + G::REC_OFF);
  float* xps = (float*)(sm + G::XP_OFF);
  uint4* s_sgn = (uint4*)(sm + G::SGN_OFF);                    // [KC][16]
  int* s_d4h = (int*)(sm + G::D4H_OFF);
  uint32_t* s_neg = (uint32_t*)(sm + G::NEG_OFF);              // [NW][16]: bit r & 31 of word r >> 5, per element
  uint32_t* s_sw = (uint32_t*)(sm + G::MSK_OFF);               // [NG] swappable rows of each 16-row group
  uint32_t* s_re = s_sw + G::NG;                               // [NG] their Re rows
  uint64_t* bars = (uint64_t*)(sm + G::BAR_OFF);
  uint64_t* sfull = bars;                                      // [NSLAB] gathered (1 arrival)
  uint64_t* sempty = bars + G::NSLAB;                          // [NSLAB] consumed by the MMAs (commit)
  uint64_t* rfull = sempty + G::NSLAB;                         // [NREC] written by a setup warp
  uint64_t* rempty = rfull + G::NREC;                          // [NREC] released by the read-back (RBW arrivals)
  uint64_t* dfull = rempty + G::NREC;                          // [2] accumulator ready (commit)
  uint64_t* dempty = dfull + 2;                                // [2] accumulator read (RBW arrivals)
  uint64_t* opfull = dempty + 2;                               // operator loaded (bulk copy)
  uint64_t* opfree = opfull + 1;                               // the class's MMAs complete (commit)
  uint32_t* tmem_slot = (uint32_t*)(bars + G::NBAR);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const uint16_t* reps16 = reinterpret_cast<const uint16_t*>(reps16_lv[b.x & 255]);   // the block level's operators
  const float* row_scale = reinterpret_cast<const float*>(rsc_lv[b.x & 255]);
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);
  const int* nr = rounds + (int64_t)blockIdx.x * NCLASS;
  const int* rt = rtab + (int64_t)blockIdx.x * NCLASS * TB;
  const uint64_t wns = ctl.wait_ns;

  for (int f = tid; f < NFAR; f += THREADS) s_d4h[f] = c_d4h[f];
  for (int e = tid; e < 16 * G::KC; e += THREADS) s_sgn[e] = reinterpret_cast<const uint4*>(perm16)[e];
  for (int g = tid; g < G::NG; g += THREADS) { s_sw[g] = swap16(g); s_re[g] = re16(g); }
  if (warp < G::NW) {                                          // the target-side negations, one ballot per element
    const int r = 32 * warp + lane;
    const uint32_t mask = r < NP ? perm_mask(r, true) : 0u;
    for (int fac = 0; fac < 16; ++fac) {
      const unsigned bal = __ballot_sync(0xffffffffu, (mask >> (2 * fac + 1)) & 1u);
      if (lane == 0) s_neg[warp * 16 + fac] = bal;
    }
  }
  if (tid == 0) {
    for (int s = 0; s < G::NSLAB; ++s) { mbar_init(&sfull[s], 1); mbar_init(&sempty[s], 1); }
    for (int s = 0; s < G::NREC; ++s) { mbar_init(&rfull[s], 1); mbar_init(&rempty[s], RBW); }
    for (int s = 0; s < 2; ++s) { mbar_init(&dfull[s], 1); mbar_init(&dempty[s], RBW); }
    mbar_init(opfull, 1);
    mbar_init(opfree, 1);
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

  if (warp < RBW) {
    // ---------------- read-back: lane quadrant q, one of RBQ ranges of the column groups
    const int q = warp & 3, part = warp >> 2, j = 32 * q + lane;
    const int g0 = part * G::NG / RBQ, g1 = (part + 1) * G::NG / RBQ;
    const uint32_t tq = tmem + ((uint32_t)(32 * q) << 16);
    float* xp = xps + warp * 32 * 17;
    const double alpha = m2l_scale[b.x & 255] * (double)lsc[b.x >> 8];   // the level factor, the segment's scale
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int R = nr[c];
      bool any = false;
      for (int r = 0; r < R; ++r, ++i) {
        const int d = i & 1, rc = i % G::NREC;
        const bool w = mbar_wait_abortable(&rfull[rc], (uint32_t)(i / G::NREC) & 1, abort_flag, wns) &&
                       mbar_wait_abortable(&dfull[d], (uint32_t)(i >> 1) & 1, abort_flag, wns);
        if (!__all_sync(0xffffffffu, w)) { ok = false; break; }   // the warp leaves together (tcgen05.ld is warp-wide)
        tc_fence_after();
        const RoundRec& rec = recs[rc];
        const int fac = rec.fac[j];
        any |= rec.src[j] >= 0;
        rb_round<KP>(tq, g0, g1, d, r == 0, (fac & 1) != 0, s_neg, fac, s_sw, s_re);
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&dempty[d]);
        if (r == R - 1)
          rb_write<KP>(tq, g0, g1, xp, lane, q, __ballot_sync(0xffffffffu, any), b.y, b.z, NP, LD, row_scale + (size_t)c * NP,
                       alpha, Pl);
        __syncwarp();
        if (lane == 0) mbar_arrive(&rempty[rc]);
      }
    }
  } else if (warp < W_SETUP) {
    // ---------------- gather: warp gw builds slabs gw, gw + NGW, ...: lane (o = lane & 7, sub = lane >> 3)
    // writes row o of every 8-row group for core column sub & 1 of the K-step, head (sub < 2) or tail
    const int gw = warp - W_GATHER, o = lane & 7, kc = (lane >> 3) & 1, half = lane >> 4;
    const uint16_t* Mx = half ? Ml : Mh;
    int total = 0;
    for (int c = 0; c < NCLASS; ++c) total += nr[c];
    const long long nslabs = (long long)total * G::SPR;
    for (long long k = gw; gw < G::NGW && k < nslabs && ok; k += G::NGW) {
      const int i = (int)(k / G::SPR), ks0 = (int)(k % G::SPR) * G::SK, rc = i % G::NREC, s = (int)(k % G::NSLAB);
      bool w = mbar_wait_abortable(&rfull[rc], (uint32_t)(i / G::NREC) & 1, abort_flag, wns);
      if (w && k >= G::NSLAB) w = mbar_wait_abortable(&sempty[s], (uint32_t)(k / G::NSLAB - 1) & 1, abort_flag, wns);
      if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
      const RoundRec& rec = recs[rc];
      unsigned char* dst0 = sSlab + s * G::SLAB + half * G::SLAB_HALF + kc * CORE + o * 16;
      // the 16 rows' chunks of the slab's K-steps copied asynchronously (zero rows where a target
      // has no pair), then the source-side signs applied in place; odd quarter-turns read the copy
      // with the odd-order pairs swapped
      uint64_t facs = 0;
      uint32_t valid = 0;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int row = 8 * u + o, src = rec.src[row], fac = rec.fac[row];
        facs |= (uint64_t)fac << (4 * u);
        valid |= (src >= 0 ? 1u : 0u) << u;
        const uint16_t* g = src >= 0 ? Mx + (int64_t)(fac & 1) * vstride + (int64_t)src * KP + 8 * (2 * ks0 + kc) : Mx;
#pragma unroll
        for (int j = 0; j < G::SK; ++j) cp_async16(dst0 + u * G::SBO_A + j * 2 * CORE, g + (src >= 0 ? 16 * j : 0), src >= 0 ? 16u : 0u);
      }
      cp_async_wait_all();
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        if (!((valid >> u) & 1u)) continue;
        const int fac = (int)((facs >> (4 * u)) & 15);
#pragma unroll
        for (int j = 0; j < G::SK; ++j) {
          uint4* pv = (uint4*)(dst0 + u * G::SBO_A + j * 2 * CORE);
          const uint4 sg = s_sgn[(2 * (ks0 + j) + kc) * 16 + fac];
          const uint4 v = *pv;
          *pv = make_uint4(v.x ^ sg.x, v.y ^ sg.y, v.z ^ sg.z, v.w ^ sg.w);
        }
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0 && k != ctl.stall_slab) mbar_arrive(&sfull[s]);
    }
  } else if (warp < W_ISSUE) {
    // ---------------- round setup (warp sw of SW takes rounds i ≡ sw mod SW): per target its r-th
    // pair of the class, its element and scale
    const int sw = warp - W_SETUP;
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int R = nr[c];
      int ent[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = lane + 32 * u;
        ent[u] = (j < TB && j < b.z) ? rt[c * TB + j] : 0;
      }
      for (int r = 0; r < R; ++r, ++i) {
        if (i % SW != sw) continue;
        const int rc = i % G::NREC;
        const bool w = i < G::NREC || mbar_wait_abortable(&rempty[rc], (uint32_t)(i / G::NREC - 1) & 1, abort_flag, wns);
        if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
        RoundRec& rec = recs[rc];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = lane + 32 * u;
          int src = -1, fac = 0;
          if (r < (ent[u] >> 16)) {
            const int2 pr = pairs[b.w + co[c] + (ent[u] & 0xffff) + r];
            src = pr.x;
            fac = s_d4h[pr.y >> 8];
          }
          rec.src[j] = src;
          rec.fac[j] = fac;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&rfull[rc]);
      }
    }
  } else if (lane == 0) {
    // ---------------- issue: the class operator when the class changes, then per round and K-step
    // three MMAs (head·head, head·tail, tail·head) of M = 128 targets, N = KP rows, K = 16
    int i = 0, ncls = 0;
    long long k = 0;
    bool a_pending = false;
    uint64_t* last_bar = nullptr;                              // the barrier of the last commit, and its parity
    uint32_t last_par = 0;
    const uint32_t idesc = instr_desc(KP, 128);
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int R = nr[c];
      if (R == 0) continue;
      // the previous class's MMAs must have completed before its operator is replaced
      if (ncls > 0 && !mbar_wait_abortable(opfree, (uint32_t)(ncls - 1) & 1, abort_flag, wns)) { ok = false; break; }
      bulk_load(sOp, reps16 + (size_t)c * lo_off, 2u * (uint32_t)lo_off, opfull);   // lo_off bytes = lo_off/2 elements per half
      a_pending = true;
      if (!mbar_wait_abortable(opfull, (uint32_t)ncls & 1, abort_flag, wns)) { ok = false; break; }
      a_pending = false;
      const uint32_t ob = smem_u32(sOp);
      for (int r = 0; r < R && ok; ++r, ++i) {
        const int d = i & 1;
        if (i >= 2 && !mbar_wait_abortable(&dempty[d], (uint32_t)((i >> 1) - 1) & 1, abort_flag, wns)) { ok = false; break; }
        const uint32_t td = tmem + (uint32_t)(d ? G::D1 : 0);
        for (int sl = 0; sl < G::SPR; ++sl, ++k) {
          const int s = (int)(k % G::NSLAB);
          if (!mbar_wait_abortable(&sfull[s], (uint32_t)(k / G::NSLAB) & 1, abort_flag, wns)) { ok = false; break; }
          tc_fence_after();
          const uint32_t ab = smem_u32(sSlab + s * G::SLAB);
#pragma unroll
          for (int j = 0; j < G::SK; ++j) {
            const int ks = sl * G::SK + j;
            const uint32_t aj = ab + (uint32_t)j * 2 * CORE;     // 16 FP16 along K: two core matrices
            const uint64_t dah = umma_desc(aj, G::SBO_A), dal = umma_desc(aj + G::SLAB_HALF, G::SBO_A);
            const uint32_t bo = ob + (uint32_t)ks * 2 * CORE;
            const uint64_t dbh = umma_desc(bo, G::KC * CORE), dbl = umma_desc(bo + (uint32_t)lo_off, G::KC * CORE);
            mma_f16(td, dah, dbh, idesc, ks > 0 ? 1u : 0u);
            mma_f16(td, dah, dbl, idesc, 1u);
            mma_f16(td, dal, dbh, idesc, 1u);
          }
          mma_commit(&sempty[s]);
          last_bar = &sempty[s];
          last_par = (uint32_t)(k / G::NSLAB) & 1;
        }
        if (!ok) break;
        mma_commit(&dfull[d]);
        last_bar = &dfull[d];
        last_par = (uint32_t)(i >> 1) & 1;
      }
      if (!ok) break;
      mma_commit(opfree);
      last_bar = opfree;
      last_par = (uint32_t)ncls & 1;
      ++ncls;
    }
    if (!ok) {
      // give the work already issued a bounded time to finish before the memory is released
      if (a_pending) mbar_wait(opfull, (uint32_t)ncls & 1, wns);
      if (last_bar) mbar_wait(last_bar, last_par, wns);
    }
  }
  if (!ok) *abort_flag = 1;
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// the largest |entry| of the multipoles of each segment (one warp per node; a plan of one point
// set has one segment per level, seg null): the bit patterns of non-negative doubles order as
// integers (a non-finite entry makes its segment's maximum non-finite, and the segment is then
// split unscaled)
__global__ void k_level_absmax(const double* __restrict__ M, const int4* __restrict__ cell, const int* __restrict__ seg,
                               int nnodes, int NP, int LD, unsigned long long* __restrict__ lvmax) {
  const int node = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (node >= nnodes) return;
  const double* m = M + (int64_t)node * LD;
  double mx = 0.0;
  for (int k = lane; k < NP; k += 32) mx = fmax(mx, fabs(m[k]));
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0 && mx != 0.0)
    atomicMax(&lvmax[seg ? seg[node] : cell[node].w], (unsigned long long)__double_as_longlong(mx));
}

// the exponent e of each level: its largest entry times 2^e lies in [2^13, 2^14); lsc = 2^-e
__device__ __forceinline__ int level_exponent(unsigned long long bits) {
  const double mx = __longlong_as_double((long long)bits);
  if (!(mx > 0.0 && mx <= 1.7e308)) return 0;     // finite and nonzero; otherwise unscaled (0 or non-finite)
  int ex;
  frexp(mx, &ex);                                  // mx = f·2^ex, f ∈ [0.5, 1)
  return max(-100, min(100, 14 - ex));             // keeps the inverse scale inside FP32's range
}
__global__ void k_level_scale(const unsigned long long* __restrict__ lvmax, int L, float* __restrict__ lsc) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < L) lsc[l] = (float)ldexp(1.0, -level_exponent(lvmax[l]));
}

// the multipoles of every node, scaled by its level's power of two, as FP16 head and tail (one
// warp per node), twice: as they are and with the two entries of every odd-order pair swapped
// (vstride further). One scale per level keeps the sums of a target's pairs in one scale (no
// per-pair factor in the read-back); an entry 2^-k of its level's largest keeps 22 significant
// bits down to k ≈ 17 and an absolute error below 2^-38 of the level's largest entry beyond.
__global__ void k_split16(const double* __restrict__ M, const int4* __restrict__ cell, const int* __restrict__ seg,
                          int nnodes, int NP, int LD, int KP, int64_t vstride, const unsigned long long* __restrict__ lvmax,
                          uint16_t* __restrict__ Mh, uint16_t* __restrict__ Ml) {
  const int node = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (node >= nnodes) return;
  const double* m = M + (int64_t)node * LD;
  const int e = level_exponent(lvmax[seg ? seg[node] : cell[node].w]);
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
  std::vector<uint32_t> perm = build_sign16(np);
  to_device(C.perm16, perm, C.ctx->stream);
  if (C.kernel != FMMB_KERNEL_YUKAWA3D) {          // Yukawa3D: the operators of each width, per level
    std::vector<uint16_t> h;
    std::vector<float> rsc;
    build_reps16(C.host, h, rsc);
    to_device(C.reps16, h, C.ctx->stream);
    to_device(C.row_scale, rsc, C.ctx->stream);
  }
  FMMB_CUDA(cudaStreamSynchronize(C.ctx->stream));
  C.split_ready = true;
}

// the per-level tables of the mixed path's operators (the cache locked by the caller): the
// cache's split operators on every level, or for Yukawa3D each level width's, split from its
// class operators (copied to the host once per width and shared by the plans that use it)
void prepare_mixed_levels(Plan& P) {
  Cache& C = *P.cache;
  if (P.d_lv_reps16.n == (size_t)P.L) return;
  cudaStream_t s = P.ctx->stream;
  std::vector<uint64_t> r16(P.L, 0), rs(P.L, 0);
  for (int l = 0; l < P.L; ++l) {
    if (C.kernel != FMMB_KERNEL_YUKAWA3D) {
      r16[l] = (uint64_t)(uintptr_t)C.reps16.p;
      rs[l] = (uint64_t)(uintptr_t)C.row_scale.p;
      continue;
    }
    if (l >= (int)P.lv_yukawa.size() || !P.lv_yukawa[l]) continue;   // no far pairs on this level
    YukawaLevel& Y = *P.lv_yukawa[l];
    std::lock_guard<std::mutex> lk(Y.mu);
    if (!Y.reps16.p) {
      HostOperators op;
      op.p = C.p; op.np = C.np; op.ld = C.ld;
      op.reps = to_host(Y.reps.p, (size_t)NCLASS * C.ld * C.ld, s);
      std::vector<uint16_t> h;
      std::vector<float> rsc;
      build_reps16(op, h, rsc);
      // held as long as the level's other operators, outside the stream-ordered pool
      const cudaStream_t keep = g_alloc_stream;
      g_alloc_stream = nullptr;
      to_device(Y.reps16, h, s);
      to_device(Y.row_scale, rsc, s);
      g_alloc_stream = keep;
      FMMB_CUDA(cudaStreamSynchronize(s));
    }
    r16[l] = (uint64_t)(uintptr_t)Y.reps16.p;
    rs[l] = (uint64_t)(uintptr_t)Y.row_scale.p;
  }
  to_device(P.d_lv_reps16, r16, s);
  to_device(P.d_lv_rsc, rs, s);
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// the bounded waits' limit and the test hook's stalled slab, for the next launches
// (fmmb_test_m2l_stall); process-wide
static std::atomic<long long> g_stall_slab{-1};
static std::atomic<uint64_t> g_wait_ns{WAIT_NS};

void set_m2l_stall(long long slab, double wait_s) {
  g_stall_slab = slab;
  g_wait_ns = wait_s > 0 ? (uint64_t)(wait_s * 1e9) : WAIT_NS;
}

namespace {
template <int KP>
void launch_tc(State& S, int nb) {
  using G = Cfg<KP>;
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  const int lo_off = rows_of(C.np) * KP * 2;
  require(P.TB <= LANES, FMMB_ERR_UNSUPPORTED, "M2L blocks hold at most 128 targets");
  FMMB_CUDA(cudaFuncSetAttribute(k_m2l_tc<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  const TcCtl ctl{g_wait_ns.load(), g_stall_slab.load()};
  k_m2l_tc<KP><<<nb, THREADS, G::SMEM, P.ctx->stream>>>(P.blocks.p, P.cls_off.p, P.pairs.p, P.rtab.p, P.rounds.p, P.TB,
                                                        P.d_lv_reps16.p, P.d_lv_rsc.p, C.perm16.p, P.d_m2l_scale.p, C.np, C.ld, lo_off,
                                                        (int64_t)P.nnodes * KP, S.Mh.p, S.Ml.p, S.Lsc.p, S.Pl.p, S.err.p, ctl);
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
  const int nseg = P.nseg;                         // one scale per segment (per level for one point set)
  const int* seg = P.ninst > 1 ? P.node_seg.p : nullptr;
  if (S.Lsc.n < (size_t)nseg) { S.Lsc.alloc(nseg); S.Lmax.alloc(nseg); }
  if (!S.err.p) {                                  // sticky until reported (mixed_error_flag clears it)
    S.err.alloc(1);
    FMMB_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), s));
  }
  const unsigned nbk = (unsigned)(((int64_t)P.nnodes * 32 + 255) / 256);
  FMMB_CUDA(cudaMemsetAsync(S.Lmax.p, 0, sizeof(unsigned long long) * nseg, s));
  k_level_absmax<<<nbk, 256, 0, s>>>(S.M.p, P.cell.p, seg, P.nnodes, C.np, C.ld, S.Lmax.p);
  FMMB_LAUNCH_CHECK();
  k_level_scale<<<(nseg + 63) / 64, 64, 0, s>>>(S.Lmax.p, nseg, S.Lsc.p);
  FMMB_LAUNCH_CHECK();
  k_split16<<<nbk, 256, 0, s>>>(S.M.p, P.cell.p, seg, P.nnodes, C.np, C.ld, KP, (int64_t)ne, S.Lmax.p, S.Mh.p, S.Ml.p);
  FMMB_LAUNCH_CHECK();
  switch (KP) {
    case 16: launch_tc<16>(S, nb); break;
    case 32: launch_tc<32>(S, nb); break;
    case 48: launch_tc<48>(S, nb); break;
    case 64: launch_tc<64>(S, nb); break;
    case 96: launch_tc<96>(S, nb); break;
    case 112: launch_tc<112>(S, nb); break;
    case 128: launch_tc<128>(S, nb); break;
    case 144: launch_tc<144>(S, nb); break;
    default: throw Error(FMMB_ERR_UNSUPPORTED, "the mixed path does not support this order");
  }
}

int mixed_error_flag(State& S) {
  if (!S.err.p) return 0;
  const int f = read_one(S.err.p, S.plan->ctx->stream);
  if (f) {
    FMMB_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), S.plan->ctx->stream));
    FMMB_CUDA(cudaStreamSynchronize(S.plan->ctx->stream));
  }
  return f;
}

}  // namespace fmmb
