// The mixed path's M2L on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// Same work decomposition as the FP64 kernel (one CTA per block of targets, the block's far
// pairs grouped by symmetry class; src/device_passes.jl:565-580, harmonics.jl:589-645), with
// the class product on the tensor cores in three-term split precision: every operand x is
// split into a TF32 head and a TF32 tail, x ≈ hi(x) + lo(x) (22 significant bits), and
//   A·B ≈ hi(A)·hi(B) + hi(A)·lo(B) + lo(A)·hi(B)
// accumulated in FP32 in tensor memory.
//
// Per CTA, three roles connected by mbarriers over a two-stage ring (warp specialisation):
//   - warps 4-7 gather chunk i (≤ 48 pairs of one class: P_sᵀ M_src from the FP32 multipoles,
//     one float4 per lane, split into head and tail) into B stage i mod 2, in the UMMA K-major
//     canonical layout (8-row × 16-byte core matrices), and arrive on full[s];
//   - one thread of warp 8 loads the class representative (split and laid out on the host)
//     by one bulk copy (cp.async.bulk, no tensor map, no multicast) when the class changes,
//     after the previous class's MMAs completed; then per chunk waits full[s] and tempty[s],
//     issues 16 K-steps × 3 MMAs (M = 128, N = chunk rounded to 16, K = 8) into accumulator
//     stage s of tensor memory and commits them to done[s];
//   - warps 0-3 wait done[s], read the accumulator back (tcgen05.ld 32x32b: thread = output
//     row), apply P_t, sum the consecutive pairs of each target and add the sum to its FP64
//     partial local with a reduction (the block owns its targets and each entry has one
//     writing thread, so the additions apply in program order: deterministic), then arrive on
//     tempty[s], which frees the stage for the next gather and MMAs.
// The signed permutations are per-thread 32-bit masks indexed by the offset's D4h element
// (2 bits per element: swap the (n, m) pair's entries, negate).
// Every wait on an mbarrier is bounded and also gives up when another role has given up; the
// CTA then waits (bounded) for the copies and MMAs it issued, records an error in a device
// flag, frees its tensor memory and returns; the host turns the flag into FMMB_ERR_TIMEOUT.
#include <cstring>

#include "d4h.cuh"
#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int KT = 128;           // padded expansion length (rows of A, K of the product)
constexpr int NCH_MAX = 48;       // pairs per MMA chunk
constexpr int CORE = 128;         // bytes of one 8 × 16 B core matrix
constexpr int KCH = KT / 4;       // 16-byte K-chunks per row (fp32)
constexpr int A_BYTES = KT * KT * 4;             // one split half of a representative
constexpr int B_BYTES = NCH_MAX * KT * 4;        // one split half of a chunk
constexpr unsigned long long SPIN_LIMIT = 1ull << 26;
constexpr uint64_t WAIT_NS = 1000000000ull;  // one second: a wait in a working pipeline takes microseconds
constexpr int TC_THREADS = 288;   // 9 warps: read-back, gather, issue
constexpr int TMEM_COLS = 128;

// canonical K-major offset (bytes) of element (row, k) in a tile with KT columns
__host__ __device__ __forceinline__ uint32_t canon_off(int row, int k) {
  return (uint32_t)(((row >> 3) * KCH + (k >> 2)) * CORE + (row & 7) * 16 + (k & 3) * 4);
}

// round-to-nearest (ties away) to TF32, as cvt.rna.tf32.f32 does
__host__ __device__ __forceinline__ float tf32_round(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fff);               // start address
  d |= (uint64_t)((CORE >> 4) & 0x3fff) << 16;          // leading byte offset: next core matrix along K
  d |= (uint64_t)(((KCH * CORE) >> 4) & 0x3fff) << 32;  // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                               // descriptor version (sm_100)
  return d;                                             // base offset 0, no swizzle
}

// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = n
__device__ __forceinline__ uint32_t instr_desc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
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

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
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

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// the 16 D4h elements' (swap, negate) codes for one entry, 2 bits per element; the source
// side (gather, phase conjugated) or the target side (scatter, sign of the partner when swapped)
__device__ __forceinline__ uint32_t perm_mask(int k, bool target) {
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

struct __align__(16) PairInfo { int src[NCH_MAX]; int fac[NCH_MAX]; int tgt[NCH_MAX]; int n; };

constexpr int STAGES = 2;            // B operand / accumulator ring
constexpr int STAGE_COLS = 64;       // tensor-memory columns per accumulator stage
constexpr int STAGE_BYTES = 2 * B_BYTES;
constexpr size_t TC_SMEM = 2 * (size_t)A_BYTES + STAGES * (size_t)STAGE_BYTES + STAGES * sizeof(PairInfo) +
                           NFAR * sizeof(int) + 16 * sizeof(uint64_t);

// roles: warps 0-3 read back and scatter (thread = output row), warps 4-7 gather, warp 8 issues
constexpr int N_EPI = 128, N_PROD = 128;

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

__global__ void __launch_bounds__(TC_THREADS, 1)
k_m2l_tc(const int4* __restrict__ blocks, const int* __restrict__ cls_off, const int2* __restrict__ pairs,
         const float* __restrict__ reps_split, const double* __restrict__ m2l_scale, int NP, int LD,
         const float* __restrict__ Mf, double* __restrict__ Pl, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sA = sm;                                         // hi then lo, A_BYTES each
  unsigned char* sB = sm + 2 * A_BYTES;                           // stage s: hi at s·STAGE_BYTES, lo after it
  PairInfo* pinfo = (PairInfo*)(sB + STAGES * STAGE_BYTES);       // per stage
  int* s_d4h = (int*)(pinfo + STAGES);
  uint64_t* bars = (uint64_t*)(s_d4h + NFAR);                     // 8-byte aligned: NFAR is even
  uint64_t* bar_a = bars;                                         // operator load
  uint64_t* full = bars + 1;                                      // [STAGES] gathered (N_PROD arrivals)
  uint64_t* done = bars + 1 + STAGES;                             // [STAGES] MMAs complete (commit)
  uint64_t* tempty = bars + 1 + 2 * STAGES;                       // [STAGES] read back (N_EPI arrivals)
  uint32_t* tmem_slot = (uint32_t*)(bars + 1 + 3 * STAGES);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);

  for (int f = tid; f < NFAR; f += TC_THREADS) s_d4h[f] = c_d4h[f];
  if (tid == 0) {
    mbar_init(bar_a, 1);
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], N_PROD);
      mbar_init(&done[s], 1);
      mbar_init(&tempty[s], N_EPI);
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

  if (warp < 4) {
    // ---------------- read back and scatter: thread = output row
    const int row = tid;
    const double alpha = m2l_scale[b.x];
    const uint32_t emask = perm_mask(row, true);
    int en, em, epart;
    coef_nmp(row, en, em, epart);
    const int partner = epart == 0 ? row : (epart == 1 ? row + 1 : row - 1);
    const int src_lane = (partner - 32 * warp) & 31;   // the partner is in the same warp for rows < 121
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int a0 = co[c], a1 = co[c + 1];
      for (int q0 = a0; q0 < a1; q0 += NCH_MAX, ++i) {
        const int s = i % STAGES;
        const uint32_t ph = (uint32_t)(i / STAGES) & 1;
        const bool w = mbar_wait_abortable(&full[s], ph, abort_flag) && mbar_wait_abortable(&done[s], ph, abort_flag);
        if (!__all_sync(0xffffffffu, w)) { ok = false; break; }   // the warp leaves together (tcgen05.ld is warp-wide)
        tc_fence_after();
        const PairInfo& pi = pinfo[s];
        const int nc = pi.n;
        float d[NCH_MAX];
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(s * STAGE_COLS);
#pragma unroll
        for (int c16 = 0; c16 < NCH_MAX / 16; ++c16) tmem_ld16(ta + 16 * c16, d + 16 * c16);
        tmem_wait_ld();
        int cur = -1;
        float run = 0.f;
#pragma unroll
        for (int q = 0; q < NCH_MAX; ++q) {
          if (q < nc) {                                   // uniform across the warp
            const float other = __shfl_sync(0xffffffffu, d[q], src_lane);
            if (row < NP) {
              const int t = pi.tgt[q];
              if (t != cur) {
                if (cur >= 0) atomicAdd(&Pl[(int64_t)(b.y + cur) * LD + row], alpha * (double)run);
                cur = t;
                run = 0.f;
              }
              const uint32_t code = emask >> (2 * pi.fac[q]);
              const float y = (code & 1) ? other : d[q];
              run += (code & 2) ? -y : y;
            }
          }
        }
        // the only writer of these entries: the reductions apply in program order
        if (cur >= 0) atomicAdd(&Pl[(int64_t)(b.y + cur) * LD + row], alpha * (double)run);
        tc_fence_before();
        mbar_arrive(&tempty[s]);
      }
    }
  } else if (warp < 8) {
    // ---------------- gather: warp w the columns (w − 4) + 4u; lane l the entries 4l..4l+3
    const int pt = tid - N_EPI, pw = warp - 4;
    uint32_t gmask[4];
    int gpart[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int n, m;
      gmask[e] = perm_mask(4 * lane + e, false);
      coef_nmp(4 * lane + e, n, m, gpart[e]);
    }
    int i = 0;
    for (int c = 0; c < NCLASS && ok; ++c) {
      const int a0 = co[c], a1 = co[c + 1];
      for (int q0 = a0; q0 < a1; q0 += NCH_MAX, ++i) {
        const int s = i % STAGES;
        if (i >= STAGES) {
          const bool w = mbar_wait_abortable(&tempty[s], (uint32_t)(i / STAGES - 1) & 1, abort_flag);
          if (!__all_sync(0xffffffffu, w)) { ok = false; break; }   // the warp leaves together (shuffles below)
        }
        const int nc = min(NCH_MAX, a1 - q0), nn = (nc + 15) & ~15;
        PairInfo& pi = pinfo[s];
        // lane u < 12 of warp w reads the pair of column w + 4u and publishes it for the other roles
        int my_src = 0, my_fac = 0;
        if (lane < NCH_MAX / 4) {
          const int j = pw + 4 * lane;
          if (j < nc) {
            const int2 pr = pairs[b.w + q0 + j];
            my_src = pr.x;
            my_fac = s_d4h[pr.y >> 8];
            pi.src[j] = pr.x; pi.fac[j] = my_fac; pi.tgt[j] = pr.y & 0xff;
          } else {
            pi.src[j] = -1; pi.fac[j] = 0; pi.tgt[j] = -1;
          }
        }
        if (pt == 0) pi.n = nc;
        unsigned char* bh = sB + s * STAGE_BYTES;
        constexpr int U = NCH_MAX / 4;
        float4 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = pw + 4 * u;
          const int src = __shfl_sync(0xffffffffu, my_src, u);
          v[u] = (j < nc && 4 * lane < LD) ? __ldg(reinterpret_cast<const float4*>(Mf + (int64_t)src * LD) + lane)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = pw + 4 * u;
          if (j >= nn) continue;                          // uniform across the warp
          const float nxt = __shfl_down_sync(0xffffffffu, v[u].x, 1);
          const float prv = __shfl_up_sync(0xffffffffu, v[u].w, 1);
          const int fac = __shfl_sync(0xffffffffu, my_fac, u);
          const float a[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
          float g[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const uint32_t code = gmask[e] >> (2 * fac);
            // the partner of entry 4l+e: the next entry for a real part, the previous for an imaginary part
            const float pv = gpart[e] == 1 ? (e < 3 ? a[e + 1] : nxt) : (e > 0 ? a[e - 1] : prv);
            g[e] = (code & 1) ? pv : a[e];
            if (code & 2) g[e] = -g[e];
          }
          const float4 hi = make_float4(tf32_round(g[0]), tf32_round(g[1]), tf32_round(g[2]), tf32_round(g[3]));
          const float4 lo = make_float4(tf32_round(g[0] - hi.x), tf32_round(g[1] - hi.y), tf32_round(g[2] - hi.z),
                                        tf32_round(g[3] - hi.w));
          const uint32_t off = canon_off(j, 4 * lane);
          *(float4*)(bh + off) = hi;
          *(float4*)(bh + B_BYTES + off) = lo;
        }
        fence_async_smem();
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
      if (i > 0 && !mbar_wait_abortable(&done[(i - 1) % STAGES], (uint32_t)((i - 1) / STAGES) & 1, abort_flag)) { ok = false; break; }
      bulk_load(sA, reps_split + (size_t)c * 2 * KT * KT, 2 * A_BYTES, bar_a);
      a_pending = true;
      if (!mbar_wait_abortable(bar_a, (uint32_t)ncls & 1, abort_flag)) { ok = false; break; }
      a_pending = false;
      ++ncls;
      for (int q0 = a0; q0 < a1; q0 += NCH_MAX, ++i) {
        const int s = i % STAGES;
        const uint32_t ph = (uint32_t)(i / STAGES) & 1;
        if (!mbar_wait_abortable(&full[s], ph, abort_flag)) { ok = false; break; }
        if (i >= STAGES && !mbar_wait_abortable(&tempty[s], ph ^ 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const int nn = (pinfo[s].n + 15) & ~15;
        const uint32_t id = instr_desc(nn);
        unsigned char* bh = sB + s * STAGE_BYTES;
        const uint64_t dah = umma_desc(smem_u32(sA)), dal = umma_desc(smem_u32(sA + A_BYTES));
        const uint64_t dbh = umma_desc(smem_u32(bh)), dbl = umma_desc(smem_u32(bh + B_BYTES));
        const uint32_t td = tmem + (uint32_t)(s * STAGE_COLS);
#pragma unroll 4
        for (int k = 0; k < KT / 8; ++k) {
          const uint64_t ko = (uint64_t)(k * 2 * CORE) >> 4;   // the start address advances 2 core matrices
          mma_tf32(td, dah + ko, dbh + ko, id, k > 0 ? 1u : 0u);
          mma_tf32(td, dah + ko, dbl + ko, id, 1u);
          mma_tf32(td, dal + ko, dbh + ko, id, 1u);
        }
        mma_commit(&done[s]);
      }
    }
    if (!ok) {
      // give the work already issued a bounded time to finish before the memory is released
      if (a_pending) mbar_wait(bar_a, (uint32_t)ncls & 1);
      if (i > 0) mbar_wait(&done[(i - 1) % STAGES], (uint32_t)((i - 1) / STAGES) & 1);
    }
  }
  if (!ok) *abort_flag = 1;
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(err, 1);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

__global__ void k_to_f32(const double* __restrict__ in, int64_t n, float* __restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}

}  // namespace

void prepare_mixed_operators(Cache& C) {
  if (C.split_ready) return;
  require(C.np <= KT, FMMB_ERR_UNSUPPORTED, "the mixed path is built for p ≤ 10");
  const int LD = C.ld;
  // per class: the hi then the lo half, each KT × KT in the canonical K-major layout
  std::vector<float> h((size_t)NCLASS * 2 * KT * KT, 0.0f);
  for (int c = 0; c < NCLASS; ++c) {
    float* hi = &h[(size_t)c * 2 * KT * KT];
    float* lo = hi + KT * KT;
    for (int k = 0; k < C.np; ++k)
      for (int r = 0; r < C.np; ++r) {
        const double a = C.host.reps[(size_t)c * LD * LD + (size_t)k * LD + r];   // column-major: A[r, k]
        const float ah = tf32_round((float)a);
        const float al = tf32_round((float)(a - (double)ah));
        const uint32_t off = canon_off(r, k) / 4;
        hi[off] = ah;
        lo[off] = al;
      }
  }
  to_device(C.reps_split, h, C.ctx->stream);
  FMMB_CUDA(cudaStreamSynchronize(C.ctx->stream));
  C.split_ready = true;
}

void m2l_mixed(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  const int nb = (int)P.h_blocks.size();
  if (nb == 0) return;
  const size_t ne = (size_t)P.nnodes * C.ld;
  if (S.Mf.n < ne) S.Mf.alloc(ne);
  if (!S.err.p) S.err.alloc(1);
  k_to_f32<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(S.M.p, (int64_t)ne, S.Mf.p);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), s));
  FMMB_CUDA(cudaFuncSetAttribute(k_m2l_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  k_m2l_tc<<<nb, TC_THREADS, TC_SMEM, s>>>(P.blocks.p, P.cls_off.p, P.pairs.p, C.reps_split.p, P.d_m2l_scale.p, C.np, C.ld,
                                          S.Mf.p, S.Pl.p, S.err.p);
  FMMB_LAUNCH_CHECK();
}

int mixed_error_flag(State& S) {
  if (!S.err.p) return 0;
  return read_one(S.err.p, S.plan->ctx->stream);
}

}  // namespace fmmb
