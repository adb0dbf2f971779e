// The mixed path's M2L on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// Same work decomposition as the FP64 kernel (one CTA per block of targets, the block's far
// pairs grouped by symmetry class, src/device_passes.jl:565-580 / harmonics.jl:589-645), with
// the class product on the tensor cores in three-term split precision: every operand x is
// split into a TF32 head and a TF32 tail, x ≈ hi(x) + lo(x) (22 significant bits), and
//   A·B ≈ hi(A)·hi(B) + hi(A)·lo(B) + lo(A)·hi(B)
// accumulated in FP32 in tensor memory. Per CTA:
//   - the class representative, split and laid out on the host in the UMMA K-major canonical
//     layout (8-row × 16-byte core matrices), arrives by one bulk copy (cp.async.bulk, no
//     tensor map, no multicast) into shared memory;
//   - each chunk of ≤ 64 pairs is gathered with the source-side signed permutation from an
//     FP32 copy of the multipoles, split, and written in the same canonical layout;
//   - one elected thread issues the 16 K-steps × 3 MMAs (M = 128, N = chunk rounded to 16,
//     K = 8 each) and commits them to an mbarrier;
//   - four warps read the accumulator back (tcgen05.ld 32x32b: thread = output row), apply
//     the target-side signed permutation with one warp shuffle (the two entries of an
//     (n, m) pair are adjacent rows of one warp for p ≤ 10), sum the consecutive pairs of a
//     target and update its FP64 partial local once (the block owns its targets: no atomics).
// Every wait on an mbarrier is bounded: after the limit the CTA records an error in a device
// flag, frees its tensor memory and returns; the host turns the flag into FMMB_ERR_TIMEOUT.
#include <cstring>

#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int KT = 128;           // padded expansion length (rows of A, K of the product)
constexpr int NCH_MAX = 64;       // pairs per MMA chunk
constexpr int CORE = 128;         // bytes of one 8 × 16 B core matrix
constexpr int KCH = KT / 4;       // 16-byte K-chunks per row (fp32)
constexpr int A_BYTES = KT * KT * 4;             // one split half of a representative
constexpr int B_BYTES = NCH_MAX * KT * 4;        // one split half of a chunk
constexpr unsigned long long SPIN_LIMIT = 1ull << 26;

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
  d |= (uint64_t)((saddr >> 4) & 0x3fff);            // start address
  d |= (uint64_t)((CORE >> 4) & 0x3fff) << 16;       // leading byte offset: next core matrix along K
  d |= (uint64_t)(((KCH * CORE) >> 4) & 0x3fff) << 32;  // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                            // descriptor version (sm_100)
  return d;                                          // base offset 0, no swizzle
}

// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = n
__device__ __forceinline__ uint32_t instr_desc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t a = smem_u32(bar);
  for (unsigned long long it = 0; it < SPIN_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
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

// the partner row of row i in the real storage: the other part of the same (n, m), or i for m = 0
__device__ __forceinline__ int partner_row(int i) {
  int n = (int)sqrtf((float)i + 0.5f);
  while (n * n > i) --n;
  while ((n + 1) * (n + 1) <= i) ++n;
  int r = i - n * n;
  if (r == 0) return i;
  return (r & 1) ? i + 1 : i - 1;
}

constexpr int TC_THREADS = 128;
constexpr size_t TC_SMEM = 2 * (size_t)A_BYTES + 2 * (size_t)B_BYTES + 4 * NCH_MAX * sizeof(int) + 64;

__global__ void __launch_bounds__(TC_THREADS, 1)
k_m2l_tc(const int4* __restrict__ blocks, const int* __restrict__ cls_off, const int2* __restrict__ pairs,
         const float* __restrict__ reps_split, const int16_t* __restrict__ gidx, const int8_t* __restrict__ gsgn,
         const int16_t* __restrict__ sidx, const int8_t* __restrict__ ssgn, const double* __restrict__ m2l_scale, int NP,
         int LD, const float* __restrict__ Mf, double* __restrict__ Pl, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sA = sm;                          // hi then lo, A_BYTES each
  unsigned char* sB = sm + 2 * A_BYTES;            // hi then lo, B_BYTES each
  int* ps = (int*)(sB + 2 * B_BYTES);              // pair source, far index, target
  int* pf = ps + NCH_MAX;
  int* pt = pf + NCH_MAX;
  uint64_t* bars = (uint64_t*)(pt + NCH_MAX);     // [0] operator load, [1] MMA done (8-byte aligned)
  uint32_t* tmem_slot = (uint32_t*)(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const double alpha = m2l_scale[b.x];
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(NCH_MAX));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  uint32_t ph_a = 0, ph_m = 0;
  bool ok = true;
  const int my_row = tid;                      // TMEM lane = output row
  const int prt = partner_row(my_row);
  const int src_lane = prt - 32 * warp;        // the partner lies in the same warp for rows < 121

  for (int c = 0; c < NCLASS && ok; ++c) {
    const int a0 = co[c], a1 = co[c + 1];
    if (a0 == a1) continue;
    // the class operator (the previous class's MMAs have completed: waited below)
    if (tid == 0) bulk_load(sA, reps_split + (size_t)c * 2 * KT * KT, 2 * A_BYTES, &bars[0]);
    for (int q0 = a0; q0 < a1 && ok; q0 += NCH_MAX) {
      const int nc = min(NCH_MAX, a1 - q0);
      const int nn = (nc + 15) & ~15;        // MMA N: a multiple of 16
      if (tid < NCH_MAX) {
        if (tid < nc) {
          int2 pr = pairs[b.w + q0 + tid];
          ps[tid] = pr.x; pf[tid] = pr.y >> 8; pt[tid] = pr.y & 0xff;
        } else { ps[tid] = -1; pf[tid] = 0; pt[tid] = -1; }
      }
      __syncthreads();
      // gather B: warp w takes columns w, w+4, ...; lane l the K-chunk l (k = 4l..4l+3)
      for (int j = warp; j < nn; j += 4) {
        float4 hi = make_float4(0, 0, 0, 0), lo = make_float4(0, 0, 0, 0);
        if (j < nc) {
          const int f = pf[j];
          const float* m = Mf + (int64_t)ps[j] * LD;
          float v[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            int k = 4 * lane + e;
            int gi = k < LD ? gidx[f * LD + k] : -1;
            v[e] = gi >= 0 ? (float)gsgn[f * LD + k] * m[gi] : 0.0f;
          }
          hi = make_float4(tf32_round(v[0]), tf32_round(v[1]), tf32_round(v[2]), tf32_round(v[3]));
          lo = make_float4(tf32_round(v[0] - hi.x), tf32_round(v[1] - hi.y), tf32_round(v[2] - hi.z), tf32_round(v[3] - hi.w));
        }
        uint32_t off = canon_off(j, 4 * lane);
        *(float4*)(sB + off) = hi;
        *(float4*)(sB + B_BYTES + off) = lo;
      }
      fence_async_smem();
      __syncthreads();
      if (q0 == a0) {                                  // the operator is in shared memory
        ok = __syncthreads_and(mbar_wait(&bars[0], ph_a));
        ph_a ^= 1;
        if (!ok) break;
      }
      if (tid == 0) {
        tc_fence_after();
        const uint32_t id = instr_desc(nn);
        const uint32_t aa = smem_u32(sA), bb = smem_u32(sB);
#pragma unroll 1
        for (int s = 0; s < KT / 8; ++s) {
          const uint32_t ko = s * 2 * CORE;
          mma_tf32(tmem, umma_desc(aa + ko), umma_desc(bb + ko), id, s > 0 ? 1u : 0u);
          mma_tf32(tmem, umma_desc(aa + ko), umma_desc(bb + B_BYTES + ko), id, 1u);
          mma_tf32(tmem, umma_desc(aa + A_BYTES + ko), umma_desc(bb + ko), id, 1u);
        }
        mma_commit(&bars[1]);
      }
      ok = __syncthreads_and(mbar_wait(&bars[1], ph_m));   // uniform across the CTA
      ph_m ^= 1;
      if (!ok) break;
      tc_fence_after();
      // epilogue: row my_row of the accumulator, nn columns
      int cur = -1;
      double run = 0.0;
      for (int c0 = 0; c0 < nn; c0 += 16) {
        float d[16];
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, d);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int qq = c0 + e;
          const float other = __shfl_sync(0xffffffffu, d[e], src_lane & 31);
          if (qq < nc && my_row < NP) {
            const int f = pf[qq], t = pt[qq];
            if (t != cur) {
              if (cur >= 0) Pl[(int64_t)(b.y + cur) * LD + my_row] += alpha * run;
              cur = t;
              run = 0.0;
            }
            const int si = sidx[f * LD + my_row];
            run += (double)ssgn[f * LD + my_row] * (double)(si == my_row ? d[e] : other);
          }
        }
      }
      if (cur >= 0) Pl[(int64_t)(b.y + cur) * LD + my_row] += alpha * run;
      tc_fence_before();
      __syncthreads();
    }
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCH_MAX));
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
      for (int i = 0; i < C.np; ++i) {
        double a = C.host.reps[(size_t)c * LD * LD + (size_t)k * LD + i];   // column-major: A[i, k]
        float ah = tf32_round((float)a);
        float al = tf32_round((float)(a - (double)ah));
        uint32_t off = canon_off(i, k) / 4;
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
  int nb = (int)P.h_blocks.size();
  if (nb == 0) return;
  size_t ne = (size_t)P.nnodes * C.ld;
  if (S.Mf.n < ne) S.Mf.alloc(ne);
  if (!S.err.p) S.err.alloc(1);
  k_to_f32<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(S.M.p, (int64_t)ne, S.Mf.p);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), s));
  FMMB_CUDA(cudaFuncSetAttribute(k_m2l_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  k_m2l_tc<<<nb, TC_THREADS, TC_SMEM, s>>>(P.blocks.p, P.cls_off.p, P.pairs.p, C.reps_split.p, C.gidx.p, C.gsgn.p, C.sidx.p,
                                          C.ssgn.p, P.d_m2l_scale.p, C.np, C.ld, S.Mf.p, S.Pl.p, S.err.p);
  FMMB_LAUNCH_CHECK();
}

int mixed_error_flag(State& S) {
  if (!S.err.p) return 0;
  return read_one(S.err.p, S.plan->ctx->stream);
}

}  // namespace fmmb
