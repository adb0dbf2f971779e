// M2L of the plain FP64 path: one launch for all levels, one CTA per block of targets
// (src/device_passes.jl:565-580, the class-wise translation of harmonics.jl:531-645).
//
// Per symmetry class and chunk of ≤ NB pairs of the block:
//   gather  G = P_sᵀ M_src for the chunk's columns into shared memory ([column][entry], one
//           coalesced load per lane and entry quartet, the D4h permutation computed from the
//           offset's group element, partner entries by warp shuffles)
//   product Y = A_class G, FP64 FMA, A streamed through shared memory in K-chunks of 16,
//           each thread a RPT × CPT register tile
//   scatter (P_t Y) summed over the consecutive pairs of each target, one update of the
//           target's partial local per run (the block owns its targets: deterministic, no atomics)
#include "d4h.cuh"
#include "passes.cuh"

namespace fmmb {

__constant__ int c_d4h[NFAR];

void upload_d4h(const HostOperators& h, cudaStream_t s) {
  std::vector<int> fac(h.d4h.begin(), h.d4h.end());
  require(fac.size() == NFAR, FMMB_ERR_DEVICE, "the D4h factor table has the wrong size");
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_d4h, fac.data(), sizeof(int) * NFAR, 0, cudaMemcpyHostToDevice, s));
}

namespace {

template <int LD, int NB>
__global__ void __launch_bounds__(256) k_m2l_f64(const int4* __restrict__ blocks, const int* __restrict__ cls_off,
                                                 const int2* __restrict__ pairs, const double* __restrict__ reps,
                                                 const double* __restrict__ m2l_scale, int NP, const double* __restrict__ M,
                                                 double* __restrict__ Pl) {
  constexpr int BK = 16, RPT = LD / 16, CPT = NB / 16, GS = LD + 1;
  // entry quartets per lane (LD = 64: lanes ≥ 16 idle). A pair of entries never straddles a
  // multiple of 128 (entries 128, 256, 384 are real parts or m = 0), so the partner of a
  // lane's first and last entry is always in the neighbouring lane of the same quartet row.
  constexpr int Q = (LD + 127) / 128;
  extern __shared__ double sm[];
  double* As = sm;                 // [BK][LD]
  double* G = As + BK * LD;        // [NB][GS]: the gathered columns, then the product
  int* ps = (int*)(G + NB * GS);
  int* pf = ps + NB;
  int* pt = pf + NB;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const double alpha = m2l_scale[b.x];
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);
  const int kmax = (NP + BK - 1) / BK * BK;
  for (int c = 0; c < NCLASS; ++c) {
    const int a0 = co[c], a1 = co[c + 1];
    const double* A = reps + (int64_t)c * LD * LD;
    for (int q0 = a0; q0 < a1; q0 += NB) {
      const int nc = min(NB, a1 - q0);
      __syncthreads();
      for (int j = tid; j < NB; j += 256) {
        if (j < nc) {
          const int2 pr = pairs[b.w + q0 + j];
          ps[j] = pr.x; pf[j] = pr.y >> 8; pt[j] = pr.y & 0xff;
        } else { ps[j] = -1; pf[j] = 0; pt[j] = -1; }
      }
      __syncthreads();
      // gather: warp w the columns w, w + 8, ...; lane l the entries 4(l + 32 r) .. + 3
      for (int j = warp; j < nc; j += 8) {
        const int fac = c_d4h[pf[j]];
        const double* src = M + (int64_t)ps[j] * LD;
#pragma unroll
        for (int r = 0; r < Q; ++r) {
          const int k0 = 4 * (lane + 32 * r);
          double a[4];
          if (k0 < LD) {
            const double2 u = __ldg(reinterpret_cast<const double2*>(src + k0));
            const double2 w = __ldg(reinterpret_cast<const double2*>(src + k0 + 2));
            a[0] = u.x; a[1] = u.y; a[2] = w.x; a[3] = w.y;
          } else { a[0] = a[1] = a[2] = a[3] = 0.0; }
          const double nxt = __shfl_down_sync(0xffffffffu, a[0], 1);
          const double prv = __shfl_up_sync(0xffffffffu, a[3], 1);
          if (k0 < LD) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              int n, m, part;
              coef_nmp(k0 + e, n, m, part);
              const int q = (-m * (fac & 3)) & 3;
              const bool sw = part != 0 && (q & 1);
              double x = a[e];
              if (sw) x = part == 1 ? (e < 3 ? a[e + 1] : nxt) : (e > 0 ? a[e - 1] : prv);
              G[j * GS + k0 + e] = k0 + e < NP ? (perm_sign(part, q, n + m, fac) < 0 ? -x : x) : 0.0;
            }
          }
        }
      }
      for (int j = nc + warp; j < NB; j += 8)
        for (int k = lane; k < LD; k += 32) G[j * GS + k] = 0.0;
      double acc[RPT][CPT];
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < CPT; ++cc) acc[r][cc] = 0.0;
      for (int k0 = 0; k0 < kmax; k0 += BK) {
        __syncthreads();
        for (int e = tid; e < BK * LD; e += 256) {
          const int i = e % LD, k = e / LD;
          As[k * LD + i] = A[(int64_t)(k0 + k) * LD + i];
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < BK; ++k) {
          double av[RPT], bv[CPT];
#pragma unroll
          for (int r = 0; r < RPT; ++r) av[r] = As[k * LD + ty + 16 * r];
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc) bv[cc] = G[(tx + 16 * cc) * GS + k0 + k];
#pragma unroll
          for (int r = 0; r < RPT; ++r)
#pragma unroll
            for (int cc = 0; cc < CPT; ++cc) acc[r][cc] = fma(av[r], bv[cc], acc[r][cc]);
        }
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int cc = 0; cc < CPT; ++cc) G[(tx + 16 * cc) * GS + ty + 16 * r] = acc[r][cc];
      __syncthreads();
      // scatter: thread j owns entry j of the targets' partial locals
      for (int j = tid; j < NP; j += 256) {
        int n, m, part;
        coef_nmp(j, n, m, part);
        const int partner = part == 0 ? j : (part == 1 ? j + 1 : j - 1);
        int cur = -1;
        double run = 0.0;
        for (int qq = 0; qq < nc; ++qq) {
          const int t = pt[qq], fac = c_d4h[pf[qq]];
          if (t != cur) {
            if (cur >= 0) Pl[(int64_t)(b.y + cur) * LD + j] += alpha * run;
            cur = t;
            run = 0.0;
          }
          const int q = (m * (fac & 3)) & 3;
          const bool sw = part != 0 && (q & 1);
          const double y = G[qq * GS + (sw ? partner : j)];
          run += perm_sign(sw ? 3 - part : part, q, n + m, fac) < 0 ? -y : y;
        }
        if (cur >= 0) Pl[(int64_t)(b.y + cur) * LD + j] += alpha * run;
      }
    }
  }
}

template <int LD, int NB>
void launch(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  const int nb = (int)P.h_blocks.size();
  if (nb == 0) return;
  const size_t smem = sizeof(double) * (16 * LD + NB * (LD + 1)) + sizeof(int) * 3 * NB;
  auto kern = k_m2l_f64<LD, NB>;
  FMMB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<nb, 256, smem, P.ctx->stream>>>(P.blocks.p, P.cls_off.p, P.pairs.p, C.reps.p, P.d_m2l_scale.p, C.np, S.M.p, S.Pl.p);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

void m2l_f64(State& S) {
  switch (S.plan->cache->ld) {
    case 64: launch<64, 64>(S); break;
    case 128: launch<128, 64>(S); break;
    case 192: launch<192, 32>(S); break;
    case 256: launch<256, 32>(S); break;
    case 320: launch<320, 16>(S); break;
    case 384: launch<384, 16>(S); break;
    case 448: launch<448, 16>(S); break;
    default: throw Error(FMMB_ERR_UNSUPPORTED, "no M2L kernel for this expansion length");
  }
}

}  // namespace fmmb
