// M2L of the plain FP64 path: one launch for all levels, one CTA per block of targets
// (src/device_passes.jl:565-580, the class-wise translation of harmonics.jl:531-645).
//
// Per symmetry class and chunk of ≤ NB pairs of the block:
//   gather  G = P_sᵀ M_src for the chunk's columns into shared memory ([column][entry], one
//           coalesced load per lane and entry quartet, the D4h permutation of each entry looked
//           up in a table of its swaps and signs over the 16 group elements, built once per
//           CTA; partner entries by warp shuffles)
//   product Y = A_class G on the FP64 tensor cores (mma.sync m8n8k4 f64, DMMA: there is no FP64
//           tcgen05 kind), A streamed through shared memory in K-slabs of 16 with the next slab
//           prefetched into registers; each warp an (LD/8 rows) × NB register tile
//   scatter (P_t Y) into the targets' partial locals: each target's entry takes its pairs one by
//           one in the list's order, starting from the value in memory (the block owns its
//           targets: deterministic, no atomics, and the sums do not depend on where the chunks
//           end nor on the other targets of the block); the partial locals of four targets are
//           read at once
#include "d4h.cuh"
#include "passes.cuh"

namespace fmmb {

__constant__ int c_d4h[NFAR];
__constant__ int c_faroff[NFAR * 3];   // the far offsets, source cell − target cell

void upload_d4h(const HostOperators& h, cudaStream_t s) {
  std::vector<int> fac(h.d4h.begin(), h.d4h.end());
  require(fac.size() == NFAR, FMMB_ERR_DEVICE, "the D4h factor table has the wrong size");
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_d4h, fac.data(), sizeof(int) * NFAR, 0, cudaMemcpyHostToDevice, s));
  std::vector<int> off(h.faroff.begin(), h.faroff.end());
  require(off.size() == 3 * NFAR, FMMB_ERR_DEVICE, "the far offset table has the wrong size");
  FMMB_CUDA(cudaMemcpyToSymbolAsync(c_faroff, off.data(), sizeof(int) * 3 * NFAR, 0, cudaMemcpyHostToDevice, s));
}

namespace {

// one FP64 tensor-core MMA, D(8×8) += A(8×4)·B(4×8): this lane holds A[g][t], B[t][g] and
// D[g][2t], D[g][2t+1] (g = lane / 4, t = lane % 4)
__device__ __forceinline__ void dmma(double* d, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// over the 16 D4h elements (bit f for element f): whether entry k takes its partner's value
// (low half) and whether it is negated (high half); the source side (P_sᵀ, q = −m·rot) names the
// sign by the entry's own part, the target side (P_t, q = +m·rot) by the part it reads
__device__ __forceinline__ uint32_t perm_masks(int k, bool target) {
  int n, m, part;
  coef_nmp(k, n, m, part);
  uint32_t swap = 0, neg = 0;
  for (int f = 0; f < 16; ++f) {
    const int q = ((target ? m : -m) * (f & 3)) & 3;
    const bool sw = part != 0 && (q & 1);
    swap |= (uint32_t)sw << f;
    neg |= (uint32_t)(perm_sign(target && sw ? 3 - part : part, q, n + m, f) < 0) << f;
  }
  return swap | neg << 16;
}

template <int LD, int NB>
constexpr size_t m2l_f64_smem() {
  return sizeof(double) * (16 * (LD + 4) + NB * (LD + 4)) + sizeof(int) * 4 * NB + sizeof(uint32_t) * LD + LD;
}
// two CTAs per SM where their shared memory fits (the registers are then capped at 128)
template <int LD, int NB>
constexpr int m2l_f64_ctas() { return m2l_f64_smem<LD, NB>() <= 113 * 1024 ? 2 : 1; }

template <int LD, int NB>
__global__ void __launch_bounds__(256, m2l_f64_ctas<LD, NB>()) k_m2l_f64(const int4* __restrict__ blocks, const int* __restrict__ cls_off,
                                                 const int2* __restrict__ pairs, const uint64_t* __restrict__ reps_lv,
                                                 const double* __restrict__ m2l_scale, int NP, const double* __restrict__ M,
                                                 double* __restrict__ Pl, int64_t pitch, int stokes) {
  // the expansion block of this CTA; the Stokes Ψ̂ block (the fourth) adds the coupling
  const int comp = blockIdx.y, psi = stokes && comp == 3;
  // row tiles per warp, column tiles; strides ≡ 4 (mod 16) doubles keep the fragment loads free
  // of shared-memory bank conflicts
  constexpr int BK = 16, MT = LD / 64, NT = NB / 8, GS = LD + 4, LDA = LD + 4, AL = (BK * LD + 255) / 256;
  // entry quartets per lane (LD = 64: lanes ≥ 16 idle). A pair of entries never straddles a
  // multiple of 128 (entries 128, 256, 384 are real parts or m = 0), so the partner of a
  // lane's first and last entry is always in the neighbouring lane of the same quartet row.
  constexpr int Q = (LD + 127) / 128;
  extern __shared__ double sm[];
  double* As = sm;                 // [BK][LDA]
  double* G = As + BK * LDA;       // [NB][GS]: the gathered columns, then the product
  int* ps = (int*)(G + NB * GS);
  int* pf = ps + NB;
  int* pt = pf + NB;
  int* pfac = pt + NB;               // the pairs' D4h elements
  uint32_t* smsk = (uint32_t*)(pfac + NB);   // [LD]: the gather's masks per entry (0 past NP)
  int8_t* sdir = (int8_t*)(smsk + LD);       // [LD]: where each entry's partner is (+1 Re, −1 Im, 0)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 b = blocks[blockIdx.x];
  const int level = b.x & 255;
  const double alpha = m2l_scale[level];
  const int* co = cls_off + (int64_t)blockIdx.x * (NCLASS + 1);
  const int kmax = (NP + BK - 1) / BK * BK, RT = (NP + 7) / 8;
  for (int k = tid; k < LD; k += 256) {
    int n, m, part;
    coef_nmp(k, n, m, part);
    smsk[k] = k < NP ? perm_masks(k, false) : 0u;
    sdir[k] = (int8_t)(k < NP && part != 0 ? (part == 1 ? 1 : -1) : 0);
  }
  // the scatter's entries of this thread (j = tid + 256 i): their partners and target-side masks
  constexpr int EPT = (LD + 255) / 256;
  uint32_t tmsk[EPT];
  int tpart[EPT];
#pragma unroll
  for (int i = 0; i < EPT; ++i) {
    const int j = tid + 256 * i;
    tmsk[i] = 0;
    tpart[i] = j;
    if (j < NP) {
      int n, m, part;
      coef_nmp(j, n, m, part);
      tpart[i] = part == 0 ? j : (part == 1 ? j + 1 : j - 1);
      tmsk[i] = perm_masks(j, true);
    }
  }
  for (int c = 0; c < NCLASS; ++c) {
    const int a0 = co[c], a1 = co[c + 1];
    const double* A = reinterpret_cast<const double*>(reps_lv[level]) + (int64_t)c * LD * LD;   // the level's representatives
    for (int q0 = a0; q0 < a1; q0 += NB) {
      const int nc = min(NB, a1 - q0);
      __syncthreads();
      for (int j = tid; j < NB; j += 256) {
        if (j < nc) {
          const int2 pr = pairs[b.w + q0 + j];
          ps[j] = pr.x; pf[j] = pr.y >> 8; pt[j] = pr.y & 0xff; pfac[j] = c_d4h[pr.y >> 8];
        } else { ps[j] = -1; pf[j] = 0; pt[j] = -1; pfac[j] = 0; }
      }
      __syncthreads();
      // gather: warp w the columns w, w + 8, ..., two at a time (both columns' loads in flight
      // before either is permuted); lane l the entries 4(l + 32 r) .. + 3
      for (int j0 = warp; j0 < nc; j0 += 16) {
        double a[2][Q][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + 8 * h;
          const bool on = j < nc;
          const double* src = M + (int64_t)(on ? ps[j] : 0) * pitch + (int64_t)comp * LD;
          // the Stokes Ψ̂ block: its source is Ψ̂ + o·Φ of the source box, o the far offset
          // (harmonics_stokes.jl: M2L Ψ̂_B = Ψ̂_A + o·Φ, linear in the source)
          double o3[3] = {0.0, 0.0, 0.0};
          if (psi && on)
            for (int d = 0; d < 3; ++d) o3[d] = (double)c_faroff[3 * pf[j] + d];
#pragma unroll
          for (int r = 0; r < Q; ++r) {
            const int k0 = 4 * (lane + 32 * r);
            if (on && k0 < LD) {
              const double2 u = __ldg(reinterpret_cast<const double2*>(src + k0));
              const double2 w = __ldg(reinterpret_cast<const double2*>(src + k0 + 2));
              a[h][r][0] = u.x; a[h][r][1] = u.y; a[h][r][2] = w.x; a[h][r][3] = w.y;
              if (psi) {
                const double* base = M + (int64_t)ps[j] * pitch;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const double2 u2 = __ldg(reinterpret_cast<const double2*>(base + (int64_t)d * LD + k0));
                  const double2 w2 = __ldg(reinterpret_cast<const double2*>(base + (int64_t)d * LD + k0 + 2));
                  a[h][r][0] += o3[d] * u2.x; a[h][r][1] += o3[d] * u2.y;
                  a[h][r][2] += o3[d] * w2.x; a[h][r][3] += o3[d] * w2.y;
                }
              }
            } else {
              a[h][r][0] = a[h][r][1] = a[h][r][2] = a[h][r][3] = 0.0;
            }
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = j0 + 8 * h;
          if (j >= nc) continue;                       // warp-uniform
          const int fac = pfac[j];
#pragma unroll
          for (int r = 0; r < Q; ++r) {
            const int k0 = 4 * (lane + 32 * r);
            const double nxt = __shfl_down_sync(0xffffffffu, a[h][r][0], 1);
            const double prv = __shfl_up_sync(0xffffffffu, a[h][r][3], 1);
            if (k0 < LD) {
              // a swapped entry takes its partner: the next one for a real part, the previous
              // for an imaginary part
              const uint4 mk = *reinterpret_cast<const uint4*>(smsk + k0);
              const char4 dr = *reinterpret_cast<const char4*>(sdir + k0);
              const uint32_t mm[4] = {mk.x, mk.y, mk.z, mk.w};
              const int dd[4] = {dr.x, dr.y, dr.z, dr.w};
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                double x = a[h][r][e];
                if ((mm[e] >> fac) & 1) x = dd[e] > 0 ? (e < 3 ? a[h][r][e + 1] : nxt) : (e > 0 ? a[h][r][e - 1] : prv);
                G[j * GS + k0 + e] = k0 + e < NP ? ((mm[e] >> (16 + fac)) & 1 ? -x : x) : 0.0;
              }
            }
          }
        }
      }
      for (int j = nc + warp; j < NB; j += 8)
        for (int k = lane; k < LD; k += 32) G[j * GS + k] = 0.0;
      // product Y = A·G on the FP64 tensor cores: warp w the row tiles w, w + 8, w + 16, ... below
      // the last real row (RT tiles of 8 rows; the rows past NP are zero and are not multiplied)
      // × all NB columns (NT tiles of 8), K-steps of 4; A streamed through shared memory in slabs
      // of BK rows of K, the next slab prefetched into registers
      double acc[MT][NT][2];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
      const int g = lane >> 2, t = lane & 3;
      double ra[AL];
      auto load_a = [&](int k0) {
#pragma unroll
        for (int u = 0; u < AL; ++u) {
          const int e = tid + 256 * u, i = e % LD, k = e / LD;
          ra[u] = (e < BK * LD && k0 + k < kmax && i < 8 * RT) ? A[(int64_t)(k0 + k) * LD + i] : 0.0;
        }
      };
      load_a(0);
      for (int k0 = 0; k0 < kmax; k0 += BK) {
        __syncthreads();
#pragma unroll
        for (int u = 0; u < AL; ++u) {
          const int e = tid + 256 * u;
          if (e < BK * LD) As[(e / LD) * LDA + e % LD] = ra[u];
        }
        __syncthreads();
        if (k0 + BK < kmax) load_a(k0 + BK);
#pragma unroll
        for (int ks = 0; ks < BK; ks += 4) {
          double af[MT], bf[NT];
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) af[mt] = As[(ks + t) * LDA + 8 * (warp + 8 * mt) + g];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) bf[nt] = G[(8 * nt + g) * GS + k0 + ks + t];
#pragma unroll
          for (int mt = 0; mt < MT; ++mt)
            if (warp + 8 * mt < RT)                    // warp-uniform
#pragma unroll
              for (int nt = 0; nt < NT; ++nt) dmma(acc[mt][nt], af[mt], bf[nt]);
        }
      }
      __syncthreads();
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
        if (warp + 8 * mt < RT)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) G[(8 * nt + 2 * t + i) * GS + 8 * (warp + 8 * mt) + g] = acc[mt][nt][i];
      __syncthreads();
      // scatter: thread j owns entry j of the targets' partial locals, four targets (runs of the
      // chunk's pairs) at a time
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int j = tid + 256 * i;
        if (j >= NP) continue;
        const int jp = tpart[i];
        const uint32_t mk = tmsk[i];
        double* plj = Pl + (int64_t)b.y * pitch + (int64_t)comp * LD + j;
        for (int q = 0; q < nc;) {
          int st[4], en[4], tg[4];
          double pv[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            st[r] = q;
            tg[r] = q < nc ? pt[q] : 0;
            pv[r] = q < nc ? plj[(int64_t)tg[r] * pitch] : 0.0;
            while (q < nc && pt[q] == tg[r]) ++q;
            en[r] = q;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r)
            if (st[r] < en[r]) {
              double run = pv[r];
              for (int k = st[r]; k < en[r]; ++k) {
                const int f = pfac[k];
                const double y = G[k * GS + ((mk >> f) & 1 ? jp : j)];
                run = fma(alpha, (mk >> (16 + f)) & 1 ? -y : y, run);
              }
              plj[(int64_t)tg[r] * pitch] = run;
            }
        }
      }
    }
  }
}

// the scalar blocks of the method (1 for Laplace3D; 4 for the Stokeslet: Φ₁..₃ and Ψ̂, the last
// with the coupling), nexp·LD apart per node
template <int LD, int NB>
void launch(State& S) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  const int nb = (int)P.h_blocks.size();
  if (nb == 0) return;
  const size_t smem = m2l_f64_smem<LD, NB>();
  auto kern = k_m2l_f64<LD, NB>;
  FMMB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // one launch: blockIdx.x the target block, blockIdx.y the expansion block (the CTAs of different
  // expansion blocks write disjoint slices of the targets' locals)
  const int nexp = C.nexp;
  kern<<<dim3(nb, nexp), 256, smem, P.ctx->stream>>>(P.blocks.p, P.cls_off.p, P.pairs.p, P.d_lv_reps.p, P.d_m2l_scale.p, C.np,
                                                     S.M.p, S.Pl.p, (int64_t)nexp * LD, nexp == 4);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

// two chunk widths per expansion length: the default, and the alternative the tuner may choose
// (S.f64_nb_alt); the sums do not depend on it
void m2l_f64(State& S) {
  const bool alt = S.f64_nb_alt != 0;
  switch (S.plan->cache->ld) {
    case 64: alt ? launch<64, 32>(S) : launch<64, 64>(S); break;
    case 128: alt ? launch<128, 32>(S) : launch<128, 64>(S); break;
    case 192: alt ? launch<192, 64>(S) : launch<192, 32>(S); break;
    case 256: alt ? launch<256, 16>(S) : launch<256, 32>(S); break;
    case 320: alt ? launch<320, 32>(S) : launch<320, 48>(S); break;
    case 384: alt ? launch<384, 24>(S) : launch<384, 40>(S); break;
    case 448: alt ? launch<448, 16>(S) : launch<448, 32>(S); break;
    default: throw Error(FMMB_ERR_UNSUPPORTED, "no M2L kernel for this expansion length");
  }
}

}  // namespace fmmb
