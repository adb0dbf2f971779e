// M2L of the plain FP64 path: one launch for all levels, one CTA per block of targets
// (src/device_passes.jl:565-580, the class-wise translation of harmonics.jl:531-645).
//
// Per symmetry class and chunk of ≤ NB pairs of the block:
//   gather  G = P_sᵀ M_src for the chunk's columns into shared memory ([column][entry], one
//           coalesced load per lane and entry quartet, the D4h permutation of each entry looked
//           up in a table of its swaps and signs over the 16 group elements, built once per
//           CTA; partner entries by warp shuffles)
//   product Y = A_class G on the FP64 tensor cores (mma.sync m8n8k4 f64, DMMA: there is no FP64
//           tcgen05 kind); each warp owns the row tiles w, w + 8, ... below (p+1)² (the padded
//           rows are not multiplied) × all NB columns, and copies its own rows of A, slab by slab
//           of K, into two shared-memory stages of its own with cp.async (no CTA barrier inside
//           the product; the first two slabs are in flight during the gather)
//   scatter (P_t Y) into the targets' partial locals: each target's entry takes its pairs one by
//           one in the list's order, starting from the value in memory (the block owns its
//           targets: deterministic, no atomics, and the sums do not depend on where the chunks
//           end nor on the other targets of the block); the chunk's runs of one target are found
//           once, and four runs' sums are stepped together, branch-free
// The time per chunk goes to the product (DMMA-bound while both CTAs of an SM multiply), the
// scatter (its dependent FP64 FMAs queue behind the other CTA's DMMAs on the shared FP64 pipe)
// and the gather, in that order.
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

// the class operator's rows reach each warp through its own two shared-memory stages of BK rows
// of K (cp.async, no CTA barrier): its MT row tiles, S = 8·MT + 4 doubles apart (≡ 4 or 12 mod 16:
// the fragment loads are free of bank conflicts)
template <int LD> constexpr int f64_bk() { return LD / 64 <= 3 ? 16 : 8; }
template <int LD> constexpr int f64_s() { return 8 * (LD / 64) + 4; }
template <int LD, int NB>
constexpr size_t m2l_f64_smem() {
  return sizeof(double) * (8 * 2 * f64_bk<LD>() * f64_s<LD>() + NB * (LD + 4)) + sizeof(int) * (5 * NB + 4) +
         sizeof(uint32_t) * LD + LD;
}

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
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
  constexpr int BK = f64_bk<LD>(), MT = LD / 64, NT = NB / 8, GS = LD + 4, S = f64_s<LD>(), ASTG = BK * S;
  constexpr int CPL = BK * MT * 4 / 32;   // 16-byte copies per lane and stage
  static_assert(BK * MT * 4 % 32 == 0, "a stage is whole copies per lane");
  static_assert(NB % 4 == 0, "the entry masks are read as uint4: 5·NB + 4 ints before them keep 16-byte alignment");
  // entry quartets per lane (LD = 64: lanes ≥ 16 idle). A pair of entries never straddles a
  // multiple of 128 (entries 128, 256, 384 are real parts or m = 0), so the partner of a
  // lane's first and last entry is always in the neighbouring lane of the same quartet row.
  constexpr int Q = (LD + 127) / 128;
  constexpr int HC = 2 < NB / 8 ? 2 : NB / 8;   // columns per warp with their loads in flight together
  extern __shared__ double sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* Aw = sm + warp * 2 * ASTG;   // this warp's two stages, [BK][S] each
  double* G = sm + 8 * 2 * ASTG;       // [NB][GS]: the gathered columns, then the product
  int* ps = (int*)(G + NB * GS);
  int* pf = ps + NB;
  int* pt = pf + NB;
  int* pfac = pt + NB;               // the pairs' D4h elements
  int* rst = pfac + NB;              // [NB + 4]: the chunk's runs of one target (starts, nc), their count
  uint32_t* smsk = (uint32_t*)(rst + NB + 4);   // [LD]: the gather's masks per entry (0 past NP), 16-byte aligned
  int8_t* sdir = (int8_t*)(smsk + LD);       // [LD]: where each entry's partner is (+1 Re, −1 Im, 0)
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
  // this warp's rows of the slab of A at K-row k0 into stage st (rows of tiles past RT skipped)
  auto stage_a = [&](const double* A, int k0, int st) {
    double* dst = Aw + st * ASTG;
#pragma unroll
    for (int u = 0; u < CPL; ++u) {
      const int c = lane + 32 * u, k = c / (4 * MT), rem = c % (4 * MT), mt = rem >> 2, q = rem & 3;
      if (warp + 8 * mt < RT) cpa16(dst + k * S + 8 * mt + 2 * q, A + (int64_t)(k0 + k) * LD + 8 * (warp + 8 * mt) + 2 * q);
    }
    cpa_commit();
  };
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
      // the first two slabs of A on their way while the columns are gathered
      stage_a(A, 0, 0);
      if (BK < kmax) stage_a(A, BK, 1);
      __syncthreads();
      // the runs of the chunk's pairs (the pairs of a class are grouped by target: each target
      // has one run), by the last warp
      if (warp == 7) {
        int base = 0;
        for (int q1 = 0; q1 < nc; q1 += 32) {
          const int q = q1 + lane;
          const bool start = q < nc && (q == 0 || pt[q] != pt[q - 1]);
          const unsigned bal = __ballot_sync(0xffffffffu, start);
          if (start) rst[base + __popc(bal & ((1u << lane) - 1u))] = q;
          base += __popc(bal);
        }
        if (lane == 0) { rst[base] = nc; rst[NB + 1] = base; }
      }
      // gather: warp w the columns w, w + 8, ..., HC at a time (their loads all in flight before
      // any is permuted); lane l the entries 4(l + 32 r) .. + 3
      for (int j0 = warp; j0 < nc; j0 += 8 * HC) {
        double a[HC][Q][4];
#pragma unroll
        for (int h = 0; h < HC; ++h) {
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
        for (int h = 0; h < HC; ++h) {
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
      __syncthreads();
      // product Y = A·G on the FP64 tensor cores: warp w the row tiles w, w + 8, w + 16, ... below
      // the last real row (RT tiles of 8 rows; the rows past NP are zero and are not multiplied)
      // × all NB columns (NT tiles of 8), K-steps of 4; A through the warp's two stages, the slab
      // after next copied while this one is multiplied
      double acc[MT][NT][2];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
      const int g = lane >> 2, t = lane & 3;
      int st = 0;
      for (int k0 = 0; k0 < kmax; k0 += BK, st ^= 1) {
        if (k0 + BK < kmax) cpa_wait<1>(); else cpa_wait<0>();
        __syncwarp();
        const double* As = Aw + st * ASTG;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 4) {
          double af[MT], bf[NT];
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) af[mt] = As[(ks + t) * S + 8 * mt + g];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) bf[nt] = G[(8 * nt + g) * GS + k0 + ks + t];
#pragma unroll
          for (int mt = 0; mt < MT; ++mt)
            if (warp + 8 * mt < RT)                    // warp-uniform
#pragma unroll
              for (int nt = 0; nt < NT; ++nt) dmma(acc[mt][nt], af[mt], bf[nt]);
        }
        __syncwarp();                                  // the stage is read: refill it
        if (k0 + 2 * BK < kmax) stage_a(A, k0 + 2 * BK, st);
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
      // scatter: thread j owns entry j of the targets' partial locals; RB runs (targets) at a time,
      // each summed in the list's order from its value in memory, the runs stepped together
      constexpr int RB = 4;
      const int nrun = rst[NB + 1];
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int j = tid + 256 * i;
        if (j >= NP) continue;
        const int jp = tpart[i];
        const uint32_t mk = tmsk[i];
        double* plj = Pl + (int64_t)b.y * pitch + (int64_t)comp * LD + j;
        for (int r0 = 0; r0 < nrun; r0 += RB) {
          int rs[RB], re[RB];
          int64_t to[RB];
          double run[RB];
          int len = 0;
#pragma unroll
          for (int r = 0; r < RB; ++r) {
            const bool on = r0 + r < nrun;
            rs[r] = on ? rst[r0 + r] : 0;
            re[r] = on ? rst[r0 + r + 1] : 0;
            to[r] = (int64_t)(on ? pt[rs[r]] : 0) * pitch;
            run[r] = on ? plj[to[r]] : 0.0;
            len = max(len, re[r] - rs[r]);
          }
          // branch-free steps: every run's loads issued before any sum (a run past its end reads
          // pair 0 and keeps its value)
          for (int e = 0; e < len; ++e) {
            double y[RB];
            uint32_t ng[RB];
#pragma unroll
            for (int r = 0; r < RB; ++r) {
              const int k = rs[r] + e < re[r] ? rs[r] + e : 0;
              const int f = pfac[k];
              y[r] = G[k * GS + ((mk >> f) & 1 ? jp : j)];
              ng[r] = (mk >> (16 + f)) & 1;
            }
#pragma unroll
            for (int r = 0; r < RB; ++r) {
              const double v = fma(alpha, ng[r] ? -y[r] : y[r], run[r]);
              run[r] = rs[r] + e < re[r] ? v : run[r];
            }
          }
#pragma unroll
          for (int r = 0; r < RB; ++r)
            if (r0 + r < nrun) plj[to[r]] = run[r];
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
