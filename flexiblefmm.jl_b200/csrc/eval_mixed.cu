// The mixed path's evaluation: L2P in FP64 from the leaf's local expansion, and the near
// field (src/evaluate.jl:12-48, src/device.jl:89-100,189-206) in FP32 with two safeguards:
//   - coordinates relative to the target leaf's centre: each source is staged once per
//     warp as float(x − c) computed in FP64, so the FP32 differences carry an absolute
//     error of ~2⁻²⁴·w instead of 2⁻²⁴·|x| (close pairs keep their accuracy)
//   - compensated sums: each staged batch of ≤ 32 sources is summed in FP32 and the batch
//     sums are accumulated in FP64
// One warp per group of targets in one real leaf, lanes over the targets, the staged
// sources read from shared memory by all lanes (broadcast).
#include "passes.cuh"

namespace fmmb {
namespace {

// TPL·32 targets of one leaf starting at target index k0 (nrem of them remain): L2P in FP64,
// then the near field of the 27 colleagues, each source staged once per warp and used by
// TPL targets per lane
template <int P, bool SELF, int TPL>
__device__ __forceinline__ void near_chunk(int leaf, int k0, int nrem, int lane, const double* __restrict__ L, float4* stg,
                                           double cx, double cy, double cz, double s, const double* __restrict__ tx,
                                           const double* __restrict__ ty, const double* __restrict__ tz,
                                           const int* __restrict__ tout, const double* __restrict__ xs,
                                           const double* __restrict__ ys, const double* __restrict__ zs,
                                           const double* __restrict__ q, const int* __restrict__ plo,
                                           const int* __restrict__ phi, const int* __restrict__ col, int outputs,
                                           double* __restrict__ pot, double* __restrict__ grad) {
  int k[TPL];
  bool act[TPL];
  float fx[TPL], fy[TPL], fz[TPL];
  double np[TPL], nx[TPL], ny[TPL], nz[TPL];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    k[t] = k0 + lane + 32 * t;
    act[t] = lane + 32 * t < nrem;
    fx[t] = act[t] ? (float)(tx[k[t]] - cx) : 0.f;
    fy[t] = act[t] ? (float)(ty[k[t]] - cy) : 0.f;
    fz[t] = act[t] ? (float)(tz[k[t]] - cz) : 0.f;
    np[t] = nx[t] = ny[t] = nz[t] = 0.0;
  }
#pragma unroll 1
  for (int kk = 0; kk < NCOL; ++kk) {
    const int cn = col[(int64_t)leaf * NCOL + kk];
    if (cn < 0) continue;
    const int j0 = plo[cn], j1 = phi[cn];
    for (int jb = j0; jb <= j1; jb += 32) {
      const int j = jb + lane;
      if (j <= j1) stg[lane] = make_float4((float)(xs[j] - cx), (float)(ys[j] - cy), (float)(zs[j] - cz), (float)q[j]);
      __syncwarp();
      const int m = min(32, j1 - jb + 1);
      float bp[TPL], bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bp[t] = bx[t] = by[t] = bz[t] = 0.f;
#pragma unroll 4
      for (int i = 0; i < m; ++i) {
        const float4 sv = stg[i];
#pragma unroll
        for (int t = 0; t < TPL; ++t) {
          const float dx = fx[t] - sv.x, dy = fy[t] - sv.y, dz = fz[t] - sv.z;
          const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
          float ir = rsqrtf(r2);
          if (SELF && jb + i == k[t]) ir = 0.f;
          const float qir = sv.w * ir;
          const float qir3 = qir * ir * ir;
          bp[t] += qir;
          bx[t] = fmaf(qir3, dx, bx[t]);
          by[t] = fmaf(qir3, dy, by[t]);
          bz[t] = fmaf(qir3, dz, bz[t]);
        }
      }
#pragma unroll
      for (int t = 0; t < TPL; ++t) { np[t] += bp[t]; nx[t] += bx[t]; ny[t] += by[t]; nz[t] += bz[t]; }
      __syncwarp();
    }
  }
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    double u, gx, gy, gz;
    const double px = act[t] ? tx[k[t]] : cx, py = act[t] ? ty[k[t]] : cy, pz = act[t] ? tz[k[t]] : cz;
    l2p_f64<P>(L, (px - cx) * s, (py - cy) * s, (pz - cz) * s, u, gx, gy, gz);
    if (act[t]) {
      const int o = tout[k[t]];
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = u + KC * np[t];
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        grad[3 * (int64_t)o] = gx * s - KC * nx[t];
        grad[3 * (int64_t)o + 1] = gy * s - KC * ny[t];
        grad[3 * (int64_t)o + 2] = gz * s - KC * nz[t];
      }
    }
  }
}

template <int P, bool SELF>
__global__ void __launch_bounds__(256) k_eval_mixed(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                    const int* __restrict__ gcount, int ngroups, const double* __restrict__ tx,
                                                    const double* __restrict__ ty, const double* __restrict__ tz,
                                                    const int* __restrict__ tout, const double* __restrict__ xs,
                                                    const double* __restrict__ ys, const double* __restrict__ zs,
                                                    const double* __restrict__ q, const int4* __restrict__ cell,
                                                    const int* __restrict__ plo, const int* __restrict__ phi,
                                                    const int* __restrict__ col, const double* __restrict__ Pl, int LD,
                                                    Geometry geo, const double* __restrict__ scale, int outputs,
                                                    double* __restrict__ pot, double* __restrict__ grad) {
  extern __shared__ double sl[];
  const int nw = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * nw + warp;
  if (grp >= ngroups) return;
  double* L = sl + warp * LD;
  float4* stg = reinterpret_cast<float4*>(sl + nw * LD) + warp * 32;
  const int leaf = gnode[grp];
  for (int i = lane; i < LD; i += 32) L[i] = Pl[(int64_t)leaf * LD + i];
  __syncwarp();
  const int4 c = cell[leaf];
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = geo.center(0, c.x, w), cy = geo.center(1, c.y, w), cz = geo.center(2, c.z, w);
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt;) {
    // 64 targets (two per lane) while more than 32 remain, then 32
    if (nt - base > 32) {
      near_chunk<P, SELF, 2>(leaf, t0 + base, nt - base, lane, L, stg, cx, cy, cz, s, tx, ty, tz, tout, xs, ys, zs, q, plo, phi,
                             col, outputs, pot, grad);
      base += 64;
    } else {
      near_chunk<P, SELF, 1>(leaf, t0 + base, nt - base, lane, L, stg, cx, cy, cz, s, tx, ty, tz, tout, xs, ys, zs, q, plo, phi,
                             col, outputs, pot, grad);
      base += 32;
    }
  }
}

template <int P, bool SELF>
void launch(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx, const double* ty,
            const double* tz, const int* tout, int outputs, double* pot, double* grad) {
  Plan& P_ = *S.plan;
  if (ng == 0) return;
  const int warps = 8;
  size_t smem = sizeof(double) * warps * P_.cache->ld + sizeof(float4) * 32 * warps;
  k_eval_mixed<P, SELF><<<(ng + warps - 1) / warps, 32 * warps, smem, P_.ctx->stream>>>(
      gnode, gstart, gcount, ng, tx, ty, tz, tout, S.xs.p, S.ys.p, S.zs.p, S.q.p, P_.cell.p, P_.plo.p, P_.phi.p, P_.col.p,
      S.Pl.p, P_.cache->ld, geometry(P_), P_.d_scale.p, outputs, pot, grad);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

void eval_mixed(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx, const double* ty,
                const double* tz, const int* tout, bool self, int outputs, double* pot, double* grad) {
  switch (S.plan->cache->p) {
#define X(pp)                                                                                \
  case pp:                                                                                   \
    if (self) launch<pp, true>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad); \
    else launch<pp, false>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, outputs, pot, grad);     \
    break;
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "the mixed path is built for p ≤ 11");
  }
}

}  // namespace fmmb
