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
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : cx, y = act ? ty[k] : cy, z = act ? tz[k] : cz;
    double u, gx, gy, gz;
    l2p_f64<P>(L, (x - cx) * s, (y - cy) * s, (z - cz) * s, u, gx, gy, gz);
    const float fx = (float)(x - cx), fy = (float)(y - cy), fz = (float)(z - cz);
    double np = 0, nx = 0, ny = 0, nz = 0;
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
        float bp = 0.f, bx = 0.f, by = 0.f, bz = 0.f;
        for (int i = 0; i < m; ++i) {
          const float4 sv = stg[i];
          const float dx = fx - sv.x, dy = fy - sv.y, dz = fz - sv.z;
          const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
          float ir = rsqrtf(r2);
          if (SELF && jb + i == k) ir = 0.f;
          const float qir = sv.w * ir;
          const float qir3 = qir * ir * ir;
          bp += qir;
          bx = fmaf(qir3, dx, bx);
          by = fmaf(qir3, dy, by);
          bz = fmaf(qir3, dz, bz);
        }
        np += bp; nx += bx; ny += by; nz += bz;
        __syncwarp();
      }
    }
    if (act) {
      const int o = tout[k];
      if (outputs & FMMB_OUTPUT_POTENTIAL) pot[o] = u + KC * np;
      if (outputs & FMMB_OUTPUT_GRADIENT) {
        grad[3 * (int64_t)o] = gx * s - KC * nx;
        grad[3 * (int64_t)o + 1] = gy * s - KC * ny;
        grad[3 * (int64_t)o + 2] = gz * s - KC * nz;
      }
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
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "the mixed path is built for p ≤ 10");
  }
}

}  // namespace fmmb
