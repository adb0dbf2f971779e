// StokesHarmonics(Stokeslet3D(); p) on the plain FP64 path (src/operators/harmonics_stokes.jl):
// the Stokeslet through four Laplace potentials, Φ_k = Σ f_k/(4πr) and Ψ_c = Σ (y − c)·f/(4πr),
// u = ½[Φ − (x − c)·∇Φ + ∇Ψ_c]. Every node holds the four scalar expansions [Φ₁; Φ₂; Φ₃; Ψ̂]
// (Ψ̂ = Ψ_c/w in the box's own coordinates), nexp·LD apart; they use the scalar operators of
// SphericalHarmonics with the couplings of the reference:
//   P2M  block k: charges f_k; block 4: charges ŷ·f (ŷ = (y − c)/w)        (harmonics_stokes.jl:322-328)
//   M2M  Ψ̂_P = ½ Ψ̂_C + δ̂·Φ_C folded into the stacked children before the product (:136-158)
//   M2L  Ψ̂_B += T(Ψ̂_A + o·Φ_A), o the far offset (linear in the source: the gather of the fourth
//        launch of the class-wise M2L forms it, m2l_f64.cu)                 (:77-97)
//   L2L  children blocks 1–3 = L2L·P_a; block 4 = 2·L2L·P₄ − 2 δ̂·(L2L·P_Φ) (:159-183)
//   L2P  u = ½[Φ − x̂·∇̂Φ + ∇̂Ψ̂] from the values and scaled gradients of the four blocks (:283-287)
//   near c(f/r + d(d·f)/r³), c = 1/(8π), self excluded by index (src/kernels.jl:253-272)
// Stresslets (f, ν) and doublets g (src/sources.jl:203-281) enter as dipole densities
// (harmonics_stokes.jl:205-216,382-393): block k takes the dipole −(f_k ν + ν_k f), block 4 the
// dipole −((ν·ŷ) f + (f·ŷ) ν) + g/w; the translations and L2P are the same. The pressure is
// −∇·Φ (−s·tr of the scaled gradients of blocks 1–3, :343-346) plus the near-field pressures
// 2c(d·f)/r³ and 4c[(f·ν)/r³ − 3(d·f)(d·ν)/r⁵] (a doublet has none).
#include <type_traits>

#include "passes.cuh"

namespace fmmb {
namespace {

constexpr double KSTOKES = 0.039788735772973833942;   // 1/(8π)
constexpr int SW = 4;                                  // warps per block of the evaluation kernels

inline unsigned nblk(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// δ̂ of child slot j along d: (c_child − c_parent)/w_parent ∈ {±1/4} (bit d of j = coordinate d)
__device__ __forceinline__ double dhat(int j, int d) { return (((j >> d) & 1) ? 0.25 : -0.25); }

// points and densities in tree order (perm: sorted position → original index), weighted: the
// Stokeslets into f3 (zeros when absent), the stresslet strengths, stressvecs and doublets into
// sd (3 × n planar each, zeros when absent) when sd is given
__global__ void k_stokes_gather(const double* __restrict__ xyz, StokesDensities d, const int* __restrict__ perm,
                                int64_t n, double* __restrict__ xs, double* __restrict__ ys, double* __restrict__ zs,
                                double* __restrict__ f3, double* __restrict__ sd) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j = perm[i];
  xs[i] = xyz[3 * j];
  ys[i] = xyz[3 * j + 1];
  zs[i] = xyz[3 * j + 2];
  const double wt = d.weights ? d.weights[j] : 1.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) f3[k * n + i] = d.stokeslets ? wt * d.stokeslets[3 * j + k] : 0.0;
  if (sd) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sd[k * n + i] = d.stresslets ? wt * d.stresslets[3 * j + k] : 0.0;
      sd[(3 + k) * n + i] = d.stresslets ? d.stressvecs[3 * j + k] : 0.0;
      sd[(6 + k) * n + i] = d.doublets ? wt * d.doublets[3 * j + k] : 0.0;
    }
  }
}

// the fourth P2M block's charges ŷ·f, ŷ = (y − c)·s relative to the centre c of the node whose
// multipole the point enters, s = 1/w; with DENS also the four blocks' dipoles (3 × n planar per
// block, in physical units: the P2M scales them by s): −(f_k ν + ν_k f) for block k and
// −((ν·ŷ) f + (f·ŷ) ν) + g·s for block 4 (f, ν the stresslet, g the doublet)
template <bool DENS>
__global__ void k_stokes_q4(const int* __restrict__ nodes, int nn, const int4* __restrict__ cell,
                            const int* __restrict__ plo, const int* __restrict__ phi, Geometry geo,
                            const double* __restrict__ scale, int64_t n, const double* __restrict__ xs,
                            const double* __restrict__ ys, const double* __restrict__ zs, const double* __restrict__ f3,
                            const double* __restrict__ sd, double* __restrict__ q4, double* __restrict__ dip4) {
  // one warp per childless node with sources (the nodes P2M runs on, ghost children of a leaf
  // included): Ψ̂ is centred on the node whose multipole it starts
  const int wid = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (wid >= nn) return;
  const int node = nodes[wid];
  const int4 c = cell[node];
  const Geometry gn = geo.at(node);
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  for (int i = plo[node] + lane; i <= phi[node]; i += 32) {
    const double y[3] = {(xs[i] - cx) * s, (ys[i] - cy) * s, (zs[i] - cz) * s};
    q4[i] = y[0] * f3[i] + y[1] * f3[n + i] + y[2] * f3[2 * n + i];
    if (DENS) {
      double f[3], nu[3], g[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        f[k] = sd[k * n + i];
        nu[k] = sd[(3 + k) * n + i];
        g[k] = sd[(6 + k) * n + i];
      }
      const double ny = nu[0] * y[0] + nu[1] * y[1] + nu[2] * y[2], fy = f[0] * y[0] + f[1] * y[1] + f[2] * y[2];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int e = 0; e < 3; ++e) dip4[(3 * k + e) * n + i] = -(f[k] * nu[e] + nu[k] * f[e]);
        dip4[(9 + k) * n + i] = -(ny * f[k] + fy * nu[k]) + g[k] * s;
      }
    }
  }
}

// M2M input of block a for the ng sibling groups of children starting at c0: the eight
// children's block a stacked (8·LD per group); block 4 with ½Ψ̂ + δ̂·Φ
__global__ void k_stokes_m2m_in(const double* __restrict__ M, int c0, int ng, int LD, int a, double* __restrict__ X) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)ng * 8 * LD) return;
  const int i = (int)(e % LD), j = (int)((e / LD) % 8), g = (int)(e / (8 * LD));
  const double* ch = M + (int64_t)(c0 + 8 * g + j) * 4 * LD;
  double v;
  if (a < 3) v = ch[(int64_t)a * LD + i];
  else v = 0.5 * ch[3 * (int64_t)LD + i] + dhat(j, 0) * ch[i] + dhat(j, 1) * ch[LD + i] + dhat(j, 2) * ch[2 * (int64_t)LD + i];
  X[e] = v;
}

// L2L output: R_a = L2L·P_a (8·LD per group, a = 0..3) added to the children's partial locals,
// block 4 as 2·R₄ − 2 δ̂·(R₁, R₂, R₃)
__global__ void k_stokes_l2l_out(double* __restrict__ Pl, const double* __restrict__ R, int c0, int ng, int LD, int NP) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)ng * 8 * LD;
  if (e >= per) return;
  const int i = (int)(e % LD), j = (int)((e / LD) % 8), g = (int)(e / (8 * LD));
  if (i >= NP) return;
  double* ch = Pl + (int64_t)(c0 + 8 * g + j) * 4 * LD;
  const double r1 = R[e], r2 = R[per + e], r3 = R[2 * per + e], r4 = R[3 * per + e];
  ch[i] += r1;
  ch[LD + i] += r2;
  ch[2 * (int64_t)LD + i] += r3;
  ch[3 * (int64_t)LD + i] += 2.0 * r4 - 2.0 * (dhat(j, 0) * r1 + dhat(j, 1) * r2 + dhat(j, 2) * r3);
}

// the far field at the targets of one leaf: u = ½[Φ − x̂·∇̂Φ + ∇̂Ψ̂] from the leaf's four local blocks
// (staged in shared memory per warp), lanes over the targets; writes the velocities, or with PRES
// the pressures −s·tr(∇̂Φ) (blocks 1–3 only)
template <int P, bool PRES>
__global__ void __launch_bounds__(SW * 32) k_stokes_l2p(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                        const int* __restrict__ gcount, int ngroups,
                                                        const double* __restrict__ tx, const double* __restrict__ ty,
                                                        const double* __restrict__ tz, const int* __restrict__ tout,
                                                        const int4* __restrict__ cell, const double* __restrict__ Pl, int LD,
                                                        Geometry geo, const double* __restrict__ scale,
                                                        double* __restrict__ vel) {
  extern __shared__ double sl[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * SW + warp;
  if (grp >= ngroups) return;
  double* L = sl + (int64_t)warp * 4 * LD;
  const int leaf = gnode[grp];
  for (int i = lane; i < 4 * LD; i += 32) L[i] = Pl[(int64_t)leaf * 4 * LD + i];
  __syncwarp();
  const int4 c = cell[leaf];
  const Geometry gn = geo.at(leaf);
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double xh[3] = {act ? (tx[k] - cx) * s : 0.0, act ? (ty[k] - cy) * s : 0.0, act ? (tz[k] - cz) * s : 0.0};
    double phi[3], G[3][3], gpsi[3];   // G[i][k] = ∂̂_i Φ_k
    for (int a = 0; a < (PRES ? 3 : 4); ++a) {
      double u, g[3];
      l2p<P, double>(L + (int64_t)a * LD, xh[0], xh[1], xh[2], u, g[0], g[1], g[2]);
      if (a < 3) {
        phi[a] = u;
        for (int i = 0; i < 3; ++i) G[i][a] = g[i];
      } else {
        for (int i = 0; i < 3; ++i) gpsi[i] = g[i];
      }
    }
    if (act) {
      const int o = tout[k];
      if (PRES)
        vel[o] = -s * (G[0][0] + G[1][1] + G[2][2]);
      else
        for (int i = 0; i < 3; ++i)
          vel[3 * (int64_t)o + i] = 0.5 * (phi[i] - (xh[0] * G[i][0] + xh[1] * G[i][1] + xh[2] * G[i][2]) + gpsi[i]);
    }
  }
}

// the scaled gradient of a local expansion L of degree P as three expansions of degree P − 1 in
// the real storage (n², and re/im of order m at n² + 2m − 1, n² + 2m), from the derivative
// identities (harmonics_stokes.jl:231-240, harmonics.jl:465-486): (D₋L)_n^m = −cm(n+1, m+1) L_{n+1}^{m+1},
// (D₊L)_n^m = cp(n+1, m−1) L_{n+1}^{m−1}, (D_zL)_n^m = cz(n+1, m) L_{n+1}^m, ∂̂_x = ½(D₋ + D₊),
// ∂̂_y = (i/2)(D₊ − D₋), ∂̂_z = D_z; the lanes of a warp share the P² entries
template <int P>
__device__ void grad_sets(const double* __restrict__ L, double* __restrict__ Ax, double* __restrict__ Ay,
                          double* __restrict__ Az, int lane) {
  for (int e = lane; e < P * P; e += 32) {
    int n = (int)sqrtf((float)e);
    while (n * n > e) --n;
    while ((n + 1) * (n + 1) <= e) ++n;
    const int k = e - n * n, m = (k + 1) / 2, n1 = n + 1, b = n1 * n1;
    const bool im = k > 0 && (k & 1) == 0;
    if (m == 0) {
      const double cmv = c_tab[3 * TRI_MAX + tri(n1, 1)];
      Ax[e] = -cmv * L[b + 1];
      Ay[e] = -cmv * L[b + 2];
      Az[e] = c_tab[2 * TRI_MAX + tri(n1, 0)] * L[b];
    } else {
      const double ur = L[b + 2 * (m + 1) - 1], ui = L[b + 2 * (m + 1)];
      const double dr = m == 1 ? L[b] : L[b + 2 * (m - 1) - 1], di = m == 1 ? 0.0 : L[b + 2 * (m - 1)];
      const double cu = 0.5 * c_tab[3 * TRI_MAX + tri(n1, m + 1)], cd = 0.5 * c_tab[4 * TRI_MAX + tri(n1, m - 1)];
      const double czv = c_tab[2 * TRI_MAX + tri(n1, m)];
      Ax[e] = im ? -cu * ui + cd * di : -cu * ur + cd * dr;
      Ay[e] = im ? cu * ur + cd * dr : -(cu * ui + cd * di);
      Az[e] = czv * (im ? L[b + 2 * m] : L[b + 2 * m - 1]);
    }
  }
}

constexpr int GW = 2;   // warps per block of the velocity-gradient L2P

// the far-field velocity gradient at the targets of one leaf (harmonics_stokes.jl:347-350):
// ∂u_i/∂t_j = (s/2)[∂̂_jΦ_i − ∂̂_iΦ_j − Σ_k x̂_k ∂̂_i∂̂_jΦ_k + ∂̂_i∂̂_jΨ̂], written at 9·o + 3i + j. Per
// warp the leaf's four blocks and their twelve gradient expansions sit in shared memory; per target
// twelve degree-(P−1) L2Ps give the first and second derivatives.
template <int P>
__global__ void __launch_bounds__(GW * 32) k_stokes_l2p_grad(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                             const int* __restrict__ gcount, int ngroups,
                                                             const double* __restrict__ tx, const double* __restrict__ ty,
                                                             const double* __restrict__ tz, const int* __restrict__ tout,
                                                             const int4* __restrict__ cell, const double* __restrict__ Pl,
                                                             int LD, Geometry geo, const double* __restrict__ scale,
                                                             double* __restrict__ out) {
  extern __shared__ double sg[];
  constexpr int NG = P * P;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * GW + warp;
  if (grp >= ngroups) return;
  double* L = sg + (int64_t)warp * (4 * LD + 12 * NG);
  double* A = L + 4 * LD;   // block a, direction j at A + (3a + j)·NG
  const int leaf = gnode[grp];
  for (int i = lane; i < 4 * LD; i += 32) L[i] = Pl[(int64_t)leaf * 4 * LD + i];
  __syncwarp();
  for (int a = 0; a < 4; ++a) grad_sets<P>(L + a * LD, A + 3 * a * NG, A + (3 * a + 1) * NG, A + (3 * a + 2) * NG, lane);
  __syncwarp();
  const int4 c = cell[leaf];
  const Geometry gn = geo.at(leaf);
  const double w = ldexp(geo.W0, -c.w), s = scale[c.w];
  const double cx = gn.center(0, c.x, w), cy = gn.center(1, c.y, w), cz = gn.center(2, c.z, w);
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double xh[3] = {act ? (tx[k] - cx) * s : 0.0, act ? (ty[k] - cy) * s : 0.0, act ? (tz[k] - cz) * s : 0.0};
    double gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 4; ++a) {
      const double coef = a < 3 ? -xh[a] : 1.0;
      for (int j = 0; j < 3; ++j) {
        double v, h[3];
        l2p<P - 1, double>(A + (3 * a + j) * NG, xh[0], xh[1], xh[2], v, h[0], h[1], h[2]);
        if (a < 3) {   // v = ∂̂_jΦ_a: +v at (a, j), −v at (j, a)
          gr[a][j] += v;
          gr[j][a] -= v;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) gr[i][j] += coef * h[i];   // h_i = ∂̂_i∂̂_j of block a
      }
    }
    if (act) {
      const int o = tout[k];
#pragma unroll
      for (int e = 0; e < 9; ++e) out[9 * (int64_t)o + e] = 0.5 * s * gr[e / 3][e % 3];
    }
  }
}

struct alignas(16) S8 { double x, y, z, fx, fy, fz, pad0, pad1; };
struct alignas(16) S16 { double x, y, z, fx, fy, fz, sx, sy, sz, nx, ny, nz, gx, gy, gz, pad; };

// the near field: the sources of the 27 colleagues, flattened into batches of 32 staged per warp
// (the next batch's loads in flight), lanes over the targets; adds c·Σ to the velocities (OUT 0),
// the pressures (OUT 1) or the velocity gradients (OUT 2, ∂u_i/∂t_j at 9·o + 3i + j). DENS adds
// the stresslets and doublets of sd (3 × n planar: strengths, stressvecs, doublets) to the
// Stokeslets (src/sources.jl:203-281):
//   u = c[f/r + g/r³ + d((d·f)/r³ − 3(d·g)/r⁵ − 6(d·f_s)(d·ν)/r⁵)],  p = c[2(d·f)/r³ + 4(f_s·ν)/r³ − 12(d·f_s)(d·ν)/r⁵]
//   ∂u_i/∂t_j = c[d_i(A d_j + v_j) + w_i d_j + B δ_ij] with A = −3(d·f)/r⁵ + (30(d·f_s)(d·ν) + 15(d·g))/r⁷,
//   B = (d·f)/r³ − (6(d·f_s)(d·ν) + 3(d·g))/r⁵, v = f/r³ − 6((d·ν) f_s + (d·f_s) ν)/r⁵ − 3g/r⁵,
//   w = −f/r³ − 3g/r⁵ (the closed forms of the three gradients, summed)
template <bool SELF, bool DENS, int OUT>
__global__ void __launch_bounds__(SW * 32) k_stokes_near(const int* __restrict__ gnode, const int* __restrict__ gstart,
                                                         const int* __restrict__ gcount, int ngroups,
                                                         const double* __restrict__ tx, const double* __restrict__ ty,
                                                         const double* __restrict__ tz, const int* __restrict__ tout,
                                                         const double* __restrict__ xs, const double* __restrict__ ys,
                                                         const double* __restrict__ zs, const double* __restrict__ f3,
                                                         const double* __restrict__ sd, int64_t n,
                                                         const int* __restrict__ plo, const int* __restrict__ phi,
                                                         const int* __restrict__ col, double* __restrict__ out) {
  using SV = std::conditional_t<DENS, S16, S8>;
  __shared__ SV stg[SW][2][32];
  __shared__ int s_lo[SW][32], s_pre[SW][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x * SW + warp;
  if (grp >= ngroups) return;
  const int leaf = gnode[grp];
  const int cn = lane < NCOL ? col[(int64_t)leaf * NCOL + lane] : -1;
  int lo = 0, len = 0;
  if (cn >= 0) {
    lo = plo[cn];
    len = max(0, phi[cn] - lo + 1);
  }
  int incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int S = __shfl_sync(0xffffffffu, incl, 31);
  s_lo[warp][lane] = lo;
  s_pre[warp][lane] = incl - len;
  const unsigned selfm = __ballot_sync(0xffffffffu, cn == leaf);
  const int slot = selfm ? __ffs(selfm) - 1 : 0;
  const int pself = selfm ? __shfl_sync(0xffffffffu, incl - len, slot) : -1;
  const int loself = __shfl_sync(0xffffffffu, lo, slot), lenself = selfm ? __shfl_sync(0xffffffffu, len, slot) : 0;
  __syncwarp();
  auto load = [&](int b, SV& v) {
    const int f = 32 * b + lane;
    v = SV{};
    if (f < S) {
      int idx = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1)
        if (s_pre[warp][idx + step] <= f) idx += step;
      const int64_t j = s_lo[warp][idx] + (f - s_pre[warp][idx]);
      if constexpr (DENS)
        v = SV{xs[j],         ys[j],         zs[j],         f3[j],         f3[n + j],     f3[2 * n + j],
               sd[j],         sd[n + j],     sd[2 * n + j], sd[3 * n + j], sd[4 * n + j], sd[5 * n + j],
               sd[6 * n + j], sd[7 * n + j], sd[8 * n + j], 0};
      else
        v = SV{xs[j], ys[j], zs[j], f3[j], f3[n + j], f3[2 * n + j], 0, 0};
    }
  };
  const int t0 = gstart[grp], nt = gcount[grp];
  for (int base = 0; base < nt; base += 32) {
    const int k = t0 + base + lane;
    const bool act = base + lane < nt;
    const double x = act ? tx[k] : 0.0, y = act ? ty[k] : 0.0, z = act ? tz[k] : 0.0;
    const int fself = SELF && act && selfm ? pself + (k - loself) : -1;
    double ux = 0, uy = 0, uz = 0;
    double gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    SV nxt;
    load(0, nxt);
    for (int b = 0; 32 * b < S; ++b) {
      SV* st = stg[warp][b & 1];
      st[lane] = nxt;
      __syncwarp();
      if (32 * (b + 1) < S) load(b + 1, nxt);
      const int m = min(32, S - 32 * b);
      const bool chk = SELF && selfm && 32 * b < pself + lenself && 32 * b + 32 > pself;   // uniform
      const int is = fself - 32 * b;
      for (int i = 0; i < m; ++i) {
        const SV sv = st[i];
        const double dx = x - sv.x, dy = y - sv.y, dz = z - sv.z;
        const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
        double ir = rsqrt(r2);
        if (chk && i == is) ir = 0.0;
        const double ir3 = ir * ir * ir;
        const double df = dx * sv.fx + dy * sv.fy + dz * sv.fz;
        if constexpr (OUT == 2) {
          const double ir2 = ir * ir, ir5 = ir3 * ir2;
          const double d[3] = {dx, dy, dz};
          double A = -3.0 * df * ir5, B = df * ir3;
          double v[3] = {sv.fx * ir3, sv.fy * ir3, sv.fz * ir3}, w[3] = {-v[0], -v[1], -v[2]};
          if constexpr (DENS) {
            const double ds = dx * sv.sx + dy * sv.sy + dz * sv.sz, dn = dx * sv.nx + dy * sv.ny + dz * sv.nz;
            const double dg = dx * sv.gx + dy * sv.gy + dz * sv.gz;
            A += (30.0 * ds * dn + 15.0 * dg) * ir5 * ir2;
            B -= (6.0 * ds * dn + 3.0 * dg) * ir5;
            const double fs[3] = {sv.sx, sv.sy, sv.sz}, nu[3] = {sv.nx, sv.ny, sv.nz}, g[3] = {sv.gx, sv.gy, sv.gz};
#pragma unroll
            for (int e = 0; e < 3; ++e) {
              v[e] -= (6.0 * (dn * fs[e] + ds * nu[e]) + 3.0 * g[e]) * ir5;
              w[e] -= 3.0 * g[e] * ir5;
            }
          }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b) gr[a][b] += d[a] * (A * d[b] + v[b]) + w[a] * d[b] + (a == b ? B : 0.0);
          }
        } else if constexpr (DENS) {
          const double ir5 = ir3 * ir * ir;
          const double ds = dx * sv.sx + dy * sv.sy + dz * sv.sz, dn = dx * sv.nx + dy * sv.ny + dz * sv.nz;
          if constexpr (OUT == 1) {
            const double sn = sv.sx * sv.nx + sv.sy * sv.ny + sv.sz * sv.nz;
            ux += 2.0 * df * ir3 + 4.0 * sn * ir3 - 12.0 * ds * dn * ir5;
          } else {
            const double dg = dx * sv.gx + dy * sv.gy + dz * sv.gz;
            const double c = df * ir3 - (3.0 * dg + 6.0 * ds * dn) * ir5;
            ux += sv.fx * ir + sv.gx * ir3 + dx * c;
            uy += sv.fy * ir + sv.gy * ir3 + dy * c;
            uz += sv.fz * ir + sv.gz * ir3 + dz * c;
          }
        } else if constexpr (OUT == 1) {
          ux += 2.0 * df * ir3;
        } else {
          const double c = df * ir3;
          ux += sv.fx * ir + dx * c;
          uy += sv.fy * ir + dy * c;
          uz += sv.fz * ir + dz * c;
        }
      }
    }
    if (act) {
      const int o = tout[k];
      if (OUT == 2) {
#pragma unroll
        for (int e = 0; e < 9; ++e) out[9 * (int64_t)o + e] += KSTOKES * gr[e / 3][e % 3];
      } else if (OUT == 1) {
        out[o] += KSTOKES * ux;
      } else {
        out[3 * (int64_t)o] += KSTOKES * ux;
        out[3 * (int64_t)o + 1] += KSTOKES * uy;
        out[3 * (int64_t)o + 2] += KSTOKES * uz;
      }
    }
    __syncwarp();
  }
}

template <int P>
void launch_stokes_l2p(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx,
                       const double* ty, const double* tz, const int* tout, int output, double* out) {
  Plan& P_ = *S.plan;
  const int LD = P_.cache->ld;
  if (output == FMMB_STOKES_GRADIENT) {
    const size_t smem = sizeof(double) * GW * (4 * LD + 12 * P * P);
    FMMB_CUDA(cudaFuncSetAttribute(k_stokes_l2p_grad<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_stokes_l2p_grad<P><<<(ng + GW - 1) / GW, GW * 32, smem, P_.ctx->stream>>>(
        gnode, gstart, gcount, ng, tx, ty, tz, tout, P_.cell.p, S.Pl.p, LD, geometry(P_), P_.d_scale.p, out);
    FMMB_LAUNCH_CHECK();
    return;
  }
  const bool pres = output == FMMB_STOKES_PRESSURE;
  const size_t smem = sizeof(double) * SW * 4 * LD;
  auto kern = pres ? k_stokes_l2p<P, true> : k_stokes_l2p<P, false>;
  FMMB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(ng + SW - 1) / SW, SW * 32, smem, P_.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, P_.cell.p, S.Pl.p,
                                                              LD, geometry(P_), P_.d_scale.p, out);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

// build_expansions! of a Stokes state from the densities of stokes_fmm_eval! (device, original
// order)
void stokes_build(State& S, const double* xyz_dev, const StokesDensities& d) {
  Plan& P = *S.plan;
  Cache& C = *P.cache;
  cudaStream_t s = P.ctx->stream;
  const int LD = C.ld;
  const int64_t n = P.N, pitch = 4 * (int64_t)LD;
  const bool dens = d.stresslets || d.doublets;
  if (S.f3.n < (size_t)(3 * n)) S.f3.alloc(3 * n);
  if (S.q.n < (size_t)n) S.q.alloc(n);
  if (dens && S.sd.n < (size_t)(9 * n)) S.sd.alloc(9 * n);
  if (dens && S.dip4.n < (size_t)(12 * n)) S.dip4.alloc(12 * n);
  k_stokes_gather<<<nblk(n), 256, 0, s>>>(xyz_dev, d, P.perm.p, n, S.xs.p, S.ys.p, S.zs.p, S.f3.p,
                                          dens ? S.sd.p : nullptr);
  FMMB_LAUNCH_CHECK();
  S.stokes_dens = dens;
  if (P.n_s2m > 0) {
    auto kern = dens ? k_stokes_q4<true> : k_stokes_q4<false>;
    kern<<<nblk((int64_t)P.n_s2m * 32), 256, 0, s>>>(P.s2m_nodes.p, P.n_s2m, P.cell.p, P.plo.p, P.phi.p, geometry(P),
                                                     P.d_scale.p, n, S.xs.p, S.ys.p, S.zs.p, S.f3.p,
                                                     dens ? S.sd.p : nullptr, S.q.p, dens ? S.dip4.p : nullptr);
    FMMB_LAUNCH_CHECK();
  }
  // P2M, one block at a time (charges, and the dipoles of the stresslets and doublets)
  for (int a = 0; a < 3; ++a)
    p2m_block(S, S.f3.p + a * n, dens ? S.dip4.p + 3 * a * n : nullptr, S.M.p + (int64_t)a * LD, pitch);
  p2m_block(S, S.q.p, dens ? S.dip4.p + 9 * n : nullptr, S.M.p + 3 * (int64_t)LD, pitch);
  // M2M, level by level: the stacked children of each block (Ψ̂ with the coupling), one product each
  for (int l = P.L - 2; l >= 2; --l) {
    const int c0 = P.level_start[l + 1], ng = P.level_groups[l + 1];
    if (ng == 0) continue;
    DBuf<double> X((size_t)ng * NCH * LD);
    for (int a = 0; a < 4; ++a) {
      k_stokes_m2m_in<<<nblk((int64_t)ng * NCH * LD), 256, 0, s>>>(S.M.p, c0, ng, LD, a, X.p);
      FMMB_LAUNCH_CHECK();
      ColMap bm{X.p, nullptr, 0, NCH}, cm{S.M.p + (int64_t)a * LD, P.group_parent[l + 1].p, 0, 0, pitch};
      gemm_expansions(LD, NCH * LD, P.lv_m2m[l], bm, cm, ng, LD, C.np, 0, P.ctx->num_sms, s);
    }
  }
  // M2L of every block (the Ψ̂ launch with the coupling), then L2L level by level
  m2l_stage(S);
  for (int l = 3; l < P.L; ++l) {
    const int c0 = P.level_start[l], ng = P.level_groups[l];
    if (ng == 0) continue;
    const int64_t per = (int64_t)ng * NCH * LD;
    DBuf<double> R(4 * per);
    for (int a = 0; a < 4; ++a) {
      ColMap bm{S.Pl.p + (int64_t)a * LD, P.group_parent[l].p, 0, 0, pitch}, cm{R.p + a * per, nullptr, 0, NCH};
      gemm_expansions(NCH * LD, LD, P.lv_l2l[l - 1], bm, cm, ng, LD, C.np, 0, P.ctx->num_sms, s);
    }
    k_stokes_l2l_out<<<nblk(per), 256, 0, s>>>(S.Pl.p, R.p, c0, ng, LD, C.np);
    FMMB_LAUNCH_CHECK();
  }
  S.built = true;
}

namespace {

// the far and near fields at ng groups of targets (per leaf: node, first, count), targets in
// group order with their output indices tout; self: the targets are the sources (i = j skipped)
void stokes_evaluate_groups(State& S, const int* gnode, const int* gstart, const int* gcount, int ng, const double* tx,
                            const double* ty, const double* tz, const int* tout, bool self, int output, double* out) {
  Plan& P = *S.plan;
  require(output == FMMB_STOKES_VELOCITY || output == FMMB_STOKES_PRESSURE || output == FMMB_STOKES_GRADIENT,
          FMMB_ERR_UNSUPPORTED, "Stokes outputs are the velocity, the pressure and the velocity gradient");
  if (ng == 0) return;
  switch (P.cache->p) {
#define X(pp) case pp: launch_stokes_l2p<pp>(S, gnode, gstart, gcount, ng, tx, ty, tz, tout, output, out); break;
    FMMB_P_CASES(X)
#undef X
    default: throw Error(FMMB_ERR_UNSUPPORTED, "p out of range");
  }
  const bool d = S.stokes_dens;
  using K = decltype(&k_stokes_near<true, true, 0>);
  const K table[2][2][3] = {{{k_stokes_near<false, false, 0>, k_stokes_near<false, false, 1>, k_stokes_near<false, false, 2>},
                             {k_stokes_near<false, true, 0>, k_stokes_near<false, true, 1>, k_stokes_near<false, true, 2>}},
                            {{k_stokes_near<true, false, 0>, k_stokes_near<true, false, 1>, k_stokes_near<true, false, 2>},
                             {k_stokes_near<true, true, 0>, k_stokes_near<true, true, 1>, k_stokes_near<true, true, 2>}}};
  const K kern = table[self][d][output];
  kern<<<(ng + SW - 1) / SW, SW * 32, 0, P.ctx->stream>>>(gnode, gstart, gcount, ng, tx, ty, tz, tout, S.xs.p, S.ys.p,
                                                          S.zs.p, S.f3.p, d ? S.sd.p : nullptr, P.N, P.plo.p, P.phi.p,
                                                          P.col.p, out);
  FMMB_LAUNCH_CHECK();
}

}  // namespace

// evaluate_at_sources! of a Stokes state: velocities (3 × n) or pressures (n), original order,
// device, self excluded
void stokes_evaluate_sources(State& S, int output, double* out_dev) {
  Plan& P = *S.plan;
  stokes_evaluate_groups(S, P.leaves.p, P.leaf_start.p, P.leaf_count.p, P.n_leaves, S.xs.p, S.ys.p, S.zs.p, P.perm.p, true,
                         output, out_dev);
}

// evaluate! of a Stokes state at nt targets (device, 3 × nt): velocities (3 × nt) or pressures
// (nt) in the targets' order, device
void stokes_evaluate_targets(State& S, const double* tg_dev, int64_t nt, int output, double* out_dev) {
  if (nt == 0) return;
  const int ng = group_targets(S, tg_dev, nt);
  const int* g = S.t_groups.p;
  stokes_evaluate_groups(S, g, g + ng, g + 2 * ng, ng, S.t_x.p, S.t_y.p, S.t_z.p, S.t_out.p, false, output, out_dev);
}

}  // namespace fmmb
