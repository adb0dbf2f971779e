// CubeKernelIndependent{3}(Laplace3D(); p, pc, d): host operators (ki_operators.cpp) and the
// device passes (ki.cu).
#pragma once
#include <vector>

#include "common.cuh"

namespace fmmb {

constexpr int KI_PMAX = 12;   // points per edge of the small surface; the spectral lattice is (2p)³

struct KIHost {
  int p = 0, pc = 0, ns = 0, nl = 0;   // points per edge, small / large surface points
  double d = 0, w = 0, h = 0;          // margin, the width built at, the small lattice's spacing
  std::vector<double> small, large;    // 3 × ns, 3 × nl, relative to the box centre at width w
  std::vector<int> embed;              // ns: index in the (2p)³ lattice, coordinate 1 fastest
  int rank_up = 0, rank_down = 0;
  std::vector<double> up_v, up_su;     // P_up = V (ns × r) · S⁺Uᴴ (r × nl)
  std::vector<double> down_v, down_su; // P_down = V (nl × r) · S⁺Uᴴ (r × ns)
  std::vector<double> m2m, l2l;        // ns × 8ns, 8ns × ns (column-major, pseudo-inverses folded in)
  // the spectral M2L (spectral_m2l.jl:174-193): per far offset the DFT of the kernel table
  // κ_o(m) = K(o·w, h·m), m ∈ [−(p−1), p−1]³ at wrapped index m mod 2p, over the half spectrum
  // (k1 ≤ p; (p+1)·(2p)² entries, k1 fastest), as (re, im) pairs
  int nfreq = 0;
  std::vector<double> tables;          // NFAR × nfreq × 2
};
KIHost build_ki_operators(int p, int pc, double d, double rtol, double w);

// KernelIndependent(Laplace2D(); nequiv) (src/operators/kifmm.jl): circles of N equispaced
// points, radius √2/2·w (small: upward equivalent, downward check) and (4 − √2)/2·w (large),
// the operators of one width (the log kernel is not homogeneous), column-major and zero-padded
// to CLD = roundup(N, 64): the factored pseudo-inverses (V, S⁺Uᴴ each CLD × CLD), M2M
// (CLD × 8·CLD) and L2L (8·CLD × CLD) over the eight child slots of the embedding octree (a slot's
// circle centre is its (x, y) offset; both z halves map alike), and the M2L check maps of the 316
// far offsets (CLD × CLD each; only the in-plane offsets, oz = 0, are filled)
struct KICircleLevel {
  int n = 0, ld = 0, rank_up = 0, rank_down = 0;
  std::vector<double> up_v, up_su, down_v, down_su, m2m, l2l, m2l;
};
KICircleLevel build_ki_circle_level(int n, double rtol, double w);
constexpr double KIC_SMALL = 0.70710678118654752440;   // √2/2
constexpr double KIC_LARGE = 1.29289321881345247560;   // (4 − √2)/2

}  // namespace fmmb
