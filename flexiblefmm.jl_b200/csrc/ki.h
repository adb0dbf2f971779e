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

}  // namespace fmmb
