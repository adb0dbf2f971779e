// The D4h signed permutations of the real harmonic storage, computed from each far offset's
// group element (src/operators/symmetry.jl:252-319): for an entry of order m, a rotation by
// kπ/2 multiplies the coefficient by i^{±mk} (a quarter-turn count q swaps the real and
// imaginary entries when odd), εz multiplies by (−1)^{n+m}, εy conjugates. The source side
// (P_sᵀ, the gather) uses −mk, the target side (P_t, the scatter) +mk.
#pragma once
#include "common.cuh"

namespace fmmb {

// per far offset: rotation k (bits 0-1) | εy << 2 | εz << 3, uploaded by upload_d4h
extern __constant__ int c_d4h[NFAR];
void upload_d4h(const HostOperators& h, cudaStream_t s);

// (n, m, part) of entry k of the real storage: part 0 for m = 0, 1 for Re, 2 for Im
__host__ __device__ __forceinline__ void coef_nmp(int k, int& n, int& m, int& part) {
  n = (int)sqrtf((float)k + 0.5f);
  while (n * n > k) --n;
  while ((n + 1) * (n + 1) <= k) ++n;
  const int r = k - n * n;
  m = (r + 1) >> 1;
  part = r == 0 ? 0 : ((r & 1) ? 1 : 2);
}

// the sign of an entry of the given part, for q quarter-turns and n + m
__host__ __device__ __forceinline__ int perm_sign(int part, int q, int npm, int fac) {
  const int s = ((fac & 8) && (npm & 1)) ? -1 : 1;
  if (part == 0) return s;
  if (part == 1) return q < 2 ? s : -s;
  const int sig = (fac & 4) ? -1 : 1;
  return (q == 0 || q == 3) ? s * sig : -s * sig;
}

}  // namespace fmmb
