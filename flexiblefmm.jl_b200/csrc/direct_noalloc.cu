// fmmb_direct_noalloc_dev: the FP64 direct sums of fmmb_direct_dev without any device
// allocation. It exists for callers that cannot call cudaMalloc: an application whose
// device memory is held by a pool of its own (CUDA.jl's allocator keeps what it reserved,
// and a cudaMalloc outside it can fail once that pool holds the device), or a time-stepping
// loop that must not pay cudaMalloc's implicit device synchronisation on every error check.
// The caller passes the inputs and outputs; the partial sums go to a fixed scratch array
// compiled into the library.
//
// The scratch: a file-scope __device__ array of SCRATCH_DOUBLES doubles (4 MiB) that every GPU
// loading the library holds until the process exits. A call splits the sources into at most
// 32 ranges and needs 4 doubles per (range, target), so it takes at most 131,072 targets
// (nt · 4 ≤ SCRATCH_DOUBLES with one range); larger nt is rejected with FMMB_ERR_ARGUMENT.
// Every entry the reduction reads is written by the same call first, so nothing has to
// start at zero; the array keeps the last call's partial sums. All calls share the one
// array: calls that overlap on the GPU (several streams, several host threads) race on it.
//
// Host code cannot use the array's name as a device address (it names a host-side
// stand-in); the device address comes from cudaGetSymbolAddress, taken once per device on
// the first call made with that device current. Make that first call before any stream
// capture begins.
#include <mutex>

#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int64_t SCRATCH_DOUBLES = 1 << 19;   // 4 MiB
constexpr int MAX_SPLIT = 32;
constexpr int NT = 128;                        // targets per CTA and sources per staged tile

static __device__ __align__(256) double g_direct_scratch[SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_ptr[MAX_DEVICES] = {};

// the scratch array's device address on the current device (set up once per device)
double* scratch_address() {
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < MAX_DEVICES, FMMB_ERR_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    FMMB_CUDA(cudaGetSymbolAddress(&p, g_direct_scratch));
    g_scratch_ptr[dev] = (double*)p;
  }
  return g_scratch_ptr[dev];
}

__global__ void __launch_bounds__(NT) k_direct_partial(const double* __restrict__ src, const double* __restrict__ tau,
                                                       int64_t ns, const double* __restrict__ tgt,
                                                       const int64_t* __restrict__ self_idx, int64_t nt, int nsplit,
                                                       double* __restrict__ part) {
  __shared__ double sx[NT], sy[NT], sz[NT], sq[NT];
  const int64_t t = (int64_t)blockIdx.x * NT + threadIdx.x;
  const int sp = blockIdx.y;
  const int64_t s0 = ns * sp / nsplit, s1 = ns * (sp + 1) / nsplit;
  const bool act = t < nt;
  const double x = act ? tgt[3 * t] : 0, y = act ? tgt[3 * t + 1] : 0, z = act ? tgt[3 * t + 2] : 0;
  const int64_t me = (act && self_idx) ? self_idx[t] : -1;
  double u = 0, gx = 0, gy = 0, gz = 0;
  for (int64_t b = s0; b < s1; b += NT) {
    __syncthreads();
    const int64_t j = b + threadIdx.x;
    if (j < s1) { sx[threadIdx.x] = src[3 * j]; sy[threadIdx.x] = src[3 * j + 1]; sz[threadIdx.x] = src[3 * j + 2]; sq[threadIdx.x] = tau[j]; }
    __syncthreads();
    const int m = (int)min((int64_t)NT, s1 - b);
    for (int i = 0; i < m; ++i) {
      const double dx = x - sx[i], dy = y - sy[i], dz = z - sz[i];
      const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
      const double ir = (b + i == me) ? 0.0 : 1.0 / sqrt(r2);
      const double qi = sq[i] * ir, qi3 = qi * ir * ir;
      u += qi; gx += qi3 * dx; gy += qi3 * dy; gz += qi3 * dz;
    }
  }
  if (act) {
    double* o = part + ((int64_t)sp * nt + t) * 4;
    o[0] = u; o[1] = gx; o[2] = gy; o[3] = gz;
  }
}

__global__ void k_direct_sum(const double* __restrict__ part, int64_t nt, int nsplit, double* __restrict__ pot,
                             double* __restrict__ grad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double u = 0, gx = 0, gy = 0, gz = 0;
  for (int sp = 0; sp < nsplit; ++sp) {
    const double* o = part + ((int64_t)sp * nt + t) * 4;
    u += o[0]; gx += o[1]; gy += o[2]; gz += o[3];
  }
  if (pot) pot[t] = KC * u;
  if (grad) { grad[3 * t] = -KC * gx; grad[3 * t + 1] = -KC * gy; grad[3 * t + 2] = -KC * gz; }
}

}  // namespace

// enqueues on the context's stream; no allocation, no synchronisation
void direct_noalloc(Ctx& ctx, const double* src, const double* tau, int64_t ns, const double* tgt, const int64_t* self_idx,
                    int64_t nt, double* pot, double* grad) {
  require(nt * 4 <= SCRATCH_DOUBLES, FMMB_ERR_ARGUMENT,
          "fmmb_direct_noalloc_dev takes at most " + std::to_string(SCRATCH_DOUBLES / 4) + " targets (scratch of " +
              std::to_string(SCRATCH_DOUBLES * 8 >> 20) + " MiB); got " + std::to_string(nt));
  if (nt == 0) return;
  double* part = scratch_address();
  const int tb = (int)((nt + NT - 1) / NT);
  int nsplit = std::max(1, std::min<int>(MAX_SPLIT, (4 * ctx.num_sms + tb - 1) / tb));
  nsplit = (int)std::max<int64_t>(1, std::min<int64_t>(nsplit, SCRATCH_DOUBLES / (4 * nt)));
  k_direct_partial<<<dim3(tb, nsplit), NT, 0, ctx.stream>>>(src, tau, ns, tgt, self_idx, nt, nsplit, part);
  FMMB_LAUNCH_CHECK();
  k_direct_sum<<<(unsigned)((nt + 255) / 256), 256, 0, ctx.stream>>>(part, nt, nsplit, pot, grad);
  FMMB_LAUNCH_CHECK();
}

}  // namespace fmmb
