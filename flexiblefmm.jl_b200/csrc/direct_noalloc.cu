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
// stand-in); the device address comes from cudaGetSymbolAddress. The library takes it when a
// context is created (fmmb_ctx_create, with its device current), so the module holding the
// array is loaded at set-up rather than inside the first call; it is kept per CUDA context, so
// a reset device (a new primary context) resolves it again on its next call. Create the context
// before any stream capture begins.
#include <cuda.h>

#include <mutex>
#include <utility>
#include <vector>

#include "passes.cuh"

namespace fmmb {
namespace {

constexpr int64_t SCRATCH_DOUBLES = 1 << 19;   // 4 MiB
constexpr int MAX_SPLIT = 32;

static __device__ __align__(256) double g_direct_scratch[SCRATCH_DOUBLES];

std::mutex g_mu;
std::vector<std::pair<CUcontext, double*>> g_scratch;   // per CUDA context: the array's address

// the current CUDA context (the driver's cuCtxGetCurrent, through the runtime's entry-point query)
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    FMMB_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q));
    require(f != nullptr && q == cudaDriverEntryPointSuccess, FMMB_ERR_DEVICE, "cuCtxGetCurrent is not available");
    fn = (Fn)f;
  }
  CUcontext c = nullptr;
  require(fn(&c) == CUDA_SUCCESS && c != nullptr, FMMB_ERR_DEVICE, "no current CUDA context");
  return c;
}

// the scratch array's device address in the current context (resolved once per context)
double* scratch_address() {
  FMMB_CUDA(cudaFree(nullptr));                     // makes the device's primary context current
  const CUcontext c = current_context();
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& e : g_scratch)
    if (e.first == c) return e.second;
  void* p = nullptr;
  FMMB_CUDA(cudaGetSymbolAddress(&p, g_direct_scratch));
  g_scratch.emplace_back(c, (double*)p);
  return (double*)p;
}

}  // namespace

void direct_noalloc_prepare() { scratch_address(); }

// enqueues on the context's stream; no allocation, no synchronisation. The partial sums use the
// kernels of fmmb_direct_dev; only the split of the sources differs (at most MAX_SPLIT ranges,
// and as many as the scratch holds for nt targets)
void direct_noalloc(Ctx& ctx, const double* src, const double* tau, int64_t ns, const double* tgt, const int64_t* self_idx,
                    int64_t nt, double* pot, double* grad) {
  require(nt * 4 <= SCRATCH_DOUBLES, FMMB_ERR_ARGUMENT,
          "fmmb_direct_noalloc_dev takes at most " + std::to_string(SCRATCH_DOUBLES / 4) + " targets (scratch of " +
              std::to_string(SCRATCH_DOUBLES * 8 >> 20) + " MiB); got " + std::to_string(nt));
  if (nt == 0) return;
  double* part = scratch_address();
  const int tb = (int)((nt + DT - 1) / DT);
  int nsplit = std::max(1, std::min<int>(MAX_SPLIT, (4 * ctx.num_sms + tb - 1) / tb));
  nsplit = (int)std::max<int64_t>(1, std::min<int64_t>(nsplit, SCRATCH_DOUBLES / (4 * nt)));
  k_direct<<<dim3(tb, nsplit), DT, 0, ctx.stream>>>(src, tau, ns, tgt, self_idx, nt, nsplit, part);
  FMMB_LAUNCH_CHECK();
  k_direct_reduce<<<(unsigned)((nt + 255) / 256), 256, 0, ctx.stream>>>(part, nt, nsplit, pot, grad);
  FMMB_LAUNCH_CHECK();
}

}  // namespace fmmb
