// Shared definitions of the fmmb library: errors, device buffers, the plan/state structs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fmmb.h"

namespace fmmb {

// An exception carrying an ABI status code; the entry points turn it into a return value.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FMMB_CUDA(call)                                                                                \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      throw ::fmmb::Error(e_ == cudaErrorMemoryAllocation ? FMMB_ERR_MEMORY : FMMB_ERR_DEVICE,          \
                          std::string(#call) + ": " + cudaGetErrorString(e_));                          \
  } while (0)
#define FMMB_LAUNCH_CHECK() FMMB_CUDA(cudaGetLastError())

inline void require(bool ok, int code, const std::string& msg) {
  if (!ok) throw Error(code, msg);
}

// The stream the calling thread's allocations are ordered on (the context's stream, set by
// every entry point): device buffers come from the stream-ordered allocator, so allocating and
// freeing never synchronises the whole device (independent requests on other streams keep
// running). Outside an entry point (no stream set) plain cudaMalloc/cudaFree are used.
inline thread_local cudaStream_t g_alloc_stream = nullptr;

// A device allocation owned by its holder (moves only); freed on the stream it was allocated on.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  static void raw_alloc(T** q, size_t count, cudaStream_t st) {
    if (st) FMMB_CUDA(cudaMallocAsync((void**)q, count * sizeof(T), st));
    else FMMB_CUDA(cudaMalloc((void**)q, count * sizeof(T)));
  }
  void alloc(size_t count) {
    release();
    n = count;
    s = g_alloc_stream;
    if (count) raw_alloc(&p, count, s);
  }
  // grow to at least `count` entries, keeping the first `keep`
  void grow(size_t count, size_t keep, cudaStream_t st) {
    if (count <= n) return;
    size_t cap = std::max(count, n * 2);
    T* q = nullptr;
    raw_alloc(&q, cap, g_alloc_stream);
    if (keep && p) FMMB_CUDA(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st));
    FMMB_CUDA(cudaStreamSynchronize(st));
    release();
    p = q;
    n = cap;
    s = g_alloc_stream;
  }
  void release() {
    if (p) {
      if (s) cudaFreeAsync(p, s);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

template <class T>
inline void to_device(DBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
  d.alloc(h.size());
  if (!h.empty()) FMMB_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}
template <class T>
inline std::vector<T> to_host(const T* d, size_t n, cudaStream_t s) {
  std::vector<T> h(n);
  if (n) FMMB_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  return h;
}
template <class T>
inline T read_one(const T* d, cudaStream_t s) {
  T v;
  FMMB_CUDA(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  return v;
}

constexpr int NCH = 8;     // children per node (3D)
constexpr int NCOL = 27;   // colleague slots
constexpr int NFAR = 316;  // far offsets
constexpr int NCLASS = 34; // D4h classes of the far offsets
constexpr int PMAX = 20;

// node flags
constexpr uint8_t F_LEAF = 1, F_GHOST = 2, F_XLIST = 4, F_SOURCE = 8;

inline int ld_of(int p) {  // padded leading dimension of an expansion column
  int np = (p + 1) * (p + 1);
  return (np + 63) / 64 * 64;
}

// ---------------------------------------------------------------- host-side operators
// (built in operators.cpp; FP64, column-major, padded to LD)
struct HostOperators {
  int p = 0, np = 0, ld = 0;
  std::vector<double> m2m;    // LD × 8LD: block k (child slot) in columns k·LD ..
  std::vector<double> l2l;    // 8LD × LD: block k in rows k·LD ..
  std::vector<double> reps;   // 34 × (LD × LD), c_K / W_ref folded in
  std::vector<int> cls;       // 316: class of each far offset
  std::vector<int> reps_off;  // 34 × 3 canonical offsets
  std::vector<int16_t> gidx;  // 316 × LD: gather source row (P_sᵀ), -1 on padding rows
  std::vector<int8_t> gsgn;   // 316 × LD
  std::vector<int16_t> sidx;  // 316 × LD: scatter source row (P_t applied as a gather)
  std::vector<int8_t> ssgn;   // 316 × LD
  std::vector<int8_t> faroff; // 316 × 3: the far offsets (source cell − target cell), table order
  std::vector<uint8_t> d4h;   // 316: the D4h element mapping the class representative to the
                              // offset, as rotation k (bits 0-1) | εy << 2 | εz << 3
  std::vector<double> tables; // a, b, cz, cm, cp (each ntri) then e (p): the recurrences
  int ntri = 0;
};
HostOperators build_operators(int p, double ref_width);

}  // namespace fmmb
