// Exclusive prefix sums and an LSD radix sort of 64-bit keys with 32-bit payloads.
//
// The reference builds its tree with the backend's sortperm! and a serial-per-block
// KernelAbstractions scan (src/tree/device_builder.jl:413, src/device_lists.jl:173-210).
// Here: a three-phase scan (tile sums, scan of the sums, tile scan with offsets) over
// 4096-element tiles, and an 8-bit-digit LSD radix sort whose passes are a per-tile digit
// histogram, a digit-major scan of the histograms and a stable per-tile scatter (warp
// multisplit with __match_any_sync: ranks within a warp by lane order, across the warps of a
// tile by warp order, across tiles by the digit-major scan). Both are HBM-bound integer work.
#include "scan_sort.cuh"

namespace fmmb {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// inclusive scan of one value per thread across a block of blockDim.x threads (≤ 1024)
template <class T>
__device__ T block_inclusive_scan(T v, T* smem_warp) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) smem_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nw ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T u = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += u;
    }
    if (lane < nw) smem_warp[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += smem_warp[warp - 1];
  __syncthreads();
  return v;
}

__global__ void k_tile_sums(const int* __restrict__ in, int64_t n, int* __restrict__ sums) {
  __shared__ int sw[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  int s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t j = base + (int64_t)i * SCAN_THREADS + threadIdx.x;
    if (j < n) s += in[j];
  }
  s = block_inclusive_scan(s, sw);
  if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = s;
}

__global__ void k_tile_scan(const int* __restrict__ in, int64_t n, const int* __restrict__ offs, int* __restrict__ out) {
  __shared__ int sw[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t j = base + i;
    v[i] = j < n ? in[j] : 0;
    s += v[i];
  }
  int incl = block_inclusive_scan(s, sw);
  int run = incl - s + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t j = base + i;
    if (j < n) out[j] = run;
    run += v[i];
  }
}

// ---- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;                      // per thread
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;    // 4096 keys per tile
constexpr int RS_BINS = 256;

__global__ void k_digit_hist(const uint64_t* __restrict__ keys, int64_t n, int shift, int ntiles, int* __restrict__ hist) {
  __shared__ int h[RS_BINS];
  for (int b = threadIdx.x; b < RS_BINS; b += blockDim.x) h[b] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * RS_TILE;
  for (int i = threadIdx.x; i < RS_TILE; i += RS_THREADS) {
    int64_t j = base + i;
    if (j < n) atomicAdd(&h[(int)((keys[j] >> shift) & 0xff)], 1);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < RS_BINS; b += blockDim.x) hist[(int64_t)b * ntiles + blockIdx.x] = h[b];
}

// stable scatter of one tile: the keys of warp w are tile positions w·512 + it·32 + lane
__global__ void k_digit_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, int64_t n, int shift,
                                int ntiles, const int* __restrict__ offs, uint64_t* __restrict__ kout,
                                uint32_t* __restrict__ vout) {
  __shared__ int wc[RS_WARPS][RS_BINS];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int b = threadIdx.x; b < RS_WARPS * RS_BINS; b += RS_THREADS) (&wc[0][0])[b] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)warp * (RS_ITEMS * 32);
  uint64_t key[RS_ITEMS];
  uint32_t val[RS_ITEMS];
  int rank[RS_ITEMS];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < RS_ITEMS; ++it) {
    int64_t j = base + it * 32 + lane;
    bool ok = j < n;
    key[it] = ok ? kin[j] : 0;
    val[it] = ok ? vin[j] : 0;
    int d = ok ? (int)((key[it] >> shift) & 0xff) : RS_BINS;   // out-of-range keys in their own group
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(peers) - 1;
    int before = 0;
    if (ok && lane == leader) {
      before = wc[warp][d];
      wc[warp][d] = before + __popc(peers);
    }
    before = __shfl_sync(0xffffffffu, before, leader);
    rank[it] = before + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // per digit: the exclusive prefix over the warps of the tile
  for (int b = threadIdx.x; b < RS_BINS; b += RS_THREADS) {
    int run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
      int t = wc[w][b];
      wc[w][b] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < RS_ITEMS; ++it) {
    int64_t j = base + it * 32 + lane;
    if (j < n) {
      int d = (int)((key[it] >> shift) & 0xff);
      int64_t pos = (int64_t)offs[(int64_t)d * ntiles + blockIdx.x] + wc[warp][d] + rank[it];
      kout[pos] = key[it];
      vout[pos] = val[it];
    }
  }
}

}  // namespace

void scan_exclusive(const int* in, int* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  int64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  require(ntiles < (1ll << 31), FMMB_ERR_ARGUMENT, "scan too large");
  if (ntiles == 1) {
    k_tile_scan<<<1, SCAN_THREADS, 0, s>>>(in, n, nullptr, out);
    FMMB_LAUNCH_CHECK();
    return;
  }
  DBuf<int> sums(ntiles), offs(ntiles);
  k_tile_sums<<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, n, sums.p);
  FMMB_LAUNCH_CHECK();
  scan_exclusive(sums.p, offs.p, ntiles, s);
  k_tile_scan<<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, n, offs.p, out);
  FMMB_LAUNCH_CHECK();
  FMMB_CUDA(cudaStreamSynchronize(s));   // the temporaries are freed on return
}

int64_t scan_exclusive_total(const int* in, int* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0;
  scan_exclusive(in, out, n, s);
  int a = read_one(out + n - 1, s), b = read_one(in + n - 1, s);
  return (int64_t)a + b;
}

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, int bits, cudaStream_t s) {
  if (n <= 1) return;
  require(n < (1ll << 31), FMMB_ERR_ARGUMENT, "sort too large");
  int ntiles = (int)((n + RS_TILE - 1) / RS_TILE);
  DBuf<uint64_t> k2(n);
  DBuf<uint32_t> v2(n);
  DBuf<int> hist((size_t)RS_BINS * ntiles), offs((size_t)RS_BINS * ntiles);
  uint64_t *ka = keys, *kb = k2.p;
  uint32_t *va = vals, *vb = v2.p;
  int passes = (bits + 7) / 8;
  for (int ps = 0; ps < passes; ++ps) {
    int shift = 8 * ps;
    k_digit_hist<<<ntiles, RS_THREADS, 0, s>>>(ka, n, shift, ntiles, hist.p);
    FMMB_LAUNCH_CHECK();
    scan_exclusive(hist.p, offs.p, (int64_t)RS_BINS * ntiles, s);
    k_digit_scatter<<<ntiles, RS_THREADS, 0, s>>>(ka, va, n, shift, ntiles, offs.p, kb, vb);
    FMMB_LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    FMMB_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb
