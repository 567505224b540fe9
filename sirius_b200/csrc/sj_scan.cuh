// Device-wide exclusive prefix sum (reduce -> scan of block sums -> downsweep), used for the
// grouped build's per-slot offsets and for the grouped probe's output offsets. The element count
// may live in device memory (written by an earlier kernel on the same stream), so no host
// synchronisation is needed between a count pass and the scan that follows it.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sj {

constexpr int kScanBlocks = 1024;  // CTAs of the reduce / downsweep kernels
constexpr int kScanThreads = 256;

template <int BLOCK>
__device__ __forceinline__ int64_t block_exclusive_sum(int64_t v, int64_t* s_warp, int64_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NW = BLOCK / 32;
  int64_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < NW ? s_warp[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += y;
    }
    if (lane < NW) s_warp[lane] = w;
  }
  __syncthreads();
  const int64_t base = wid ? s_warp[wid - 1] : 0;
  total = s_warp[NW - 1];
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ int64_t scan_n(const unsigned long long* d_n, int64_t n_host) {
  return d_n ? (int64_t)*d_n : n_host;
}

template <typename Tin>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const Tin* __restrict__ in,
                                                                   const unsigned long long* d_n,
                                                                   int64_t n_host, int64_t* bsum) {
  __shared__ int64_t s_warp[kScanThreads / 32];
  const int64_t n = scan_n(d_n, n_host);
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  int64_t acc = 0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kScanThreads) acc += (int64_t)in[i];
  int64_t tot;
  block_exclusive_sum<kScanThreads>(acc, s_warp, tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// One CTA of 1024 threads: exclusive scan of kScanBlocks block sums, in place.
static __global__ void __launch_bounds__(1024) scan_bsum_kernel(int64_t* bsum) {
  __shared__ int64_t s_warp[32];
  int64_t v = threadIdx.x < kScanBlocks ? bsum[threadIdx.x] : 0;
  int64_t tot;
  int64_t ex = block_exclusive_sum<1024>(v, s_warp, tot);
  if (threadIdx.x < kScanBlocks) bsum[threadIdx.x] = ex;
}

// out has n + 1 entries; out[n] = total.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const Tin* __restrict__ in,
                                                                 const unsigned long long* d_n,
                                                                 int64_t n_host,
                                                                 const int64_t* __restrict__ bsum,
                                                                 Tout* __restrict__ out) {
  __shared__ int64_t s_warp[kScanThreads / 32];
  const int64_t n = scan_n(d_n, n_host);
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  if (n == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = (Tout)0;
    return;
  }
  int64_t run = bsum[blockIdx.x];
  for (int64_t t0 = lo; t0 < hi; t0 += kScanThreads) {
    const int64_t i = t0 + threadIdx.x;
    const int64_t v = i < hi ? (int64_t)in[i] : 0;
    int64_t tot;
    const int64_t ex = block_exclusive_sum<kScanThreads>(v, s_warp, tot);
    if (i < hi) out[i] = (Tout)(run + ex);
    if (i < hi && i == n - 1) out[n] = (Tout)(run + ex + v);  // the total
    run += tot;
  }
}

// Host launcher. d_n: optional device count (overrides n_host). tmp: kScanBlocks int64.
template <typename Tin, typename Tout>
inline void device_exclusive_scan(const Tin* in, Tout* out, const unsigned long long* d_n,
                                  int64_t n_host, int64_t* tmp, cudaStream_t s) {
  scan_reduce_kernel<Tin><<<kScanBlocks, kScanThreads, 0, s>>>(in, d_n, n_host, tmp);
  scan_bsum_kernel<<<1, 1024, 0, s>>>(tmp);
  scan_down_kernel<Tin, Tout><<<kScanBlocks, kScanThreads, 0, s>>>(in, d_n, n_host, tmp, out);
}

}  // namespace sj
