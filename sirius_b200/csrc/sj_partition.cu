// Radix partitioning for the partitioned join variant (tables larger than L2).
//
// Rows are split by the top `pbits` bits of mix64(key) — the same bits that select a key's
// segment of the partitioned hash table — so after partitioning, partition p's probe rows only
// touch table segment p and the build payload rows stored with it. Processing partitions in order
// keeps one segment (a few MB) resident in the 126 MB L2 while its probes stream through, which
// turns the probe's random DRAM accesses (~40 G/s on B200) into L2 hits.
//
// Two passes over the input, both with a fixed grid of G CTAs where CTA c owns the contiguous row
// range [c*chunk, (c+1)*chunk):
//   1. histogram: per-CTA counts of the valid rows of each partition (shared-memory atomics,
//      warp-aggregated with __match_any_sync), stored partition-major as hist[p * G + c];
//   2. an exclusive scan of hist gives every (partition, CTA) its output offset; the scatter pass
//      re-reads the rows tile by tile, counting-sorts each tile by partition in shared memory and
//      writes key, row id and payloads (validity as one byte per row) as contiguous runs.
//      NULL-key rows are dropped (they never match).
// The outputs are partition-major: partition p occupies [off[p*G], off[(p+1)*G]).
#include <algorithm>

#include "sj_partition.cuh"
#include "sj_scan.cuh"

namespace sj {

constexpr int kPartThreads = 256;
constexpr int kMaxPartBits = kMaxPartitionBits;

__device__ __forceinline__ int partition_of(uint64_t kb, int pbits) {
  return pbits ? (int)(mix64(kb) >> (64 - pbits)) : 0;
}

template <typename K>
__global__ void __launch_bounds__(kPartThreads) part_hist_kernel(PartSrc s, int pbits, int64_t chunk, bool vec,
                                                                 int32_t* hist) {
  extern __shared__ int32_t h[];
  const int P = 1 << pbits;
  for (int p = threadIdx.x; p < P; p += blockDim.x) h[p] = 0;
  __syncthreads();
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < s.n ? lo + chunk : s.n;
  const K* keys = static_cast<const K*>(s.keys);
  for (int64_t i0 = lo + (int64_t)threadIdx.x * 4; i0 < hi; i0 += (int64_t)blockDim.x * 4) {
    K k[4];
    if (vec && i0 + 4 <= hi) {
      if (sizeof(K) == 4) {
        const int4 x = __ldcs(reinterpret_cast<const int4*>(keys + i0));
        k[0] = (K)x.x; k[1] = (K)x.y; k[2] = (K)x.z; k[3] = (K)x.w;
      } else {
        const longlong2 x = __ldcs(reinterpret_cast<const longlong2*>(keys + i0));
        const longlong2 y = __ldcs(reinterpret_cast<const longlong2*>(keys + i0) + 1);
        k[0] = (K)x.x; k[1] = (K)x.y; k[2] = (K)y.x; k[3] = (K)y.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) k[j] = i0 + j < hi ? __ldcs(keys + i0 + j) : (K)0;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (i0 + j < hi && bit_valid(s.kvalid, s.kvoff, i0 + j)) atomicAdd(&h[partition_of(key_u64<K>(k[j]), pbits)], 1);
  }
  __syncthreads();
  for (int p = threadIdx.x; p < P; p += blockDim.x) hist[(int64_t)p * gridDim.x + blockIdx.x] = h[p];
}

// Scatter pass, staged through shared memory one tile of kTile rows at a time: the tile's rows
// are counted per partition, sorted by partition in shared memory (counting sort), and every
// partition's run is then written to its output range with consecutive threads on consecutive
// positions, so each write front advances in whole sectors instead of one row per warp store.
constexpr int kTileRowsPerThread = 8;
constexpr int kTile = kPartThreads * kTileRowsPerThread;

struct ScatterSmem {
  // offsets into the dynamic shared-memory block; payloads stay in the tile's natural row order
  // (loaded together with the keys) and are reached from a sorted slot through `nat`
  size_t cur, tcnt, toff, key, rid, part, nat, pay[kMaxPayload], val[kMaxPayload], total;
};

static ScatterSmem scatter_smem(int pbits, int kw, const PartSrc& s) {
  const size_t P = (size_t)1 << pbits;
  ScatterSmem m{};
  size_t o = 0;
  auto take = [&](size_t b) {
    size_t r = o;
    o += (b + 15) & ~(size_t)15;
    return r;
  };
  m.cur = take(P * 8);
  m.tcnt = take(P * 4);
  m.toff = take(P * 4);
  m.key = take((size_t)kTile * kw);
  m.rid = take((size_t)kTile * 4);
  m.part = take((size_t)kTile * 2);
  m.nat = take((size_t)kTile * 2);
  for (int c = 0; c < s.n_pay; ++c) {
    m.pay[c] = take((size_t)kTile * s.pay[c].width);
    m.val[c] = s.pay[c].valid ? take(kTile) : 0;
  }
  m.total = o;
  return m;
}

template <typename K>
__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(PartSrc s, int pbits, int64_t chunk,
                                                                    const int64_t* __restrict__ off, PartDst d,
                                                                    ScatterSmem m) {
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned long long* cur = reinterpret_cast<unsigned long long*>(sm + m.cur);
  unsigned int* tcnt = reinterpret_cast<unsigned int*>(sm + m.tcnt);
  unsigned int* toff = reinterpret_cast<unsigned int*>(sm + m.toff);
  K* skey = reinterpret_cast<K*>(sm + m.key);
  int32_t* srid = reinterpret_cast<int32_t*>(sm + m.rid);
  uint16_t* spart = reinterpret_cast<uint16_t*>(sm + m.part);
  uint16_t* snat = reinterpret_cast<uint16_t*>(sm + m.nat);
  __shared__ unsigned int s_wsum[kPartThreads / 32];
  const int P = 1 << pbits;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int p = tid; p < P; p += kPartThreads) cur[p] = (unsigned long long)off[(int64_t)p * gridDim.x + blockIdx.x];
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < s.n ? lo + chunk : s.n;
  const K* keys = static_cast<const K*>(s.keys);
  K* okeys = static_cast<K*>(d.keys);
  for (int64_t t0 = lo; t0 < hi; t0 += kTile) {
    for (int p = tid; p < P; p += kPartThreads) tcnt[p] = 0;
    __syncthreads();
    // 1. load rows, partition, rank within the tile's partition
    int pr[kTileRowsPerThread];
    unsigned rank[kTileRowsPerThread];
    K kk[kTileRowsPerThread];
#pragma unroll
    for (int j = 0; j < kTileRowsPerThread; ++j) {
      const int64_t i = t0 + j * kPartThreads + tid;
      pr[j] = -1;
      kk[j] = 0;
      if (i < hi && bit_valid(s.kvalid, s.kvoff, i)) {
        kk[j] = __ldcs(keys + i);
        pr[j] = partition_of(key_u64<K>(kk[j]), pbits);
        const int nat = j * kPartThreads + tid;
        for (int c = 0; c < s.n_pay; ++c) {
          const PayloadIn& in = s.pay[c];
          store_elem(sm + m.pay[c], nat, in.width, load_elem(in.data, i, in.width));
          if (in.valid) sm[m.val[c] + nat] = bit_valid(in.valid, in.voff, i) ? 1 : 0;
        }
      }
      const unsigned peers = __match_any_sync(kFullMask, pr[j]);
      const int leader = __ffs(peers) - 1;
      unsigned base = 0;
      if (pr[j] >= 0 && lane == leader) base = atomicAdd(&tcnt[pr[j]], (unsigned)__popc(peers));
      base = __shfl_sync(kFullMask, base, leader);
      rank[j] = base + __popc(peers & ((1u << lane) - 1));
    }
    __syncthreads();
    // 2. exclusive scan of the tile histogram (P <= 1024 bins, 4 per thread at most)
    constexpr int kBinsPerThread = (1 << kMaxPartitionBits) / kPartThreads;
    unsigned v[kBinsPerThread], acc = 0;
#pragma unroll
    for (int q = 0; q < kBinsPerThread; ++q) {
      const int p = tid * kBinsPerThread + q;
      v[q] = p < P ? tcnt[p] : 0;
      acc += v[q];
    }
    unsigned incl = acc;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const unsigned o = __shfl_up_sync(kFullMask, incl, dd);
      if (lane >= dd) incl += o;
    }
    if (lane == 31) s_wsum[wid] = incl;
    __syncthreads();
    unsigned wbase = 0;
    for (int w = 0; w < wid; ++w) wbase += s_wsum[w];
    unsigned run = wbase + incl - acc;
#pragma unroll
    for (int q = 0; q < kBinsPerThread; ++q) {
      const int p = tid * kBinsPerThread + q;
      if (p < P) toff[p] = run;
      run += v[q];
    }
    unsigned tile_valid = 0;
    for (int w = 0; w < kPartThreads / 32; ++w) tile_valid += s_wsum[w];
    __syncthreads();
    // 3. counting-sort the tile into shared memory
#pragma unroll
    for (int j = 0; j < kTileRowsPerThread; ++j) {
      if (pr[j] < 0) continue;
      const int64_t i = t0 + j * kPartThreads + tid;
      const unsigned slot = toff[pr[j]] + rank[j];
      skey[slot] = kk[j];
      srid[slot] = (int32_t)i;
      spart[slot] = (uint16_t)pr[j];
      snat[slot] = (uint16_t)(j * kPartThreads + tid);
    }
    __syncthreads();
    // 4. write the partition runs: consecutive slots of one partition go to consecutive positions
    for (unsigned slot = tid; slot < tile_valid; slot += kPartThreads) {
      const int p = spart[slot];
      const int64_t pos = (int64_t)cur[p] + (slot - toff[p]);
      okeys[pos] = skey[slot];
      *reinterpret_cast<int32_t*>(reinterpret_cast<char*>(d.rid) + pos * (d.stride ? d.stride : 4)) = srid[slot];
      const int nat = snat[slot];
      for (int c = 0; c < s.n_pay; ++c) {
        const int w = s.pay[c].width;
        store_elem(static_cast<char*>(d.pay[c]) + pos * (d.stride ? d.stride : w), 0, w,
                   load_elem_smem(sm + m.pay[c], nat, w));
        if (d.valid8[c]) d.valid8[c][pos * (d.stride ? d.stride : 1)] = sm[m.val[c] + nat];
      }
    }
    __syncthreads();
    for (int p = tid; p < P; p += kPartThreads) cur[p] += tcnt[p];
    __syncthreads();
  }
}

static int part_grid(int device) { return sm_count(device) * 4; }

size_t partition_scratch_bytes(int pbits, int device) {
  const size_t PG = ((size_t)1 << pbits) * part_grid(device);
  return ((PG * 4 + 255) & ~(size_t)255) + (((PG + 1) * 8 + 255) & ~(size_t)255) + kScanBlocks * 8 + 256;
}

// Partition `src` into `dst` (arrays of src.n entries each). `scratch` must hold
// partition_scratch_bytes(pbits). On return (stream-ordered), *d_total_out points at the device
// int64 count of rows written and *d_part_off at the partition-major offsets (p * G entries).
sj_status radix_partition(const PartSrc& src, int key_type, int pbits, const PartDst& dst, void* scratch,
                          int device, cudaStream_t s, const int64_t** d_total_out, const int64_t** d_offs_out,
                          int* grid_out) {
  if (pbits < 0 || pbits > kMaxPartBits) return set_error(SJ_ERR_INVALID, "partition bits out of range");
  const int G = part_grid(device);
  const int P = 1 << pbits;
  const size_t PG = (size_t)P * G;
  char* base = static_cast<char*>(scratch);
  int32_t* hist = reinterpret_cast<int32_t*>(base);
  int64_t* offs = reinterpret_cast<int64_t*>(base + ((PG * 4 + 255) & ~(size_t)255));
  int64_t* tmp = reinterpret_cast<int64_t*>(base + ((PG * 4 + 255) & ~(size_t)255) + (((PG + 1) * 8 + 255) & ~(size_t)255));
  // chunks start on 4-row boundaries so the histogram can use 16-byte key loads
  const int64_t chunk = std::max<int64_t>(4, ((src.n + G - 1) / G + 3) / 4 * 4);
  const bool vec = ((uintptr_t)src.keys & 15u) == 0;
  {
    KernelTimer timer("partition_hist", s);
    if (key_type == SJ_INT32)
      part_hist_kernel<int32_t><<<G, kPartThreads, P * sizeof(int32_t), s>>>(src, pbits, chunk, vec, hist);
    else
      part_hist_kernel<int64_t><<<G, kPartThreads, P * sizeof(int32_t), s>>>(src, pbits, chunk, vec, hist);
  }
  {
    KernelTimer timer("partition_scan", s);
    device_exclusive_scan<int32_t, int64_t>(hist, offs, nullptr, (int64_t)PG, tmp, s);
  }
  const ScatterSmem m = scatter_smem(pbits, key_type == SJ_INT32 ? 4 : 8, src);
  if (key_type == SJ_INT32) {
    SJ_CUDA_TRY(cudaFuncSetAttribute(part_scatter_kernel<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)m.total));
    KernelTimer timer("partition_scatter", s);
    part_scatter_kernel<int32_t><<<G, kPartThreads, m.total, s>>>(src, pbits, chunk, offs, dst, m);
  } else {
    SJ_CUDA_TRY(cudaFuncSetAttribute(part_scatter_kernel<int64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)m.total));
    KernelTimer timer("partition_scatter", s);
    part_scatter_kernel<int64_t><<<G, kPartThreads, m.total, s>>>(src, pbits, chunk, offs, dst, m);
  }
  SJ_CUDA_TRY(cudaGetLastError());
  *d_total_out = offs + PG;
  *d_offs_out = offs;
  *grid_out = G;
  return SJ_OK;
}

}  // namespace sj
