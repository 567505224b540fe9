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
#include <type_traits>

#include "sj_partition.cuh"
#include "sj_scan.cuh"

namespace sj {

constexpr int kPartThreads = 256;
constexpr int kMaxPartBits = kMaxPartitionBits;

__device__ __forceinline__ int partition_of(uint64_t kb, int pbits) {
  return pbits ? (int)(mix64(kb) >> (64 - pbits)) : 0;
}

template <typename K>
__device__ __forceinline__ void hist_load4(const K* keys, int64_t i0, int64_t hi, bool vec, K (&k)[4]) {
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
}

// Histogram pass: each thread loads 4 groups of 4 consecutive keys (16-byte loads) per step, all
// before counting them, so 8 (int64) or 4 (int32) vector loads per thread are in flight.
template <typename K>
__global__ void __launch_bounds__(kPartThreads) part_hist_kernel(PartSrc s, int pbits, int64_t chunk, bool vec,
                                                                 int32_t* hist) {
  extern __shared__ int32_t h[];
  constexpr int kGroups = 4;
  const int P = 1 << pbits;
  for (int p = threadIdx.x; p < P; p += blockDim.x) h[p] = 0;
  __syncthreads();
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < s.n ? lo + chunk : s.n;
  const K* keys = static_cast<const K*>(s.keys);
  const int64_t step = (int64_t)blockDim.x * 4;
  for (int64_t base = lo; base < hi; base += step * kGroups) {
    K k[kGroups][4];
#pragma unroll
    for (int g = 0; g < kGroups; ++g) hist_load4<K>(keys, base + g * step + (int64_t)threadIdx.x * 4, hi, vec, k[g]);
#pragma unroll
    for (int g = 0; g < kGroups; ++g) {
      const int64_t i0 = base + g * step + (int64_t)threadIdx.x * 4;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (i0 + j < hi && bit_valid(s.kvalid, s.kvoff, i0 + j))
          atomicAdd(&h[partition_of(key_u64<K>(k[g][j]), pbits)], 1);
    }
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

// Scatter pass for plain outputs (no row store) with at most 2 payload columns of 4 or 8 bytes
// without NULLs — the probe side's shape. Each thread holds its 8 rows of a tile (key, payloads)
// in registers, so all 8-24 loads are in flight at once; the tile is ranked and counting-sorted in
// shared memory as above (payloads placed directly at their sorted slot), and the loads of the
// NEXT tile are issued before this tile's runs are written out, so DRAM reads overlap the writes.
constexpr int kFastMaxPay = 2;

struct FastSmem {
  size_t cur, tcnt, toff, key, rid, dst, pay[kFastMaxPay], total;
};

static FastSmem fast_smem(int pbits, int kw, int n_pay) {
  const size_t P = (size_t)1 << pbits;
  FastSmem m{};
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
  m.dst = take((size_t)kTile * 4);
  for (int c = 0; c < n_pay; ++c) m.pay[c] = take((size_t)kTile * 8);
  m.total = o;
  return m;
}

bool partition_plain_shape(const PartSrc& s, const PartDst& d);
static bool fast_scatter_ok(const PartSrc& s, const PartDst& d) { return partition_plain_shape(s, d); }
bool partition_plain_shape(const PartSrc& s, const PartDst& d) {
  if (d.stride != 0 || s.n_pay > kFastMaxPay) return false;
  for (int c = 0; c < s.n_pay; ++c)
    if (s.pay[c].valid || s.pay[c].valid8 || (s.pay[c].width != 4 && s.pay[c].width != 8) ||
        s.pay[c].stride != s.pay[c].width || d.valid8[c])
      return false;
  return true;
}

// Row of a tile held by thread t as its j-th row: threads hold consecutive row pairs, so a pair is
// one 16-byte (int64) or 8-byte (int32) vector load when the columns are aligned for it.
__device__ __forceinline__ int64_t fast_row(int64_t t0, int j, int t) {
  return t0 + (int64_t)(j >> 1) * 2 * kPartThreads + 2 * t + (j & 1);
}

template <typename T, typename U>
__device__ __forceinline__ void ld_pair_cs(const T* p, U& a, U& b) {
  if constexpr (sizeof(T) == 8) {
    const ulonglong2 x = __ldcs(reinterpret_cast<const ulonglong2*>(p));
    a = (U)x.x;
    b = (U)x.y;
  } else {
    const uint2 x = __ldcs(reinterpret_cast<const uint2*>(p));
    a = (U)x.x;
    b = (U)x.y;
  }
}

// VEC: the key and payload columns start on a multiple of twice their element width (t0 is even)
template <typename K, int NP, bool VEC>
__device__ __forceinline__ void fast_load_tile(const PartSrc& s, int64_t t0, int64_t hi,
                                               K (&kk)[kTileRowsPerThread],
                                               uint64_t (&pv)[kFastMaxPay][kTileRowsPerThread], uint32_t& live) {
  const K* keys = static_cast<const K*>(s.keys);
  live = 0;
#pragma unroll
  for (int j = 0; j < kTileRowsPerThread; j += 2) {
    const int64_t i = fast_row(t0, j, threadIdx.x);
    kk[j] = kk[j + 1] = 0;
#pragma unroll
    for (int c = 0; c < kFastMaxPay; ++c) pv[c][j] = pv[c][j + 1] = 0;
    if (VEC && i + 1 < hi) {
      ld_pair_cs(keys + i, kk[j], kk[j + 1]);
#pragma unroll
      for (int c = 0; c < NP; ++c) {
        if (s.pay[c].width == 8) {
          ld_pair_cs(static_cast<const unsigned long long*>(s.pay[c].data) + i, pv[c][j], pv[c][j + 1]);
        } else {
          unsigned a, b;
          ld_pair_cs(static_cast<const unsigned int*>(s.pay[c].data) + i, a, b);
          pv[c][j] = a;
          pv[c][j + 1] = b;
        }
      }
    } else {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (i + h >= hi) continue;
        kk[j + h] = __ldcs(keys + i + h);
#pragma unroll
        for (int c = 0; c < NP; ++c)
          pv[c][j + h] = s.pay[c].width == 8
                             ? __ldcs(static_cast<const unsigned long long*>(s.pay[c].data) + i + h)
                             : (uint64_t)__ldcs(static_cast<const unsigned int*>(s.pay[c].data) + i + h);
      }
    }
    if (i < hi && bit_valid(s.kvalid, s.kvoff, i)) live |= 1u << j;
    if (i + 1 < hi && bit_valid(s.kvalid, s.kvoff, i + 1)) live |= 1u << (j + 1);
  }
}

// LOCAL: no global offsets — every tile is written back in place, sorted by partition, and its
// per-partition runs go to run_off / run_cnt[tile * P + p] (the probe walks them partition-major).
// VEC: the source columns take pair loads (fast_load_tile) and, when LOCAL, the destination
// columns pair stores. 16-byte loads and stores took the tile-local scatter of 64M int64 rows with
// one 8-byte payload from 0.492 to 0.482 ms (same box, 30 steps, two runs each).
template <typename K, int NP, bool LOCAL = false, bool VEC = false>
__global__ void __launch_bounds__(kPartThreads, 3) part_scatter_fast_kernel(PartSrc s, int pbits, int64_t chunk,
                                                                         const int64_t* __restrict__ off, PartDst d,
                                                                         FastSmem m, int32_t* run_off = nullptr,
                                                                         int32_t* run_cnt = nullptr) {
  extern __shared__ __align__(16) unsigned char sm[];
  unsigned long long* cur = reinterpret_cast<unsigned long long*>(sm + m.cur);
  unsigned int* tcnt = reinterpret_cast<unsigned int*>(sm + m.tcnt);
  unsigned int* toff = reinterpret_cast<unsigned int*>(sm + m.toff);
  K* skey = reinterpret_cast<K*>(sm + m.key);
  int32_t* srid = reinterpret_cast<int32_t*>(sm + m.rid);
  uint32_t* sdst = reinterpret_cast<uint32_t*>(sm + m.dst);
  __shared__ unsigned int s_wsum[kPartThreads / 32];
  const int P = 1 << pbits;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (!LOCAL)
    for (int p = tid; p < P; p += kPartThreads) cur[p] = (unsigned long long)off[(int64_t)p * gridDim.x + blockIdx.x];
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < s.n ? lo + chunk : s.n;
  K* okeys = static_cast<K*>(d.keys);
  K kk[kTileRowsPerThread];
  uint64_t pv[kFastMaxPay][kTileRowsPerThread];
  uint32_t live = 0;
  if (lo < hi) fast_load_tile<K, NP, VEC>(s, lo, hi, kk, pv, live);
  for (int64_t t0 = lo; t0 < hi; t0 += kTile) {
    for (int p = tid; p < P; p += kPartThreads) tcnt[p] = 0;
    __syncthreads();
    // 1. partition and rank within the tile's partition
    int pr[kTileRowsPerThread];
    unsigned rank[kTileRowsPerThread];
#pragma unroll
    for (int j = 0; j < kTileRowsPerThread; ++j) {
      pr[j] = (live >> j & 1u) ? partition_of(key_u64<K>(kk[j]), pbits) : -1;
      const unsigned peers = __match_any_sync(kFullMask, pr[j]);
      const int leader = __ffs(peers) - 1;
      unsigned base = 0;
      if (pr[j] >= 0 && lane == leader) base = atomicAdd(&tcnt[pr[j]], (unsigned)__popc(peers));
      base = __shfl_sync(kFullMask, base, leader);
      rank[j] = base + __popc(peers & ((1u << lane) - 1));
    }
    __syncthreads();
    // 2. exclusive scan of the tile histogram
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
    if (LOCAL) {  // after the barrier: toff[p] is written by thread p / kBinsPerThread
      const int64_t ti = t0 / kTile;
      for (int p = tid; p < P; p += kPartThreads) {
        run_off[ti * P + p] = (int32_t)(t0 + toff[p]);
        run_cnt[ti * P + p] = (int32_t)tcnt[p];
      }
    }
    // 3. counting-sort the tile into shared memory (payloads straight to their sorted slot, with
    //    each row's output position, so the write-out reads nothing per partition)
#pragma unroll
    for (int j = 0; j < kTileRowsPerThread; ++j) {
      if (pr[j] < 0) continue;
      const unsigned slot = toff[pr[j]] + rank[j];
      skey[slot] = kk[j];
      srid[slot] = (int32_t)fast_row(t0, j, tid);
      if (!LOCAL) sdst[slot] = (uint32_t)cur[pr[j]] + rank[j];  // LOCAL: the tile's own rows
#pragma unroll
      for (int c = 0; c < NP; ++c) reinterpret_cast<uint64_t*>(sm + m.pay[c])[slot] = pv[c][j];
    }
    __syncthreads();
    // 4. loads of the next tile go out before this tile's write-out
    if (t0 + kTile < hi) fast_load_tile<K, NP, VEC>(s, t0 + kTile, hi, kk, pv, live);
    if constexpr (LOCAL && VEC) {  // row pairs: t0 and the staging slots are even
      using K2 = std::conditional_t<sizeof(K) == 8, longlong2, int2>;
      for (unsigned slot = 2 * tid; slot < tile_valid; slot += 2 * kPartThreads) {
        const uint32_t pos = (uint32_t)t0 + slot;
        if (slot + 1 < tile_valid) {
          *reinterpret_cast<K2*>(okeys + pos) = *reinterpret_cast<const K2*>(skey + slot);
          *reinterpret_cast<int2*>(d.rid + pos) = *reinterpret_cast<const int2*>(srid + slot);
#pragma unroll
          for (int c = 0; c < NP; ++c) {
            const ulonglong2 x = reinterpret_cast<const ulonglong2*>(sm + m.pay[c])[slot >> 1];
            if (s.pay[c].width == 8) *reinterpret_cast<ulonglong2*>(static_cast<unsigned long long*>(d.pay[c]) + pos) = x;
            else *reinterpret_cast<uint2*>(static_cast<unsigned int*>(d.pay[c]) + pos) = make_uint2((unsigned)x.x, (unsigned)x.y);
          }
        } else {
          okeys[pos] = skey[slot];
          d.rid[pos] = srid[slot];
#pragma unroll
          for (int c = 0; c < NP; ++c) {
            const uint64_t x = reinterpret_cast<const uint64_t*>(sm + m.pay[c])[slot];
            if (s.pay[c].width == 8) static_cast<unsigned long long*>(d.pay[c])[pos] = x;
            else static_cast<unsigned int*>(d.pay[c])[pos] = (unsigned int)x;
          }
        }
      }
    } else {
      for (unsigned slot = tid; slot < tile_valid; slot += kPartThreads) {
        const uint32_t pos = LOCAL ? (uint32_t)t0 + slot : sdst[slot];
        okeys[pos] = skey[slot];
        d.rid[pos] = srid[slot];
#pragma unroll
        for (int c = 0; c < NP; ++c) {
          const uint64_t x = reinterpret_cast<const uint64_t*>(sm + m.pay[c])[slot];
          if (s.pay[c].width == 8) static_cast<unsigned long long*>(d.pay[c])[pos] = x;
          else static_cast<unsigned int*>(d.pay[c])[pos] = (unsigned int)x;
        }
      }
    }
    __syncthreads();
    if (!LOCAL) {
      for (int p = tid; p < P; p += kPartThreads) cur[p] += tcnt[p];
      __syncthreads();
    }
  }
}

// The source key and payload columns start on a multiple of twice their element width, so the
// row pairs of fast_load_tile are aligned vector loads (chunks and tiles start on even rows).
static bool pair_aligned_src(const PartSrc& src, int kw) {
  bool ok = ((uintptr_t)src.keys % (2 * kw)) == 0;
  for (int c = 0; c < src.n_pay; ++c) ok = ok && ((uintptr_t)src.pay[c].data % (2 * src.pay[c].width)) == 0;
  return ok;
}

template <typename K>
static sj_status launch_fast_scatter(const PartSrc& src, int pbits, int64_t chunk, const int64_t* offs,
                                     const PartDst& dst, int G, cudaStream_t s) {
  const FastSmem m = fast_smem(pbits, sizeof(K), src.n_pay);
  auto go = [&](auto kernel) -> sj_status {
    SJ_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.total));
    KernelTimer timer("partition_scatter", s);
    kernel<<<G, kPartThreads, m.total, s>>>(src, pbits, chunk, offs, dst, m, nullptr, nullptr);
    return SJ_OK;
  };
  if (pair_aligned_src(src, sizeof(K))) {
    if (src.n_pay == 0) return go(part_scatter_fast_kernel<K, 0, false, true>);
    if (src.n_pay == 1) return go(part_scatter_fast_kernel<K, 1, false, true>);
    return go(part_scatter_fast_kernel<K, 2, false, true>);
  }
  if (src.n_pay == 0) return go(part_scatter_fast_kernel<K, 0>);
  if (src.n_pay == 1) return go(part_scatter_fast_kernel<K, 1>);
  return go(part_scatter_fast_kernel<K, 2>);
}

// Upper bound of the partition grid (scratch sizing); the grid used is never larger.
static int part_grid(int device) { return sm_count(device) * 4; }

static int scatter_per_sm(const PartSrc& src, int key_type, int pbits, bool fast) {
  int r = 0;
  if (fast) {
    const FastSmem m = fast_smem(pbits, key_type == SJ_INT32 ? 4 : 8, src.n_pay);
    const void* k = nullptr;
    if (key_type == SJ_INT32)
      k = src.n_pay == 0 ? (const void*)part_scatter_fast_kernel<int32_t, 0>
          : src.n_pay == 1 ? (const void*)part_scatter_fast_kernel<int32_t, 1>
                           : (const void*)part_scatter_fast_kernel<int32_t, 2>;
    else
      k = src.n_pay == 0 ? (const void*)part_scatter_fast_kernel<int64_t, 0>
          : src.n_pay == 1 ? (const void*)part_scatter_fast_kernel<int64_t, 1>
                           : (const void*)part_scatter_fast_kernel<int64_t, 2>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.total);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k, kPartThreads, m.total);
  } else {
    const ScatterSmem m = scatter_smem(pbits, key_type == SJ_INT32 ? 4 : 8, src);
    const void* k = key_type == SJ_INT32 ? (const void*)part_scatter_kernel<int32_t>
                                         : (const void*)part_scatter_kernel<int64_t>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.total);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k, kPartThreads, m.total);
  }
  cudaGetLastError();
  return std::max(1, std::min(4, r));
}

// Tile-local partition: one pass, no histogram. Returns the number of tiles (run table rows).
sj_status local_partition(const PartSrc& src, int key_type, int pbits, const PartDst& dst, int32_t* run_off,
                          int32_t* run_cnt, int device, cudaStream_t s) {
  if (!fast_scatter_ok(src, dst)) return set_error(SJ_ERR_INVALID, "tile-local partition needs the plain shape");
  const int P = 1 << pbits;
  const int64_t tiles = (src.n + kTile - 1) / kTile;
  const int per_sm = scatter_per_sm(src, key_type, pbits, true);
  const int64_t G = std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count(device) * per_sm));
  const int64_t chunk = (tiles + G - 1) / G * kTile;  // whole tiles per CTA
  const int grid = (int)((src.n + chunk - 1) / chunk);
  if (src.n == 0) return SJ_OK;
  const int kw = key_type == SJ_INT32 ? 4 : 8;
  // pair loads and stores when the source columns and the partitioned copies are aligned for them
  bool vec = pair_aligned_src(src, kw) && ((uintptr_t)dst.keys % (2 * kw)) == 0 && ((uintptr_t)dst.rid % 8) == 0;
  for (int c = 0; c < src.n_pay; ++c) vec = vec && ((uintptr_t)dst.pay[c] % (2 * src.pay[c].width)) == 0;
  auto go = [&](auto kernel) -> sj_status {
    const FastSmem m = fast_smem(pbits, kw, src.n_pay);
    SJ_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.total));
    KernelTimer timer("partition_scatter", s);
    kernel<<<grid, kPartThreads, m.total, s>>>(src, pbits, chunk, nullptr, dst, m, run_off, run_cnt);
    return SJ_OK;
  };
  (void)P;
  auto pick = [&](auto k, auto v) -> sj_status {
    using K = decltype(k);
    constexpr bool V = decltype(v)::value;
    return src.n_pay == 0 ? go(part_scatter_fast_kernel<K, 0, true, V>)
         : src.n_pay == 1 ? go(part_scatter_fast_kernel<K, 1, true, V>)
                          : go(part_scatter_fast_kernel<K, 2, true, V>);
  };
  sj_status st;
  if (key_type == SJ_INT32)
    st = vec ? pick(int32_t{}, std::true_type{}) : pick(int32_t{}, std::false_type{});
  else
    st = vec ? pick(int64_t{}, std::true_type{}) : pick(int64_t{}, std::false_type{});
  SJ_TRY(st);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

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
  // Every CTA owns one chunk (no grid-stride loop), so the grid must be resident in one wave:
  // G = SMs x (the scatter kernel's resident CTAs per SM, at most 4).
  const bool fast = fast_scatter_ok(src, dst);
  const int G = sm_count(device) * scatter_per_sm(src, key_type, pbits, fast);
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
  if (fast) {
    SJ_TRY(key_type == SJ_INT32 ? launch_fast_scatter<int32_t>(src, pbits, chunk, offs, dst, G, s)
                                : launch_fast_scatter<int64_t>(src, pbits, chunk, offs, dst, G, s));
    SJ_CUDA_TRY(cudaGetLastError());
    *d_total_out = offs + PG;
    *d_offs_out = offs;
    *grid_out = G;
    return SJ_OK;
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
