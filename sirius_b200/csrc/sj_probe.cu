// INNER probe fused with the payload gather for the sm_100a equi-join. Replaces
// hash_join::inner_join / distinct_hash_join::inner_join / cudf::inner_join
// (src/op/sirius_physical_hash_join.cpp:1671, :1688, :1872) and the two cudf::gather calls of
// gather_join_output (:1299-1359): the output row (probe rid, build rid, probe payloads, build
// payloads) is written once, by the kernel that found the match.
//
// DISTINCT tables (one slot per build row, unique keys) take a single pass:
//   - every thread owns KPT = 4 consecutive probe rows and reads their keys with 128-bit
//     streaming loads (ld.global.cs: the probe stream must not evict the table from L2);
//   - keys outside [key_min, key_max] or NULL are rejected without touching the table;
//   - the thread issues the KPT bucket loads (32 B = one sector each) back to back, so a warp
//     keeps 128 independent sector reads in flight;
//   - matches are compacted warp-aggregated: __shfl_up prefix of the per-lane hit counts and one
//     atomicAdd per warp reserves the warp's output range;
//   - payloads are gathered straight into the reserved positions (build columns by row id).
// GROUPED tables (duplicated keys, or NULLs equal) take count -> scan -> expand:
//   - pass A finds each probe row's group and appends (probe row, group start, group size) to a
//     compacted match list (warp-aggregated), summing the output size M;
//   - an exclusive scan turns group sizes into output offsets;
//   - the expand kernel gives every CTA a contiguous range of output tiles and each thread one
//     output position per step (load-balanced search over the offsets staged in shared memory),
//     so a probe key matching 10^6 build rows is spread over the whole GPU instead of one thread.
#include <algorithm>

#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_partition.cuh"
#include "sj_probe_direct.h"
#include "sj_scan.cuh"

namespace sj {

TableDev table_dev(const sj_table* t);

constexpr int KPT = 4;  // probe rows per thread per tile

template <typename K>
__device__ __forceinline__ void load_keys(const K* __restrict__ keys, int64_t row0, int64_t n, bool vec,
                                          K (&k)[KPT]) {
  if (vec && row0 + KPT <= n) {
    if (sizeof(K) == 4) {
      const int4 x = __ldcs(reinterpret_cast<const int4*>(keys + row0));
      k[0] = (K)x.x;
      k[1] = (K)x.y;
      k[2] = (K)x.z;
      k[3] = (K)x.w;
    } else {
      const longlong2* p = reinterpret_cast<const longlong2*>(keys + row0);
      const longlong2 x = __ldcs(p), y = __ldcs(p + 1);
      k[0] = (K)x.x;
      k[1] = (K)x.y;
      k[2] = (K)y.x;
      k[3] = (K)y.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < KPT; ++j) k[j] = row0 + j < n ? __ldcs(keys + row0 + j) : (K)0;
  }
}

__device__ __forceinline__ uint64_t load_elem_cs(const void* base, int64_t i, int w) {
  switch (w) {
    case 8: return __ldcs(reinterpret_cast<const unsigned long long*>(base) + i);
    case 4: return __ldcs(reinterpret_cast<const unsigned int*>(base) + i);
    case 2: return __ldcs(reinterpret_cast<const unsigned short*>(base) + i);
    default: return __ldg(reinterpret_cast<const unsigned char*>(base) + i);
  }
}

// Rows of a probe tile that can match: in range, valid. Bit j = row0 + j.
template <typename K>
__device__ __forceinline__ uint32_t live_rows(const TableDev& t, const K (&k)[KPT], int64_t row0, int64_t n,
                                              const uint32_t* kv, int64_t kvoff) {
  uint32_t act = 0;
#pragma unroll
  for (int j = 0; j < KPT; ++j) {
    const int64_t r = row0 + j;
    if (r < n && bit_valid(kv, kvoff, r) && in_range(t, k[j])) act |= 1u << j;
  }
  return act;
}

// ------------------------------------------------------------------------------------------------
// Warp write-out. A warp stages its matches (probe row, build row id) in shared memory in
// compacted order, reserves one output range with a single atomicAdd, and then writes every
// output column with consecutive lanes on consecutive positions: full 32-byte sectors reach L2
// instead of lane-strided partial ones, and the probe payload is read in near-sequential order.
// ------------------------------------------------------------------------------------------------
constexpr int kProbeThreads = 256;
constexpr int kWarpsPerCta = kProbeThreads / 32;
constexpr int kStage = 32 * KPT;  // matches one warp can stage per tile

template <bool STREAM>
__device__ __forceinline__ void emit_column(const PayloadIn& in, const PayloadOut& o, const int32_t* s_idx,
                                            uint32_t tot, int64_t base, int64_t cap) {
  const int lane = threadIdx.x & 31;
  uint64_t v[KPT];
#pragma unroll
  for (int u = 0; u < KPT; ++u) {
    const uint32_t i = lane + 32u * u;
    v[u] = 0;
    if (i < tot) v[u] = STREAM && in.stride == in.width ? load_elem_cs(in.data, s_idx[i], in.width) : pl_load(in, s_idx[i]);
  }
#pragma unroll
  for (int u = 0; u < KPT; ++u) {
    const uint32_t i = lane + 32u * u;
    const int64_t p = base + i;
    const bool live = i < tot && p < cap;
    if (live) store_elem(o.data, p, in.width, v[u]);
    if (has_validity(in)) {
      const unsigned bits = __ballot_sync(kFullMask, live && payload_valid(in, s_idx[i]));
      if (lane == 0 && bits) {
        const int64_t p0 = base + 32u * u;
        const int sh = (int)(p0 & 31);
        atomicOr(o.valid + (p0 >> 5), bits << sh);
        if (sh && (bits >> (32 - sh))) atomicOr(o.valid + (p0 >> 5) + 1, bits >> (32 - sh));
      }
    }
  }
}

// s_row: probe array indices (row ids unless the probe was partitioned: prid_map).
// s_rid: table positions (build row ids unless the table maps them: brid_map); rewritten in
// place to build row ids after the position-ordered attached payloads have been gathered.
// Row-store write-out: one record load per match gives the build row id and all attached fields.
__device__ __forceinline__ void write_records(const Record (&r)[KPT / 2], int half, uint32_t tot, int64_t base,
                                              const GatherArgs& g) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int h = 0; h < KPT / 2; ++h) {
    const uint32_t i = lane + 32u * (half * (KPT / 2) + h);
    const int64_t p = base + i;
    const bool live = i < tot && p < g.capacity;
    if (live && g.out_brid) g.out_brid[p] = (int32_t)r[h].w[0];
    for (int c = 0; c < g.n_bin; ++c) {
      const int w = g.bin[c].width;
      if (live) store_elem(g.bout[c].data, p, w, record_field(r[h], g.rec_off[c], w));
      if (g.rec_voff[c] >= 0) {
        const unsigned bits = __ballot_sync(kFullMask, live && record_field(r[h], g.rec_voff[c], 1) != 0);
        if (lane == 0 && bits) {
          const int64_t p0 = base + 32u * (half * (KPT / 2) + h);
          const int sh = (int)(p0 & 31);
          atomicOr(g.bout[c].valid + (p0 >> 5), bits << sh);
          if (sh && (bits >> (32 - sh))) atomicOr(g.bout[c].valid + (p0 >> 5) + 1, bits >> (32 - sh));
        }
      }
    }
  }
}

__device__ __forceinline__ void load_records(Record (&r)[KPT / 2], int half, const int32_t* s_rid, uint32_t tot,
                                             const GatherArgs& g) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int h = 0; h < KPT / 2; ++h) {
    const uint32_t i = lane + 32u * (half * (KPT / 2) + h);
    if (i < tot)
      r[h] = load_record(static_cast<const char*>(g.rec) + (int64_t)s_rid[i] * g.rec_stride, g.rec_stride);
  }
}

// s_row: probe array indices (row ids unless the probe was partitioned: prid_map).
// s_rid: table positions (build row ids unless the table maps them: brid_map); rewritten in
// place to build row ids after the position-ordered attached payloads have been gathered.
// base: the warp's first output position; when `deferred` it is lane 0's still-pending atomicAdd
// result, broadcast only after this warp's gather loads are in flight.
__device__ __forceinline__ void warp_write_out(const int32_t* s_row, int32_t* s_rid, uint32_t tot,
                                               unsigned long long base_in, bool deferred, const GatherArgs& g) {
  const int lane = threadIdx.x & 31;
  if (g.rec) {
    const int64_t base = (int64_t)(deferred ? __shfl_sync(kFullMask, base_in, 0) : base_in);
    if (g.out_prid) {
      for (uint32_t i = lane; i < tot; i += 32) {
        const int64_t p = base + i;
        if (p < g.capacity) g.out_prid[p] = g.prid_map ? __ldg(g.prid_map + s_row[i]) : s_row[i];
      }
    }
    Record r[KPT / 2];
    load_records(r, 0, s_rid, tot, g);
    write_records(r, 0, tot, base, g);
    load_records(r, 1, s_rid, tot, g);
    write_records(r, 1, tot, base, g);
    for (int c = 0; c < g.n_pin; ++c) emit_column<true>(g.pin[c], g.pout[c], s_row, tot, base, g.capacity);
    return;
  }
  const int64_t base = (int64_t)(deferred ? __shfl_sync(kFullMask, base_in, 0) : base_in);
  if (g.out_prid) {
    for (uint32_t i = lane; i < tot; i += 32) {
      const int64_t p = base + i;
      if (p < g.capacity) g.out_prid[p] = g.prid_map ? __ldg(g.prid_map + s_row[i]) : s_row[i];
    }
  }
  if (g.bin_by_pos)
    for (int c = 0; c < g.n_bin; ++c) emit_column<false>(g.bin[c], g.bout[c], s_rid, tot, base, g.capacity);
  if (g.brid_map) {
    for (uint32_t i = lane; i < tot; i += 32) s_rid[i] = brid_of(g, s_rid[i]);
    __syncwarp();
  }
  if (g.out_brid) {
    for (uint32_t i = lane; i < tot; i += 32) {
      const int64_t p = base + i;
      if (p < g.capacity) g.out_brid[p] = s_rid[i];
    }
  }
  if (!g.bin_by_pos)
    for (int c = 0; c < g.n_bin; ++c) emit_column<false>(g.bin[c], g.bout[c], s_rid, tot, base, g.capacity);
  for (int c = 0; c < g.n_pin; ++c) emit_column<true>(g.pin[c], g.pout[c], s_row, tot, base, g.capacity);
}

// ------------------------------------------------------------------------------------------------
// DISTINCT: probe + gather in one pass
// ------------------------------------------------------------------------------------------------
// CTA_AGG: the CTA sums its warps' match counts and reserves the whole tile's output range with
// one atomicAdd (instead of one per warp), which matters when a probe of tens of millions of rows
// would otherwise queue ~10^5-10^6 atomics on the single output counter.
template <typename K, bool WIDE, bool VEC, bool COUNT_ONLY, bool CTA_AGG>
__global__ void __launch_bounds__(kProbeThreads, 4) probe_distinct_kernel(TableDev t, const K* __restrict__ keys,
                                                                           const uint32_t* __restrict__ kv,
                                                                           int64_t kvoff, int64_t n_host,
                                                                           const int64_t* d_n, GatherArgs g) {
  using Ops = SlotOps<WIDE>;
  __shared__ int32_t s_row[kWarpsPerCta][kStage];
  __shared__ int32_t s_rid[kWarpsPerCta][kStage];
  __shared__ unsigned s_wtot[kWarpsPerCta], s_wbase[kWarpsPerCta];
  __shared__ unsigned long long s_cta_base;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t n = d_n ? *d_n : n_host;
  const int64_t per_cta = (int64_t)blockDim.x * KPT;
  const int64_t tiles = (n + per_cta - 1) / per_cta;
  unsigned long long counted = 0;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row0 = tile * per_cta + (int64_t)threadIdx.x * KPT;
    K k[KPT];
    load_keys<K>(keys, row0, n, VEC, k);
    uint32_t act = live_rows<K>(t, k, row0, n, kv, kvoff);
    uint32_t b[KPT];
    uint64_t ks[KPT];
    const uint64_t kmask = ~((1ull << t.rbits) - 1);
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      const uint64_t kb = key_u64<K>(k[j]);
      b[j] = home_bucket(t, kb);
      ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
    }
    int32_t rid[KPT] = {0, 0, 0, 0};
    uint32_t hit = 0;
    for (uint32_t step = 0; act && step <= t.segmask; ++step) {
      Bucket bk[KPT];
#pragma unroll
      for (int j = 0; j < KPT; ++j)
        if (act >> j & 1u) bk[j] = load_bucket<true>(t.slots, b[j]);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        if (!(act >> j & 1u)) continue;
        bool done = false;
#pragma unroll
        for (int q = 0; q < Ops::kSlots; ++q) {
          if (!done && Ops::match_s(bk[j], q, ks[j], kmask)) {
            rid[j] = Ops::rid(bk[j], q, t.rbits);
            hit |= 1u << j;
            done = true;
          }
          done |= Ops::empty(bk[j], q);
        }
        if (done) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    const uint32_t cnt = __popc(hit);
    if (COUNT_ONLY) {
      counted += cnt;
      continue;
    }
    const uint32_t incl = warp_inclusive_sum(cnt);
    const uint32_t tot = __shfl_sync(kFullMask, incl, 31);
    if (!CTA_AGG && tot == 0) continue;
    uint32_t sp = incl - cnt;
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      if (hit >> j & 1u) {
        s_row[warp][sp] = (int32_t)(row0 + j);
        s_rid[warp][sp] = rid[j];
        ++sp;
      }
    }
    unsigned long long base = 0;
    bool deferred = false;
    if (CTA_AGG) {
      if (lane == 0) s_wtot[warp] = tot;
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned run = 0;
#pragma unroll
        for (int w = 0; w < kWarpsPerCta; ++w) {
          s_wbase[w] = run;
          run += s_wtot[w];
        }
        s_cta_base = run ? atomicAdd(g.d_count, (unsigned long long)run) : 0ull;
      }
      __syncthreads();
      base = s_cta_base + s_wbase[warp];
    } else {
      if (lane == 0) base = atomicAdd(g.d_count, (unsigned long long)tot);
      deferred = true;  // broadcast from lane 0 inside the write-out
      __syncwarp();
    }
    if (tot) warp_write_out(s_row[warp], s_rid[warp], tot, base, deferred, g);
    __syncwarp();
  }
  if (COUNT_ONLY) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) counted += __shfl_down_sync(kFullMask, counted, d);
    if (lane == 0 && counted) atomicAdd(g.d_count, counted);
  }
}

// ------------------------------------------------------------------------------------------------
// GROUPED pass A: find each probe row's group; compact (row, start, size); sum the output size.
// A warp owns 32 * kMatchR consecutive probe rows per tile, lane l rows base + 32 j + l, so every
// key load is one coalesced warp access; a bucket is tested as a whole (one slot per distinct
// key); the rows with matches of row group j are ranked with one ballot and written at
// base + (earlier groups) + popc(ballot_j & lanes below), one atomicAdd per warp tile.
// ------------------------------------------------------------------------------------------------
constexpr int kMatchR = 4;

template <typename K, bool WIDE, bool COMPACT>
__global__ void __launch_bounds__(kProbeThreads, 4) grouped_match_kernel(TableDev t, const K* __restrict__ keys,
                                                                          const uint32_t* __restrict__ kv,
                                                                          int64_t kvoff, int64_t n, int32_t* m_row,
                                                                          int32_t* m_start, int32_t* m_cnt,
                                                                          unsigned long long* d_nent,
                                                                          unsigned long long* d_total) {
  using Ops = SlotOps<WIDE>;
  constexpr int R = kMatchR;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int64_t wtiles = (n + 32 * R - 1) / (32 * R);
  const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  unsigned long long total = 0;
  for (int64_t wt = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); wt < wtiles; wt += wstride) {
    const int64_t r0 = wt * 32 * R + lane;
    K k[R];
    uint32_t act = 0;
    int32_t slot[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t r = r0 + 32 * j;
      k[j] = r < n ? __ldcs(keys + r) : (K)0;
      slot[j] = -1;
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t r = r0 + 32 * j;
      if (r >= n) continue;
      if (!bit_valid(kv, kvoff, r)) {
        if (t.null_group >= 0) slot[j] = t.null_group;  // NULLs equal: the NULL group
      } else if (in_range(t, k[j])) {
        act |= 1u << j;
      }
    }
    uint32_t b[R];
    uint64_t ks[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint64_t kb = key_u64<K>(k[j]);
      b[j] = home_bucket(t, kb);
      ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
    }
    for (uint32_t step = 0; act && step <= t.segmask; ++step) {
      Bucket bk[R];
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (act >> j & 1u) bk[j] = load_bucket<true>(t.slots, b[j]);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (!(act >> j & 1u)) continue;
        int q;
        const bool m = Ops::match_slot(bk[j], ks[j], kmask, q);
        if (m) slot[j] = (int32_t)(b[j] * Ops::kSlots + q);
        if (m || Ops::open(bk[j])) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    int32_t start[R], cnt[R];
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      start[j] = cnt[j] = 0;
      if (slot[j] >= 0) {
        start[j] = __ldg(t.grp_off + slot[j]);
        cnt[j] = __ldg(t.grp_off + slot[j] + 1) - start[j];
        if (cnt[j] > 0) hit |= 1u << j;
        total += (unsigned long long)cnt[j];
      }
    }
    if (COMPACT) {
      unsigned bal[R];
      uint32_t tot = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        bal[j] = __ballot_sync(kFullMask, (hit >> j) & 1u);
        tot += __popc(bal[j]);
      }
      if (tot) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(d_nent, (unsigned long long)tot);
        base = __shfl_sync(kFullMask, base, 0);
#pragma unroll
        for (int j = 0; j < R; ++j) {
          if (hit >> j & 1u) {
            const unsigned long long p = base + __popc(bal[j] & below);
            m_row[p] = (int32_t)(r0 + 32 * j);
            m_start[p] = start[j];
            m_cnt[p] = cnt[j];
          }
          base += __popc(bal[j]);
        }
      }
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) total += __shfl_down_sync(kFullMask, total, d);
  if (lane == 0 && total) atomicAdd(d_total, total);
}

// ------------------------------------------------------------------------------------------------
// GROUPED expand: output position j -> (entry e with m_off[e] <= j < m_off[e+1]) -> one row.
//
// Every warp works alone (no CTA barrier): it owns a contiguous range of 256-output tiles and, per
// tile, stages the entries the tile touches (at most 257: every entry has at least one output) in
// its own shared-memory area, finds each output's entry there, loads the build rows and stores.
// Lane l handles outputs j0 + 32m + l (m < 8), so each store is one coalesced warp access. A
// warp's first entry comes from a 32-ary search of m_off (5 steps for 32M entries); every later
// tile starts at the entry the previous tile ended in.
// ------------------------------------------------------------------------------------------------
constexpr int kExpandThreads = 256;
constexpr int kExpandWarps = kExpandThreads / 32;
constexpr int kExpandItems = 8;
constexpr int kExpandOut = 32 * kExpandItems;  // outputs per warp tile
constexpr int kExpandEnt = kExpandOut + 1;     // entries a tile can touch

// Largest e in [0, n) with off[e] <= j (off[0] <= j assumed), found by the whole warp: each step
// compares 32 evenly spaced candidates and keeps the gap between the last one at or below j and
// the next.
__device__ __forceinline__ int64_t warp_upper_index(const int64_t* off, int64_t n, int64_t j) {
  const int lane = threadIdx.x & 31;
  int64_t lo = 0, hi = n - 1;  // off[lo] <= j; the answer is in [lo, hi]
  while (lo < hi) {
    const int64_t span = hi - lo;
    const int64_t cand = lo + 1 + (span * lane) / 32;  // 32 candidates in (lo, hi]
    const bool le = cand <= hi && __ldg(off + cand) <= j;
    const unsigned m = __ballot_sync(kFullMask, le);
    if (m == 0) {
      hi = lo;  // every candidate (the first is lo + 1) is above j: the answer is lo
    } else {
      const int top = 31 - __clz(m);
      const int64_t c_top = lo + 1 + (span * top) / 32;
      const int64_t c_next = top < 31 ? lo + 1 + (span * (top + 1)) / 32 : hi + 1;
      lo = c_top;
      hi = c_next - 1;
    }
  }
  return lo;
}

// RS > 0: a compile-time output shape — row-store records of RS bytes holding the build row id and
// one payload of RS / 2 bytes at offset RS / 2 (no validity), no probe payloads; one load per row.
// RS = 0: the shape is read from `g` at run time.
template <int RS>
__global__ void __launch_bounds__(kExpandThreads, 4) expand_kernel(const int32_t* __restrict__ m_row,
                                                                const int32_t* __restrict__ m_start,
                                                                const int64_t* __restrict__ m_off,
                                                                const unsigned long long* d_nent,
                                                                const int32_t* __restrict__ grp_rid,
                                                                GatherArgs g) {
  __shared__ int64_t s_off_all[kExpandWarps][kExpandEnt];
  __shared__ int32_t s_row_all[kExpandWarps][kExpandEnt];
  __shared__ int32_t s_start_all[kExpandWarps][kExpandEnt];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int64_t* s_off = s_off_all[warp];
  int32_t* s_row = s_row_all[warp];
  int32_t* s_start = s_start_all[warp];
  const int64_t nent = (int64_t)*d_nent;
  if (nent == 0) return;
  const int64_t M = __ldg(m_off + nent);
  const int64_t cap = M < g.capacity ? M : g.capacity;
  const int64_t ntile = (cap + kExpandOut - 1) / kExpandOut;
  const int64_t nwarps = (int64_t)gridDim.x * kExpandWarps;
  const int64_t per_warp = (ntile + nwarps - 1) / nwarps;
  const int64_t t_lo = ((int64_t)blockIdx.x * kExpandWarps + warp) * per_warp;
  const int64_t t_hi = t_lo + per_warp < ntile ? t_lo + per_warp : ntile;
  if (t_lo >= t_hi) return;
  int64_t e0 = warp_upper_index(m_off, nent, t_lo * kExpandOut);
  for (int64_t tile = t_lo; tile < t_hi; ++tile) {
    const int64_t j0 = tile * kExpandOut;
    const int64_t j1 = j0 + kExpandOut < cap ? j0 + kExpandOut : cap;
    const int ne = (int)((nent - e0) < kExpandEnt ? (nent - e0) : kExpandEnt);
    for (int i = lane; i < ne; i += 32) {
      s_off[i] = __ldg(m_off + e0 + i);
      s_row[i] = __ldg(m_row + e0 + i);
      s_start[i] = __ldg(m_start + e0 + i);
    }
    __syncwarp();
    // 1. entries (shared memory only): eb = the entry of the warp's first position of item m; the
    //    next 31 entry starts are read one per lane and OR-ed into a mask of lane offsets, so a
    //    lane's entry is eb plus the starts at or below it
    int32_t row[kExpandItems], gi[kExpandItems];
    int eb = 0;
#pragma unroll
    for (int m = 0; m < kExpandItems; ++m) {
      const int64_t jb = j0 + 32 * m;
      const int64_t j = jb + lane;
      row[m] = 0;
      gi[m] = -1;
      if (jb >= j1) continue;  // warp-uniform
      const int nb = eb + 1 + lane;
      const int64_t rel = (lane < 31 && nb < ne) ? s_off[nb] - jb : 64;
      const unsigned starts = __reduce_or_sync(kFullMask, rel < 32 ? (1u << rel) : 0u);
      const unsigned upto = lane == 31 ? kFullMask : ((2u << lane) - 1u);
      const int e = eb + __popc(starts & upto);
      if (j < j1) {
        row[m] = s_row[e];
        gi[m] = s_start[e] + (int32_t)(j - s_off[e]);
      }
      // the entry of position jb + 32: lane 31's entry, or the next one if it starts right there
      const int e31 = __shfl_sync(kFullMask, e, 31);
      eb = e31 + ((e31 + 1 < ne && s_off[e31 + 1] == jb + 32) ? 1 : 0);
    }
    // 2. group members (table positions)
    int32_t pos[kExpandItems];
#pragma unroll
    for (int m = 0; m < kExpandItems; ++m) pos[m] = gi[m] < 0 ? 0 : grp_rid ? __ldg(grp_rid + gi[m]) : gi[m];
    // 3. build side: one row-store record per item, or row id (+ payloads by row id / position)
    if constexpr (RS == 8 || RS == 16) {
      uint32_t rid[kExpandItems];
      uint64_t fv[kExpandItems];
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) {
        rid[m] = 0;
        fv[m] = 0;
        if (gi[m] < 0) continue;
        const char* rp = static_cast<const char*>(g.rec) + (int64_t)pos[m] * RS;
        if constexpr (RS == 8) {
          const uint2 x = __ldg(reinterpret_cast<const uint2*>(rp));
          rid[m] = x.x;
          fv[m] = x.y;
        } else {
          const uint4 x = __ldg(reinterpret_cast<const uint4*>(rp));
          rid[m] = x.x;
          fv[m] = ((uint64_t)x.w << 32) | x.z;
        }
      }
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) {
        if (gi[m] < 0) continue;
        const int64_t j = j0 + 32 * m + lane;
        if (g.out_prid) __stcs(g.out_prid + j, row[m]);
        if (g.out_brid) __stcs(g.out_brid + j, (int32_t)rid[m]);
        if constexpr (RS == 8) __stcs(static_cast<unsigned int*>(g.bout[0].data) + j, (unsigned int)fv[m]);
        else __stcs(static_cast<unsigned long long*>(g.bout[0].data) + j, (unsigned long long)fv[m]);
      }
    } else if (g.rec) {
      constexpr int kHalf = kExpandItems / 2;  // 4 records (up to 32 registers) in flight at a time
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        Record r[kHalf];
#pragma unroll
        for (int q = 0; q < kHalf; ++q) {
          const int m = h * kHalf + q;
          if (gi[m] >= 0)
            r[q] = load_record(static_cast<const char*>(g.rec) + (int64_t)pos[m] * g.rec_stride, g.rec_stride);
        }
#pragma unroll
        for (int q = 0; q < kHalf; ++q) {
          const int m = h * kHalf + q;
          const int64_t j = j0 + 32 * m + lane;
          const bool live = gi[m] >= 0;
          if (live && g.out_prid) __stcs(g.out_prid + j, row[m]);
          if (live && g.out_brid) __stcs(g.out_brid + j, (int32_t)r[q].w[0]);
          for (int c = 0; c < g.n_bin; ++c) {
            const int w = g.bin[c].width;
            if (live) store_elem_cs(g.bout[c].data, j, w, record_field(r[q], g.rec_off[c], w));
            if (g.rec_voff[c] >= 0) {
              const unsigned word = __ballot_sync(kFullMask, live && record_field(r[q], g.rec_voff[c], 1) != 0);
              if (lane == 0 && j - lane < j1) g.bout[c].valid[(j - lane) >> 5] = word;
            }
          }
        }
      }
    } else {
      int32_t rid[kExpandItems];
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) rid[m] = gi[m] >= 0 ? brid_of(g, pos[m]) : 0;
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) {
        const int64_t j = j0 + 32 * m + lane;
        const bool live = gi[m] >= 0;
        if (live && g.out_prid) __stcs(g.out_prid + j, row[m]);
        if (live && g.out_brid) __stcs(g.out_brid + j, rid[m]);
        for (int c = 0; c < g.n_bin; ++c) {
          const PayloadIn in = g.bin[c];
          const int32_t idx = g.bin_by_pos ? pos[m] : rid[m];
          bool v = false;
          if (live) {
            store_elem_cs(g.bout[c].data, j, in.width, pl_load(in, idx));
            v = payload_valid(in, idx);
          }
          if (has_validity(in)) {
            const unsigned word = __ballot_sync(kFullMask, v);
            if (lane == 0 && j - lane < j1) g.bout[c].valid[(j - lane) >> 5] = word;
          }
        }
      }
    }
    // 4. probe payloads (by probe row)
    for (int c = 0; c < (RS > 0 ? 0 : g.n_pin); ++c) {
      const PayloadIn in = g.pin[c];
      uint64_t v[kExpandItems];
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) v[m] = gi[m] >= 0 ? pl_load(in, row[m]) : 0;
#pragma unroll
      for (int m = 0; m < kExpandItems; ++m) {
        const int64_t j = j0 + 32 * m + lane;
        const bool live = gi[m] >= 0;
        if (live) store_elem_cs(g.pout[c].data, j, in.width, v[m]);
        if (has_validity(in)) {
          const unsigned word = __ballot_sync(kFullMask, live && payload_valid(in, row[m]));
          if (lane == 0 && j - lane < j1) g.pout[c].valid[(j - lane) >> 5] = word;
        }
      }
    }
    e0 += eb;      // the entry of position j0 + 256: where the next tile starts
    __syncwarp();  // every lane is done with this tile's staged entries
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static int probe_grid(const sj_table* t, int64_t n, int block) {
  const int64_t tiles = (n + (int64_t)block * KPT - 1) / ((int64_t)block * KPT);
  const int64_t cap = (int64_t)sm_count(t->device) * std::max(1, t->params.ctas_per_sm);
  return (int)std::max<int64_t>(1, std::min(tiles, cap));
}

template <typename K, bool WIDE, bool VEC, bool COUNT_ONLY>
static void launch_distinct(const sj_table* t, const sj_column& p, const int64_t* d_n, const GatherArgs& g,
                            cudaStream_t s) {
  const int block = kProbeThreads;
  const int grid = probe_grid(t, p.num_rows, block);
  // output reservation: per CTA tile for large probes (or when asked), per warp otherwise
  const int agg = t->params.aggregation;
  const bool cta = agg == SJ_AGG_CTA || (agg == SJ_AGG_AUTO && p.num_rows >= (1 << 20));
  KernelTimer timer(COUNT_ONLY ? "probe_distinct_count" : "probe_distinct", s);
  if (cta && !COUNT_ONLY)
    probe_distinct_kernel<K, WIDE, VEC, COUNT_ONLY, true><<<grid, block, 0, s>>>(
        table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, d_n, g);
  else
    probe_distinct_kernel<K, WIDE, VEC, COUNT_ONLY, false><<<grid, block, 0, s>>>(
        table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, d_n, g);
}

// d_n: optional device-resident row count (a partitioned probe's valid rows); p.num_rows bounds it.
template <bool COUNT_ONLY>
static void dispatch_distinct(const sj_table* t, const sj_column& p, const int64_t* d_n, const GatherArgs& g,
                              cudaStream_t s) {
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  const bool vec = aligned16(p.data);
#define SJ_D(K, W, V) launch_distinct<K, W, V, COUNT_ONLY>(t, p, d_n, g, s)
  if (t->key_type == SJ_INT32) {
    if (wide) { if (vec) SJ_D(int32_t, true, true); else SJ_D(int32_t, true, false); }
    else { if (vec) SJ_D(int32_t, false, true); else SJ_D(int32_t, false, false); }
  } else {
    if (wide) { if (vec) SJ_D(int64_t, true, true); else SJ_D(int64_t, true, false); }
    else { if (vec) SJ_D(int64_t, false, true); else SJ_D(int64_t, false, false); }
  }
#undef SJ_D
}

template <typename K, bool WIDE, bool COMPACT>
static void launch_match(const sj_table* t, const sj_column& p, int32_t* m_row, int32_t* m_start, int32_t* m_cnt,
                         unsigned long long* d_nent, unsigned long long* d_total, cudaStream_t s) {
  const int block = kProbeThreads;
  KernelTimer timer(COMPACT ? "grouped_match" : "grouped_count", s);
  const int64_t wtiles = (p.num_rows + 32 * kMatchR - 1) / (32 * kMatchR);
  const int64_t cap = (int64_t)sm_count(t->device) * std::max(1, t->params.ctas_per_sm);
  const int grid = (int)std::max<int64_t>(1, std::min(cap, (wtiles + kWarpsPerCta - 1) / kWarpsPerCta));
  grouped_match_kernel<K, WIDE, COMPACT><<<grid, block, 0, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, m_row, m_start,
      m_cnt, d_nent, d_total);
}

template <bool COMPACT>
static void dispatch_match(const sj_table* t, const sj_column& p, int32_t* m_row, int32_t* m_start, int32_t* m_cnt,
                           unsigned long long* d_nent, unsigned long long* d_total, cudaStream_t s) {
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
#define SJ_M(K, W) launch_match<K, W, COMPACT>(t, p, m_row, m_start, m_cnt, d_nent, d_total, s)
  if (t->key_type == SJ_INT32) {
    if (wide) SJ_M(int32_t, true);
    else SJ_M(int32_t, false);
  } else {
    if (wide) SJ_M(int64_t, true);
    else SJ_M(int64_t, false);
  }
#undef SJ_M
}

static sj_status check_probe(const sj_table* t, const sj_column& p) {
  SJ_TRY(validate_column(&p, "probe key", true));
  if (p.type != t->key_type) return set_error(SJ_ERR_INVALID, "probe key type differs from the build key type");
  if (p.num_rows > INT32_MAX) return set_error(SJ_ERR_INVALID, "probe side exceeds the int32 row-id range");
  return SJ_OK;
}

sj_status probe_count(const sj_table* t, const sj_column& p, const Allocator& alloc, cudaStream_t s,
                      int64_t* d_count) {
  SJ_TRY(check_probe(t, p));
  (void)alloc;
  SJ_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(int64_t), s));
  if (p.num_rows == 0) return SJ_OK;
  unsigned long long* dc = reinterpret_cast<unsigned long long*>(d_count);
  if (t->layout == SJ_LAYOUT_DISTINCT) {
    GatherArgs g{};
    g.d_count = dc;
    dispatch_distinct<true>(t, p, nullptr, g, s);
  } else {
    dispatch_match<false>(t, p, nullptr, nullptr, nullptr, nullptr, dc, s);
  }
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

static sj_status fill_gather(const sj_table* t, const sj_column& p, const GatherSpec& gs, GatherArgs& g) {
  if (gs.n_probe_payload < 0 || gs.n_probe_payload > kMaxPayload || gs.n_build_payload < 0 ||
      gs.n_build_payload > kMaxPayload)
    return set_error(SJ_ERR_INVALID, "at most 8 payload columns per side");
  if (gs.capacity < 0) return set_error(SJ_ERR_INVALID, "capacity must be >= 0");
  if ((gs.n_probe_payload && (!gs.probe_payload || !gs.out_probe_payload)) ||
      (gs.n_build_payload && !gs.out_build_payload))
    return set_error(SJ_ERR_INVALID, "payload column arrays must not be NULL");
  const bool attached = gs.n_build_payload > 0 && gs.build_payload == nullptr;
  if (attached && gs.n_build_payload != t->n_attached)
    return set_error(SJ_ERR_INVALID, "build_payload is NULL (use the attached columns) but num_build_payload "
                                     "differs from the number of columns attached at build");
  g.n_pin = gs.n_probe_payload;
  g.n_bin = gs.n_build_payload;
  auto fill = [&](const sj_column& in, const sj_mut_column& out, int64_t rows, PayloadIn& pi, PayloadOut& po,
                  const char* side) -> sj_status {
    SJ_TRY(validate_column(&in, side, false));
    if (in.num_rows != rows)
      return set_error(SJ_ERR_INVALID, std::string(side) + " payload row count differs from its key column");
    if (out.type != in.type) return set_error(SJ_ERR_INVALID, std::string(side) + " output type differs");
    if (gs.capacity > 0 && !out.data) return set_error(SJ_ERR_INVALID, std::string(side) + " output data is NULL");
    if (in.validity && gs.capacity > 0 && !out.validity)
      return set_error(SJ_ERR_INVALID, std::string(side) + " payload has NULLs but its output has no validity");
    pi = column_payload(in.data, in.validity, in.validity_offset, type_width(in.type));
    po.data = out.data;
    po.valid = in.validity ? out.validity : nullptr;
    return SJ_OK;
  };
  for (int c = 0; c < g.n_pin; ++c)
    SJ_TRY(fill(gs.probe_payload[c], gs.out_probe_payload[c], p.num_rows, g.pin[c], g.pout[c], "probe"));
  if (attached) {
    for (int c = 0; c < g.n_bin; ++c) {
      const sj_mut_column& out = gs.out_build_payload[c];
      if (out.type != t->apay_type[c]) return set_error(SJ_ERR_INVALID, "attached build output type differs");
      if (gs.capacity > 0 && !out.data) return set_error(SJ_ERR_INVALID, "build output data is NULL");
      if (t->apay_valid[c] && gs.capacity > 0 && !out.validity)
        return set_error(SJ_ERR_INVALID, "attached build payload has NULLs but its output has no validity");
      g.bin[c] = PayloadIn{t->apay[c], nullptr, t->apay_valid[c], 0, type_width(t->apay_type[c]), t->apay_stride[c],
                           t->apay_vstride[c], 0};
      g.bout[c] = PayloadOut{out.data, t->apay_valid[c] ? out.validity : nullptr};
      if (t->arow) {
        g.rec_off[c] = (int16_t)(static_cast<const char*>(t->apay[c]) - static_cast<const char*>(t->arow));
        g.rec_voff[c] = t->apay_valid[c] ? (int16_t)(reinterpret_cast<const char*>(t->apay_valid[c]) -
                                                     static_cast<const char*>(t->arow))
                                         : (int16_t)-1;
      }
    }
    g.bin_by_pos = 1;
    if (t->arow && t->arow_stride <= 32) {
      g.rec = t->arow;
      g.rec_stride = t->arow_stride;
    }
  } else {
    for (int c = 0; c < g.n_bin; ++c)
      SJ_TRY(fill(gs.build_payload[c], gs.out_build_payload[c], t->build_rows, g.bin[c], g.bout[c], "build"));
  }
  g.brid_map = t->pos_rid;
  g.brid_stride = t->pos_stride;
  g.out_prid = gs.out_probe_rid;
  g.out_brid = gs.out_build_rid;
  g.capacity = gs.capacity;
  return SJ_OK;
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Partitioned probe of a DISTINCT table: radix-scatter the probe rows (key, row id, payloads) by
// the table's partition bits, then stream the partitioned arrays through the probe kernel, so
// each partition's probes hit its L2-resident table segment and attached payload rows.
// Probe-side radix bits: the coarsest prefix of the table's partition bits whose share of the
// table footprint (slots + position map + attached payloads) stays under 48 MB of L2 (or the
// table's probe_partition_mb). A coarse
// probe partition covers 2^(table bits - probe bits) contiguous table segments, and fewer
// partitions mean longer contiguous runs in the scatter (16M-row table, 768 MB: 12 MB shares made
// the probe 2 % faster and the scatter 15 % slower than 48 MB shares; 24 MB was in between).
static int probe_partition_bits(const sj_table* t) {
  size_t fp = t->slots_bytes + t->arow_bytes;
  const size_t share = (size_t)(t->params.probe_partition_mb > 0 ? t->params.probe_partition_mb : 48) << 20;
  int b = 1;
  while (b < t->pbits && (fp >> b) > share) ++b;
  return std::min(b, t->pbits);
}

static sj_status probe_partitioned(const sj_table* t, const sj_column& p, GatherArgs g, const Allocator& alloc,
                                   cudaStream_t s) {
  const int64_t n = p.num_rows;
  const int pbits = probe_partition_bits(t);
  const int kw = t->key_type == SJ_INT32 ? 4 : 8;
  // Tile-local partition (one pass, no histogram) + the run-walking probe, when the direct probe
  // serves the output shape and the probe payloads are plain 4/8-byte columns without NULLs.
  bool local = probe_runs_ok(t, g) && g.n_pin <= 2;
  for (int c = 0; c < g.n_pin; ++c)
    local = local && !g.pin[c].valid && !g.pin[c].valid8 && (g.pin[c].width == 4 || g.pin[c].width == 8) &&
            g.pin[c].stride == g.pin[c].width;
  const int64_t n_tiles = (n + kPartTileRows - 1) / kPartTileRows;
  const size_t run_bytes = (size_t)n_tiles * ((size_t)1 << pbits) * sizeof(int32_t);
  size_t bytes = align256((size_t)n * kw) + align256((size_t)n * 4) + 256 +
                 (local ? 2 * align256(run_bytes) : partition_scratch_bytes(pbits, t->device));
  for (int c = 0; c < g.n_pin; ++c)
    bytes += align256((size_t)n * g.pin[c].width) + (g.pin[c].valid ? align256((size_t)n) : 0);
  Scratch sc;
  SJ_TRY(sc.get(alloc, bytes, s));
  char* cur = sc.as<char>();
  auto carve = [&](size_t b) {
    char* r = cur;
    cur += align256(b);
    return r;
  };
  PartSrc ps{};
  PartDst pd{};
  ps.keys = p.data;
  ps.kvalid = p.validity;
  ps.kvoff = p.validity_offset;
  ps.n = n;
  ps.n_pay = g.n_pin;
  pd.keys = carve((size_t)n * kw);
  pd.rid = reinterpret_cast<int32_t*>(carve((size_t)n * 4));
  for (int c = 0; c < g.n_pin; ++c) {
    ps.pay[c] = g.pin[c];
    pd.pay[c] = carve((size_t)n * g.pin[c].width);
    pd.valid8[c] = g.pin[c].valid ? reinterpret_cast<uint8_t*>(carve((size_t)n)) : nullptr;
  }
  unsigned long long* tile_ctr = reinterpret_cast<unsigned long long*>(carve(8));
  if (local) {
    int32_t* run_off = reinterpret_cast<int32_t*>(carve(run_bytes));
    int32_t* run_cnt = reinterpret_cast<int32_t*>(carve(run_bytes));
    SJ_TRY(local_partition(ps, t->key_type, pbits, pd, run_off, run_cnt, t->device, s));
    g.prid_map = pd.rid;
    for (int c = 0; c < g.n_pin; ++c) g.pin[c] = column_payload(pd.pay[c], nullptr, 0, g.pin[c].width);
    const RunArgs ra{run_off, run_cnt, (uint32_t)n_tiles, 1u << pbits, 1u};  // group: set by probe_runs
    probe_runs(t, pd.keys, ra, g, s, tile_ctr);
    SJ_CUDA_TRY(cudaGetLastError());
    return SJ_OK;
  }
  void* pscratch = carve(partition_scratch_bytes(pbits, t->device));
  const int64_t *d_total, *d_offs;
  int G;
  SJ_TRY(radix_partition(ps, t->key_type, pbits, pd, pscratch, t->device, s, &d_total, &d_offs, &G));
  g.prid_map = pd.rid;
  for (int c = 0; c < g.n_pin; ++c)
    g.pin[c] = PayloadIn{pd.pay[c], nullptr, pd.valid8[c], 0, g.pin[c].width, g.pin[c].width, 1, 0};
  const sj_column pk{pd.keys, nullptr, 0, n, t->key_type, 0};
  if (!probe_direct(t, pk, d_total, g, s, alloc, tile_ctr)) dispatch_distinct<false>(t, pk, d_total, g, s);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

// Probes of at least this many rows into a partitioned table take the partitioned path.

sj_status probe_gather(const sj_table* t, const sj_column& p, const GatherSpec& gs, const Allocator& alloc,
                       cudaStream_t s, int64_t* d_count) {
  SJ_TRY(check_probe(t, p));
  GatherArgs g{};
  SJ_TRY(fill_gather(t, p, gs, g));
  g.d_count = reinterpret_cast<unsigned long long*>(d_count);
  SJ_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(int64_t), s));
  const size_t vbytes = (size_t)((gs.capacity + 31) / 32) * sizeof(uint32_t);
  for (int c = 0; c < g.n_pin; ++c)
    if (g.pout[c].valid && vbytes) SJ_CUDA_TRY(cudaMemsetAsync(g.pout[c].valid, 0, vbytes, s));
  for (int c = 0; c < g.n_bin; ++c)
    if (g.bout[c].valid && vbytes) SJ_CUDA_TRY(cudaMemsetAsync(g.bout[c].valid, 0, vbytes, s));
  if (p.num_rows == 0) return SJ_OK;

  if (t->layout == SJ_LAYOUT_DISTINCT) {
    if (t->pbits > 0 && p.num_rows >= kMinPartitionedProbe) return probe_partitioned(t, p, g, alloc, s);
    if (!probe_direct(t, p, nullptr, g, s, alloc, nullptr)) dispatch_distinct<false>(t, p, nullptr, g, s);
    SJ_CUDA_TRY(cudaGetLastError());
    return SJ_OK;
  }
  const int64_t n = p.num_rows;
  Scratch sc;
  const size_t b_row = ((size_t)n * 4 + 255) & ~(size_t)255;
  const size_t b_off = ((size_t)(n + 1) * 8 + 255) & ~(size_t)255;
  const size_t b_tmp = kScanBlocks * sizeof(int64_t);
  SJ_TRY(sc.get(alloc, 3 * b_row + b_off + b_tmp + 256, s));
  char* base = sc.as<char>();
  int32_t* m_row = reinterpret_cast<int32_t*>(base);
  int32_t* m_start = reinterpret_cast<int32_t*>(base + b_row);
  int32_t* m_cnt = reinterpret_cast<int32_t*>(base + 2 * b_row);
  int64_t* m_off = reinterpret_cast<int64_t*>(base + 3 * b_row);
  int64_t* tmp = reinterpret_cast<int64_t*>(base + 3 * b_row + b_off);
  unsigned long long* d_nent = reinterpret_cast<unsigned long long*>(base + 3 * b_row + b_off + b_tmp);
  SJ_CUDA_TRY(cudaMemsetAsync(d_nent, 0, sizeof(unsigned long long), s));
  dispatch_match<true>(t, p, m_row, m_start, m_cnt, d_nent, g.d_count, s);
  {
    KernelTimer timer("scan", s);
    device_exclusive_scan<int32_t, int64_t>(m_cnt, m_off, d_nent, 0, tmp, s);
  }
  // every block resident at once: a warp's tile range is fixed, so a second wave would be a tail
  // the compile-time shape: records [row id | one 4- or 8-byte payload], nothing else gathered
  int rs = 0;
  if (g.rec && g.n_pin == 0 && g.n_bin == 1 && g.rec_voff[0] < 0 && !g.bout[0].valid &&
      (g.rec_stride == 8 || g.rec_stride == 16) && g.bin[0].width * 2 == g.rec_stride &&
      g.rec_off[0] * 2 == g.rec_stride)
    rs = g.rec_stride;
  auto kernel = rs == 8 ? expand_kernel<8> : rs == 16 ? expand_kernel<16> : expand_kernel<0>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kExpandThreads, 0);
  const int grid = sm_count(t->device) * std::max(1, per_sm);
  KernelTimer timer("expand", s);
  kernel<<<grid, kExpandThreads, 0, s>>>(m_row, m_start, m_off, d_nent, t->grp_rid, g);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
