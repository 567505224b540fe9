// DISTINCT probe with a direct write-out, for the common output shapes:
//   build side: row ids plus up to 3 build payloads, either the 8-byte attached fields of the
//               table's row store (record = [row id | pad | field 0 | field 1 | field 2], one
//               load per match) or plain 4/8-byte columns without NULLs gathered by row id;
//   probe side: row ids plus up to 2 plain 4/8-byte payload columns without NULLs.
// Other shapes (NULL payloads, 1/2-byte payloads, more columns) take the staged write-out kernel
// in sj_probe.cu.
//
// Layout of the work: a warp owns 32*R consecutive probe rows and lane l handles rows
// base + 32*j + l (j < R), so every load of keys, probe payloads and partition row ids is one
// fully coalesced warp access. After probing, the warp's hits for row group j are ranked with one
// __ballot_sync: hit lanes of group j write positions off_j + popc(ballot_j & lanes below), so the
// 32 lanes of a group store one contiguous run of every output column — no shared-memory staging
// and no per-match shuffles. Output ranges are reserved with one atomicAdd per CTA tile (or per
// warp for small probes). All gather loads of a tile (records, payloads, row ids) are issued
// before the first store, so each lane keeps 3R-5R independent loads in flight.
#include <algorithm>

#include "sj_bulk.cuh"
#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_partition.cuh"
#include "sj_probe_direct.h"

namespace sj {

TableDev table_dev(const sj_table* t);

constexpr int kDirectThreads = 64;  // 2 warps: the reservation barriers wait on one other warp only
constexpr int kDirectWarps = kDirectThreads / 32;

__device__ __forceinline__ uint64_t ld_cs_w(const void* base, int64_t i, int w) {
  return w == 8 ? __ldcs(reinterpret_cast<const unsigned long long*>(base) + i)
                : (uint64_t)__ldcs(reinterpret_cast<const unsigned int*>(base) + i);
}
__device__ __forceinline__ uint64_t ld_nc_w(const void* a, int w) {
  return w == 8 ? __ldg(reinterpret_cast<const unsigned long long*>(a))
                : (uint64_t)__ldg(reinterpret_cast<const unsigned int*>(a));
}
__device__ __forceinline__ void st_cs_w(void* base, int64_t i, int w, uint64_t v) {
  if (w == 8) __stcs(reinterpret_cast<unsigned long long*>(base) + i, (unsigned long long)v);
  else __stcs(reinterpret_cast<unsigned int*>(base) + i, (unsigned int)v);
}

// One row-store record of 8, 16 or 32 bytes (the stride) in one load, under L2 policy `pol`.
__device__ __forceinline__ void load_rec_hint(const void* p, int stride, uint32_t (&w)[8], uint64_t pol) {
  if (stride == 32) {
    asm("ld.global.nc.L2::cache_hint.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p), "l"(pol));
  } else if (stride == 16) {
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
        : "l"(p), "l"(pol));
    w[4] = w[5] = w[6] = w[7] = 0;
  } else {
    asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(w[0]), "=r"(w[1]) : "l"(p), "l"(pol));
    w[2] = w[3] = w[4] = w[5] = w[6] = w[7] = 0;
  }
}

// One row-store record of 8, 16 or 32 bytes (the stride) in one load.
__device__ __forceinline__ void load_rec(const void* p, int stride, uint32_t (&w)[8]) {
  if (stride == 32) {
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p));
  } else if (stride == 16) {
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
    w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
    w[4] = w[5] = w[6] = w[7] = 0;
  } else {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
    w[0] = x.x; w[1] = x.y;
    w[2] = w[3] = w[4] = w[5] = w[6] = w[7] = 0;
  }
}

// SP / SB >= 0: a compile-time output shape (SP probe payloads, SB attached build fields from the
// row store, every width 8 bytes); -1: the shape is read from `a` at run time.
// AGG: 0 = one output atomicAdd per warp, static grid-stride CTA tiles; 1 = one per CTA tile (2 CTA
// barriers), CTA tiles from the shared counter; 2 = one per warp, warp tiles from the shared counter
// (no barriers).
// Field of `width` (4 or 8) bytes at byte offset `off` of a record held in 8 words, picked with
// predicated moves so the record stays in registers.
__device__ __forceinline__ uint64_t rec_word_field(const uint32_t (&w)[8], int off, int width) {
  const int wi = off >> 2;
  uint32_t lo = 0, hi = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    lo = k == wi ? w[k] : lo;
    hi = k == wi + 1 ? w[k] : hi;
  }
  return width == 8 ? ((uint64_t)hi << 32) | lo : lo;
}

template <typename K, bool WIDE, int R, int AGG, int SP = -1, int SB = -1>
__global__ void __launch_bounds__(kDirectThreads, (R <= 2 ? 1024 : R == 3 ? 768 : 512) / kDirectThreads)
    probe_direct_kernel(TableDev t, const K* __restrict__ keys, const uint32_t* __restrict__ kv, int64_t kvoff,
                        int64_t n_host, const int64_t* d_n, DirectArgs a) {
  using Ops = SlotOps<WIDE>;
  const uint64_t pol = a.l2_last ? l2_policy_evict_last() : 0ull;  // table loads' L2 policy
  constexpr bool kFixed = SP >= 0;
  const int n_pin = kFixed ? SP : a.n_pin;
  const int n_bin = kFixed ? SB : a.n_bin;
  const bool use_rec = kFixed ? SB > 0 : a.rec != nullptr;
  const int rec_stride = kFixed ? (SB == 1 ? 16 : 32) : a.rec_stride;
  __shared__ unsigned s_wtot[kDirectWarps];
  __shared__ unsigned long long s_wbase[kDirectWarps];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  // 32-bit row and position arithmetic: probe rows < 2^31 (the int32 row-id range), and a DISTINCT
  // probe never has more matches than rows
  const uint32_t n = (uint32_t)(d_n ? *d_n : n_host);
  const uint32_t cap = (uint32_t)(a.capacity < (int64_t)n ? a.capacity : (int64_t)n);
  constexpr bool CTA_AGG = AGG == 1;
  constexpr bool kWarpTiles = AGG == 2;
  constexpr uint32_t kRowsCta = kWarpTiles ? 32u * R : (uint32_t)kDirectThreads * R;  // rows per tile
  const uint32_t tiles = (n + kRowsCta - 1) / kRowsCta;
  const uint32_t units = kWarpTiles ? gridDim.x * kDirectWarps : gridDim.x;  // tile takers
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  const uint32_t lane_off = kWarpTiles ? (uint32_t)lane : (uint32_t)warp * (32 * R) + lane;  // + 32 j
  const uint32_t first = kWarpTiles ? blockIdx.x * kDirectWarps + warp : blockIdx.x;
  __shared__ uint32_t s_next;
  K k[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const uint32_t r = first * kRowsCta + lane_off + 32 * j;
    k[j] = r < n ? __ldcs(keys + r) : (K)0;
  }
  // Tiles: the first two of a CTA are static (blockIdx.x, + gridDim.x); with CTA reservation the
  // later ones come from a shared tile counter, so the CTAs sweep the (partition-ordered) probe
  // rows together and the table rows in use stay one partition's worth, resident in L2.
  uint32_t tile = first, nxt = tile + units;
  while (tile < tiles) {
    const uint32_t r0 = tile * kRowsCta + lane_off;
    uint32_t act = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint32_t r = r0 + 32 * j;
      if (r < n && bit_valid(kv, kvoff, r) && in_range(t, k[j])) act |= 1u << j;
    }
    uint32_t b[R];
    uint64_t ks[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint64_t kb = key_u64<K>(k[j]);
      b[j] = home_bucket(t, kb);
      ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
    }
    // the next tile's keys load while this tile probes, gathers and writes
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint32_t r = nxt * kRowsCta + lane_off + 32 * j;
      k[j] = r < n ? __ldcs(keys + r) : (K)0;
    }
    int32_t pos[R];
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) pos[j] = 0;
    for (uint32_t step = 0; act && step <= t.segmask; ++step) {
      Bucket bk[R];
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (act >> j & 1u) bk[j] = a.l2_last ? load_bucket_hint(t.slots, b[j], pol) : load_bucket<true>(t.slots, b[j]);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (!(act >> j & 1u)) continue;
        int32_t pj;
        const bool m = Ops::match_distinct(bk[j], ks[j], kmask, t.rbits, pj);
        if (m) {
          pos[j] = pj;
          hit |= 1u << j;
        }
        if (m || Ops::open(bk[j])) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    // ---- gather loads for every hit (they need no output position, so they are in flight
    //      while the output range is reserved) ----
    int32_t prid[R], brid[R];
    uint64_t pv[kDirectMaxProbePayload][R];
    uint64_t bv[kDirectMaxBuildPayload][R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      prid[j] = brid[j] = 0;
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c) pv[c][j] = 0;
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c) bv[c][j] = 0;
      if (!(hit >> j & 1u)) continue;
      const uint32_t r = r0 + 32 * j;
      if (a.out_prid) prid[j] = a.prid_map ? __ldcs(a.prid_map + r) : (int32_t)r;
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c)
        if (c < n_pin) pv[c][j] = ld_cs_w(a.pin[c], r, kFixed ? 8 : a.pin_w[c]);
      if (use_rec) {
        uint32_t w[8];
        const char* recp = static_cast<const char*>(a.rec) + (size_t)(uint32_t)pos[j] * rec_stride;
        if (a.l2_last) load_rec_hint(recp, rec_stride, w, pol);
        else load_rec(recp, rec_stride, w);
        brid[j] = (int32_t)w[0];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c)
          bv[c][j] = kFixed || a.rec_std ? ((uint64_t)w[3 + 2 * c] << 32) | w[2 + 2 * c]
                                         : rec_word_field(w, a.rec_off[c], a.bin_w[c]);
      } else {
        brid[j] = a.brid_map ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(a.brid_map) +
                                                                       (int64_t)pos[j] * a.brid_stride))
                             : pos[j];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c) {
          if (c < n_bin) {
            const int64_t i = a.bin_by_pos ? pos[j] : brid[j];
            bv[c][j] = ld_nc_w(static_cast<const char*>(a.bin[c]) + i * a.bin_stride[c], a.bin_w[c]);
          }
        }
      }
    }
    unsigned bal[R];
    unsigned wtot = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      bal[j] = __ballot_sync(kFullMask, (hit >> j) & 1u);
      wtot += __popc(bal[j]);
    }
    unsigned long long base;
    uint32_t nn = 0;  // AGG 2: this warp's next tile
    if (CTA_AGG) {
      if (lane == 0) s_wtot[warp] = wtot;
      __syncthreads();
      if (warp == 0) {
        const unsigned v = lane < kDirectWarps ? s_wtot[lane] : 0u;
        unsigned incl = v;
#pragma unroll
        for (int d = 1; d < kDirectWarps; d <<= 1) {
          const unsigned o = __shfl_up_sync(kFullMask, incl, d);
          if (lane >= d) incl += o;
        }
        const unsigned tot = __shfl_sync(kFullMask, incl, kDirectWarps - 1);
        unsigned long long cb = 0;
        if (lane == 0 && tot) cb = atomicAdd(a.d_count, (unsigned long long)tot);
        if (lane == 1) s_next = 2 * gridDim.x + (uint32_t)atomicAdd(a.tile_ctr, 1ull);
        cb = __shfl_sync(kFullMask, cb, 0);
        if (lane < kDirectWarps) s_wbase[lane] = cb + (incl - v);
      }
      __syncthreads();
      base = s_wbase[warp];
    } else {
      base = 0;
      if (lane == 0 && wtot) base = atomicAdd(a.d_count, (unsigned long long)wtot);
      if (kWarpTiles && lane == 1) nn = 2 * units + (uint32_t)atomicAdd(a.tile_ctr, 1ull);
      base = __shfl_sync(kFullMask, base, 0);
      if (kWarpTiles) nn = __shfl_sync(kFullMask, nn, 1);
    }
    tile = nxt;
    nxt = CTA_AGG ? s_next : kWarpTiles ? nn : nxt + units;
    if (wtot == 0) continue;
    uint32_t p[R];
    {
      uint32_t run = (uint32_t)base;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        p[j] = run + __popc(bal[j] & below);
        run += __popc(bal[j]);
      }
    }
    // ---- stores: each row group j is one contiguous run of positions per column ----
#pragma unroll
    for (int j = 0; j < R; ++j) {
      if (!(hit >> j & 1u) || p[j] >= cap) continue;
      if (a.out_prid) __stcs(a.out_prid + p[j], prid[j]);
      if (a.out_brid) __stcs(a.out_brid + p[j], brid[j]);
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c)
        if (c < n_pin) st_cs_w(a.pout[c], p[j], kFixed ? 8 : a.pin_w[c], pv[c][j]);
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c)
        if (c < n_bin) st_cs_w(a.bout[c], p[j], kFixed ? 8 : a.bin_w[c], bv[c][j]);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// The direct probe over tile-local partition runs. A work item is (partition p, 4 consecutive
// tiles): its rows are the 4 runs of p in those tiles, concatenated. Items are taken partition-major
// (all tiles of partition 0 first) from the shared counter, so the CTAs sweep one partition's table
// rows at a time. A CTA keeps two item descriptors (run offsets and a prefix of run lengths in
// shared memory) and walks their concatenation in full chunks of 128 rows (lane l of warp w: chunk
// rows 64w + 32j + l), a chunk taking the tail of one item and the head of the next; a finished item
// frees its slot for the next one. Output reservation: one atomicAdd per chunk (two CTA barriers),
// as in probe_direct_kernel.
// ------------------------------------------------------------------------------------------------
constexpr int kMaxRunGroup = 16;
constexpr int kRunItemRows = 512;

template <typename K, bool WIDE, int SP, int SB>
__global__ void __launch_bounds__(kDirectThreads, 1024 / kDirectThreads)
    probe_runs_kernel(TableDev t, const K* __restrict__ keys, RunArgs ra, DirectArgs a) {
  using Ops = SlotOps<WIDE>;
  const uint64_t pol = a.l2_last ? l2_policy_evict_last() : 0ull;  // table loads' L2 policy
  constexpr int R = 2;
  constexpr bool kFixed = SP >= 0;
  const int n_pin = kFixed ? SP : a.n_pin;
  const int n_bin = kFixed ? SB : a.n_bin;
  const bool use_rec = kFixed ? SB > 0 : a.rec != nullptr;
  const int rec_stride = kFixed ? (SB == 1 ? 16 : 32) : a.rec_stride;
  constexpr uint32_t kChunk = (uint32_t)kDirectThreads * R;
  __shared__ unsigned s_wtot[kDirectWarps];
  __shared__ unsigned long long s_wbase[kDirectWarps];
  // two item descriptors: the item being walked and the next one, so a chunk can take the tail
  // of one item and the head of the next (chunks stay full)
  __shared__ int32_t s_off[2][kMaxRunGroup];
  __shared__ int32_t s_pre[2][kMaxRunGroup + 1];  // entries past the item's tiles hold its total
  __shared__ uint32_t s_after[2];  // the item to load after the one in the slot
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  const uint32_t cap = (uint32_t)(a.capacity < (int64_t)INT32_MAX ? a.capacity : (int64_t)INT32_MAX);
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  const uint32_t lane_off = (uint32_t)warp * (32 * R) + lane;
  const uint32_t G = ra.group;
  const uint32_t n_groups = (ra.n_tiles + G - 1) / G;
  const uint32_t n_items = ra.P * n_groups;
  // warp 0: descriptor of item w into slot `sl` (w >= n_items: an empty item) and the index of the
  // item after it (taken from the shared counter) into s_after[sl]
  auto load_item = [&](int sl, uint32_t w) {
    const bool in = w < n_items;
    const uint32_t p = in ? w / n_groups : 0, g = in ? w - p * n_groups : 0;
    const uint32_t ti = g * G + lane;
    const bool ok = in && (uint32_t)lane < G && ti < ra.n_tiles;
    const int32_t cnt = ok ? __ldg(ra.run_cnt + (size_t)ti * ra.P + p) : 0;
    if (lane < kMaxRunGroup) s_off[sl][lane] = ok ? __ldg(ra.run_off + (size_t)ti * ra.P + p) : 0;
    int32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t o = __shfl_up_sync(kFullMask, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane < kMaxRunGroup) s_pre[sl][lane + 1] = incl;
    if (lane == 0) {
      s_pre[sl][0] = 0;
      s_after[sl] = in ? gridDim.x + (uint32_t)atomicAdd(a.tile_ctr, 1ull) : w;
    }
  };
  // chunk row v of the concatenation (slot cur from `base` on, then slot cur ^ 1) -> array position
  auto row_in = [&](int sl, uint32_t v) -> uint32_t {
    int q = 0;
    for (uint32_t step = G / 2; step > 0; step >>= 1)
      if ((uint32_t)s_pre[sl][q + step] <= v) q += step;
    return (uint32_t)s_off[sl][q] + (v - (uint32_t)s_pre[sl][q]);
  };
  if (warp == 0) load_item(0, blockIdx.x);
  __syncthreads();
  if (warp == 0) load_item(1, s_after[0]);
  __syncthreads();
  int cur = 0;
  uint32_t base = 0;  // rows of item `cur` already taken
  uint32_t tc = (uint32_t)s_pre[0][kMaxRunGroup], tn = (uint32_t)s_pre[1][kMaxRunGroup];
  uint32_t w_after = s_after[1];  // the item to load when a slot frees
  auto map = [&](uint32_t v, uint32_t b, uint32_t c_tot, int c_sl) -> uint32_t {
    return b + v < c_tot ? row_in(c_sl, b + v) : row_in(c_sl ^ 1, b + v - c_tot);
  };
  K k[R];
  uint32_t rp[R];
  uint32_t avail = tc - base + tn;  // rows mapped by the two loaded items
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const uint32_t v = lane_off + 32 * j;
    rp[j] = v < avail ? map(v, base, tc, cur) : 0;
    k[j] = v < avail ? __ldcs(keys + rp[j]) : (K)0;
  }
  bool prefetched = true;
  while (avail > 0) {
    const uint32_t take = avail < kChunk ? avail : kChunk;
    if (!prefetched) {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const uint32_t v = lane_off + 32 * j;
        rp[j] = v < take ? map(v, base, tc, cur) : 0;
        k[j] = v < take ? __ldcs(keys + rp[j]) : (K)0;
      }
    }
    {
      uint32_t r[R];
      uint32_t act = 0;
      uint32_t b[R];
      uint64_t ks[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        r[j] = rp[j];
        if (lane_off + 32 * j < take && in_range(t, k[j])) act |= 1u << j;
        const uint64_t kb = key_u64<K>(k[j]);
        b[j] = home_bucket(t, kb);
        ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
      }
      // the next chunk's keys load while this chunk probes, when they lie in the loaded items
      prefetched = avail - take >= kChunk;
      if (prefetched) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
          rp[j] = map(take + lane_off + 32 * j, base, tc, cur);
          k[j] = __ldcs(keys + rp[j]);
        }
      }
      int32_t pos[R];
      uint32_t hit = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) pos[j] = 0;
      for (uint32_t step = 0; act && step <= t.segmask; ++step) {
        Bucket bk[R];
#pragma unroll
        for (int j = 0; j < R; ++j)
          if (act >> j & 1u) bk[j] = a.l2_last ? load_bucket_hint(t.slots, b[j], pol) : load_bucket<true>(t.slots, b[j]);
#pragma unroll
        for (int j = 0; j < R; ++j) {
          if (!(act >> j & 1u)) continue;
          int32_t pj;
          const bool m = Ops::match_distinct(bk[j], ks[j], kmask, t.rbits, pj);
          if (m) {
            pos[j] = pj;
            hit |= 1u << j;
          }
          if (m || Ops::open(bk[j])) act &= ~(1u << j);
          else b[j] = next_bucket(b[j], t.segmask);
        }
      }
      int32_t prid[R], brid[R];
      uint64_t pv[kDirectMaxProbePayload][R];
      uint64_t bv[kDirectMaxBuildPayload][R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        prid[j] = brid[j] = 0;
#pragma unroll
        for (int c = 0; c < kDirectMaxProbePayload; ++c) pv[c][j] = 0;
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c) bv[c][j] = 0;
        if (!(hit >> j & 1u)) continue;
        if (a.out_prid) prid[j] = a.prid_map ? __ldcs(a.prid_map + r[j]) : (int32_t)r[j];
#pragma unroll
        for (int c = 0; c < kDirectMaxProbePayload; ++c)
          if (c < n_pin) pv[c][j] = ld_cs_w(a.pin[c], r[j], kFixed ? 8 : a.pin_w[c]);
        if (use_rec) {
          uint32_t wd[8];
          const char* recp = static_cast<const char*>(a.rec) + (size_t)(uint32_t)pos[j] * rec_stride;
          if (a.l2_last) load_rec_hint(recp, rec_stride, wd, pol);
          else load_rec(recp, rec_stride, wd);
          brid[j] = (int32_t)wd[0];
#pragma unroll
          for (int c = 0; c < kDirectMaxBuildPayload; ++c)
            bv[c][j] = kFixed || a.rec_std ? ((uint64_t)wd[3 + 2 * c] << 32) | wd[2 + 2 * c]
                                           : rec_word_field(wd, a.rec_off[c], a.bin_w[c]);
        } else {
          brid[j] = a.brid_map ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(a.brid_map) +
                                                                         (int64_t)pos[j] * a.brid_stride))
                               : pos[j];
#pragma unroll
          for (int c = 0; c < kDirectMaxBuildPayload; ++c) {
            if (c < n_bin) {
              const int64_t i = a.bin_by_pos ? pos[j] : brid[j];
              bv[c][j] = ld_nc_w(static_cast<const char*>(a.bin[c]) + i * a.bin_stride[c], a.bin_w[c]);
            }
          }
        }
      }
      unsigned bal[R];
      unsigned wtot = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        bal[j] = __ballot_sync(kFullMask, (hit >> j) & 1u);
        wtot += __popc(bal[j]);
      }
      if (lane == 0) s_wtot[warp] = wtot;
      __syncthreads();
      if (warp == 0) {
        const unsigned v = lane < kDirectWarps ? s_wtot[lane] : 0u;
        unsigned incl = v;
#pragma unroll
        for (int d = 1; d < kDirectWarps; d <<= 1) {
          const unsigned o = __shfl_up_sync(kFullMask, incl, d);
          if (lane >= d) incl += o;
        }
        const unsigned tot = __shfl_sync(kFullMask, incl, kDirectWarps - 1);
        unsigned long long cb = 0;
        if (lane == 0 && tot) cb = atomicAdd(a.d_count, (unsigned long long)tot);
        cb = __shfl_sync(kFullMask, cb, 0);
        if (lane < kDirectWarps) s_wbase[lane] = cb + (incl - v);
      }
      __syncthreads();
      if (wtot != 0) {
        uint32_t run = (uint32_t)s_wbase[warp];
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const uint32_t pj = run + __popc(bal[j] & below);
          run += __popc(bal[j]);
          if (!(hit >> j & 1u) || pj >= cap) continue;
          if (a.out_prid) __stcs(a.out_prid + pj, prid[j]);
          if (a.out_brid) __stcs(a.out_brid + pj, brid[j]);
#pragma unroll
          for (int c = 0; c < kDirectMaxProbePayload; ++c)
            if (c < n_pin) st_cs_w(a.pout[c], pj, kFixed ? 8 : a.pin_w[c], pv[c][j]);
#pragma unroll
          for (int c = 0; c < kDirectMaxBuildPayload; ++c)
            if (c < n_bin) st_cs_w(a.bout[c], pj, kFixed ? 8 : a.bin_w[c], bv[c][j]);
        }
      }
    }
    // advance past the rows taken; a finished item frees its slot for the next one
    avail -= take;
    base += take;
    while (base >= tc && (tc != 0 || tn != 0 || w_after < n_items)) {
      base -= tc;
      cur ^= 1;
      tc = tn;
      if (warp == 0) load_item(cur ^ 1, w_after);
      __syncthreads();
      tn = (uint32_t)s_pre[cur ^ 1][kMaxRunGroup];
      w_after = s_after[cur ^ 1];
    }
    avail = (tc > base ? tc - base : 0) + tn;
  }
}

// ------------------------------------------------------------------------------------------------
// The same probe with its streaming inputs staged by the TMA engine. The probe rows of a tile
// (keys, partition row ids, probe payloads: contiguous ranges) are bulk-copied into a 3-stage
// shared-memory ring two tiles ahead of their use, so no lane waits on DRAM for them and no
// register holds them in flight; the lanes only wait on the table (bucket, then record) in L2.
// Stage of iteration i: i % 3; tile i+2 is issued right after iteration i's first CTA barrier,
// which every reader of that stage (iteration i-1) has passed. Only full tiles are staged; the
// last, partial tile of the probe reads global memory directly. A bounded mbarrier wait that runs
// out makes the whole CTA stop after its next barrier and marks the count negative (bit 63).
// ------------------------------------------------------------------------------------------------
constexpr int kTmaR = 2;
constexpr int kTmaTile = kDirectThreads * kTmaR;
constexpr int kTmaStages = 3;

struct TmaStage {
  int32_t key_off, rid_off, pay_off[kDirectMaxProbePayload], bytes;  // within a stage
};

template <typename K>
__host__ __device__ inline TmaStage tma_stage(const DirectArgs& a) {
  TmaStage st{};
  int o = 0;
  st.key_off = o;
  o += kTmaTile * (int)sizeof(K);
  st.rid_off = o;
  if (a.prid_map) o += kTmaTile * 4;
  for (int c = 0; c < kDirectMaxProbePayload; ++c) {
    st.pay_off[c] = o;
    if (c < a.n_pin) o += kTmaTile * a.pin_w[c];
  }
  st.bytes = (o + 127) & ~127;
  return st;
}

template <typename K, bool WIDE>
__global__ void __launch_bounds__(kDirectThreads, 4)
    probe_tma_kernel(TableDev t, const K* __restrict__ keys, const uint32_t* __restrict__ kv, int64_t kvoff,
                     int64_t n_host, const int64_t* d_n, DirectArgs a, TmaStage st) {
  using Ops = SlotOps<WIDE>;
  const uint64_t pol = a.l2_last ? l2_policy_evict_last() : 0ull;  // table loads' L2 policy
  constexpr int R = kTmaR;
  extern __shared__ __align__(128) unsigned char s_ring[];
  __shared__ __align__(8) uint64_t s_bar[kTmaStages];
  __shared__ unsigned s_wtot[kDirectWarps];
  __shared__ unsigned long long s_wbase[kDirectWarps];
  __shared__ int s_abort;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  const int64_t n = d_n ? *d_n : n_host;
  const int64_t tiles = (n + kTmaTile - 1) / kTmaTile;
  const int64_t full_tiles = n / kTmaTile;
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  const int li = warp * (32 * R) + lane;  // row of group j inside a tile: li + 32 j

  auto issue = [&](int64_t tt, int sidx) {  // thread 0; tt < full_tiles
    unsigned char* sb = s_ring + sidx * st.bytes;
    uint32_t bytes = kTmaTile * (uint32_t)sizeof(K);
    if (a.prid_map) bytes += kTmaTile * 4;
    for (int c = 0; c < a.n_pin; ++c) bytes += kTmaTile * a.pin_w[c];
    mbar_arrive_expect_tx(&s_bar[sidx], bytes);
    bulk_copy_g2s(sb + st.key_off, keys + tt * kTmaTile, kTmaTile * sizeof(K), &s_bar[sidx]);
    if (a.prid_map) bulk_copy_g2s(sb + st.rid_off, a.prid_map + tt * kTmaTile, kTmaTile * 4, &s_bar[sidx]);
    for (int c = 0; c < a.n_pin; ++c)
      bulk_copy_g2s(sb + st.pay_off[c], static_cast<const char*>(a.pin[c]) + tt * kTmaTile * a.pin_w[c],
                    kTmaTile * a.pin_w[c], &s_bar[sidx]);
  };

  if (threadIdx.x == 0) {
    for (int q = 0; q < kTmaStages; ++q) mbar_init(&s_bar[q], 1);
    mbar_init_fence();
    s_abort = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (blockIdx.x < full_tiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < full_tiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int it = 0;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++it) {
    const int sidx = it % kTmaStages;
    const unsigned char* sb = s_ring + sidx * st.bytes;
    const bool staged = tile < full_tiles;
    const int64_t r0 = tile * kTmaTile + li;
    bool ok = true;
    if (staged) ok = mbar_wait_bounded(&s_bar[sidx], (uint32_t)((it / kTmaStages) & 1), kBulkWaitPolls);
    K k[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t r = r0 + 32 * j;
      if (staged) k[j] = reinterpret_cast<const K*>(sb + st.key_off)[li + 32 * j];
      else k[j] = r < n ? __ldcs(keys + r) : (K)0;
    }
    uint32_t act = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t r = r0 + 32 * j;
      if (ok && r < n && bit_valid(kv, kvoff, r) && in_range(t, k[j])) act |= 1u << j;
    }
    if (!ok) s_abort = 1;
    uint32_t b[R];
    uint64_t ks[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint64_t kb = key_u64<K>(k[j]);
      b[j] = home_bucket(t, kb);
      ks[j] = Ops::probe_key((uint64_t)(long long)k[j] - (uint64_t)t.kmin, kb, t.rbits);
    }
    int32_t pos[R];
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) pos[j] = 0;
    for (uint32_t step = 0; act && step <= t.segmask; ++step) {
      Bucket bk[R];
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (act >> j & 1u) bk[j] = a.l2_last ? load_bucket_hint(t.slots, b[j], pol) : load_bucket<true>(t.slots, b[j]);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (!(act >> j & 1u)) continue;
        int32_t pj;
        const bool m = Ops::match_distinct(bk[j], ks[j], kmask, t.rbits, pj);
        if (m) {
          pos[j] = pj;
          hit |= 1u << j;
        }
        if (m || Ops::open(bk[j])) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    // build-side gather loads (the probe-side values stay in the stage until the stores)
    int32_t brid[R];
    uint64_t bv[kDirectMaxBuildPayload][R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      brid[j] = 0;
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c) bv[c][j] = 0;
      if (!(hit >> j & 1u)) continue;
      if (a.rec) {
        uint32_t w[8];
        load_rec(static_cast<const char*>(a.rec) + (int64_t)pos[j] * a.rec_stride, a.rec_stride, w);
        brid[j] = (int32_t)w[0];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c) bv[c][j] = ((uint64_t)w[3 + 2 * c] << 32) | w[2 + 2 * c];
      } else {
        brid[j] = a.brid_map ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(a.brid_map) +
                                                                       (int64_t)pos[j] * a.brid_stride))
                             : pos[j];
#pragma unroll
        for (int c = 0; c < kDirectMaxBuildPayload; ++c) {
          if (c < a.n_bin) {
            const int64_t i = a.bin_by_pos ? pos[j] : brid[j];
            bv[c][j] = ld_nc_w(static_cast<const char*>(a.bin[c]) + i * a.bin_stride[c], a.bin_w[c]);
          }
        }
      }
    }
    unsigned bal[R];
    unsigned wtot = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      bal[j] = __ballot_sync(kFullMask, (hit >> j) & 1u);
      wtot += __popc(bal[j]);
    }
    // CTA reservation; the first barrier also frees stage (it + 2) % 3 for tile it + 2
    if (lane == 0) s_wtot[warp] = wtot;
    __syncthreads();
    if (s_abort) break;
    if (threadIdx.x == 0) {
      const int64_t t2 = tile + 2 * (int64_t)gridDim.x;
      if (t2 < full_tiles) issue(t2, (it + 2) % kTmaStages);
    }
    if (warp == 0) {
      const unsigned v = lane < kDirectWarps ? s_wtot[lane] : 0u;
      unsigned incl = v;
#pragma unroll
      for (int d = 1; d < kDirectWarps; d <<= 1) {
        const unsigned o = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += o;
      }
      const unsigned tot = __shfl_sync(kFullMask, incl, kDirectWarps - 1);
      unsigned long long cb = 0;
      if (lane == 0 && tot) cb = atomicAdd(a.d_count, (unsigned long long)tot);
      cb = __shfl_sync(kFullMask, cb, 0);
      if (lane < kDirectWarps) s_wbase[lane] = cb + (incl - v);
    }
    __syncthreads();
    if (wtot == 0) continue;
    const unsigned long long base = s_wbase[warp];
    unsigned run = 0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t p = (int64_t)(base + run + __popc(bal[j] & below));
      run += __popc(bal[j]);
      if (!(hit >> j & 1u) || p >= a.capacity) continue;
      const int64_t r = r0 + 32 * j;
      const int i = li + 32 * j;
      if (a.out_prid) {
        int32_t pr;
        if (!a.prid_map) pr = (int32_t)r;
        else if (staged) pr = reinterpret_cast<const int32_t*>(sb + st.rid_off)[i];
        else pr = __ldcs(a.prid_map + r);
        __stcs(a.out_prid + p, pr);
      }
      if (a.out_brid) __stcs(a.out_brid + p, brid[j]);
#pragma unroll
      for (int c = 0; c < kDirectMaxProbePayload; ++c) {
        if (c < a.n_pin) {
          uint64_t v;
          if (staged) v = a.pin_w[c] == 8 ? reinterpret_cast<const uint64_t*>(sb + st.pay_off[c])[i]
                                          : reinterpret_cast<const uint32_t*>(sb + st.pay_off[c])[i];
          else v = ld_cs_w(a.pin[c], r, a.pin_w[c]);
          st_cs_w(a.pout[c], p, a.pin_w[c], v);
        }
      }
#pragma unroll
      for (int c = 0; c < kDirectMaxBuildPayload; ++c)
        if (c < a.n_bin) st_cs_w(a.bout[c], p, a.bin_w[c], bv[c][j]);
    }
  }
  if (s_abort && threadIdx.x == 0) {
    atomicOr(a.d_count, 1ull << 63);
    // let copies still in flight land before the CTA's shared memory is released
    for (int q = 0; q < kTmaStages; ++q) mbar_wait_bounded(&s_bar[q], 0, 64);
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
bool direct_args(const GatherArgs& g, DirectArgs& a) {
  if (g.n_pin > kDirectMaxProbePayload || g.n_bin > kDirectMaxBuildPayload) return false;
  a = DirectArgs{};
  a.out_prid = g.out_prid;
  a.out_brid = g.out_brid;
  a.prid_map = g.prid_map;
  a.capacity = g.capacity;
  a.d_count = g.d_count;
  a.n_pin = g.n_pin;
  a.n_bin = g.n_bin;
  for (int c = 0; c < g.n_pin; ++c) {
    const PayloadIn& in = g.pin[c];
    if (in.valid || in.valid8 || (in.width != 4 && in.width != 8) || in.stride != in.width) return false;
    a.pin[c] = in.data;
    a.pin_w[c] = in.width;
    a.pout[c] = g.pout[c].data;
  }
  if (g.n_bin > 0 && g.rec) {
    if (g.rec_stride != 8 && g.rec_stride != 16 && g.rec_stride != 32) return false;
    a.rec_std = 1;
    for (int c = 0; c < g.n_bin; ++c) {
      const int w = g.bin[c].width;
      if ((w != 4 && w != 8) || g.rec_voff[c] >= 0) return false;
      if (w != 8 || g.rec_off[c] != 8 + 8 * c) a.rec_std = 0;
      a.rec_off[c] = g.rec_off[c];
      a.bin_w[c] = w;
      a.bout[c] = g.bout[c].data;
    }
    a.rec = g.rec;
    a.rec_stride = g.rec_stride;
    return true;
  }
  a.brid_map = g.brid_map;
  a.brid_stride = g.brid_stride;
  a.bin_by_pos = g.bin_by_pos;
  for (int c = 0; c < g.n_bin; ++c) {
    const PayloadIn& in = g.bin[c];
    if (in.valid || in.valid8 || (in.width != 4 && in.width != 8)) return false;
    a.bin[c] = in.data;
    a.bin_stride[c] = in.stride;
    a.bin_w[c] = in.width;
    a.bout[c] = g.bout[c].data;
  }
  return true;
}

// The compile-time shape (SP, SB) that `a` has, or (-1, -1).
static void fixed_shape(const DirectArgs& a, int& sp, int& sb) {
  sp = sb = -1;
  for (int c = 0; c < a.n_pin; ++c)
    if (a.pin_w[c] != 8) return;
  if (a.n_bin > 0 && (!a.rec || !a.rec_std || a.rec_stride != (a.n_bin == 1 ? 16 : 32))) return;
  if (a.n_bin == 0 && a.rec) return;
  sp = a.n_pin;
  sb = a.n_bin;
}

template <typename K, bool WIDE, int R, int CTA, int SP, int SB>
static void launch_direct_shape(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a,
                                cudaStream_t s) {
  int resident = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, probe_direct_kernel<K, WIDE, R, CTA, SP, SB>,
                                                kDirectThreads, 0);
  const int64_t tiles = (p.num_rows + (int64_t)kDirectThreads * R - 1) / ((int64_t)kDirectThreads * R);
  // ctas_per_sm counts 256-thread CTAs
  const int per_sm = std::min(std::max(1, resident), std::max(1, t->params.ctas_per_sm) * 256 / kDirectThreads);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count(t->device) * per_sm));
  probe_direct_kernel<K, WIDE, R, CTA, SP, SB><<<grid, kDirectThreads, 0, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, d_n, a);
}

template <typename K, bool WIDE, int R, int CTA>
static void launch_direct_kernel(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a,
                                 cudaStream_t s) {
  int sp, sb;
  fixed_shape(a, sp, sb);
  // the shapes of the large foreign-key join (1 probe, 2 build payloads) and of a served lookup
  // (1 build payload) get compile-time specialisations when 2 rows per lane are used
  if (R <= 3 && sp == 1 && sb == 2) return launch_direct_shape<K, WIDE, R, CTA, 1, 2>(t, p, d_n, a, s);
  if (R <= 3 && sp == 0 && sb == 1) return launch_direct_shape<K, WIDE, R, CTA, 0, 1>(t, p, d_n, a, s);
  launch_direct_shape<K, WIDE, R, CTA, -1, -1>(t, p, d_n, a, s);
}

template <typename K, bool WIDE>
static void launch_direct(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a, int rpl,
                          int mode, cudaStream_t s) {
  if (rpl == 3) {
    if (mode == 1) launch_direct_kernel<K, WIDE, 3, 1>(t, p, d_n, a, s);
    else launch_direct_kernel<K, WIDE, 3, 0>(t, p, d_n, a, s);
  } else if (rpl >= 4) {
    if (mode == 1) launch_direct_kernel<K, WIDE, 4, 1>(t, p, d_n, a, s);
    else launch_direct_kernel<K, WIDE, 4, 0>(t, p, d_n, a, s);
  } else {
    if (mode == 1) launch_direct_kernel<K, WIDE, 2, 1>(t, p, d_n, a, s);
    else if (mode == 2) launch_direct_kernel<K, WIDE, 2, 2>(t, p, d_n, a, s);
    else launch_direct_kernel<K, WIDE, 2, 0>(t, p, d_n, a, s);
  }
}

static bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

template <typename K, bool WIDE>
static void launch_tma(const sj_table* t, const sj_column& p, const int64_t* d_n, const DirectArgs& a,
                       cudaStream_t s) {
  const TmaStage st = tma_stage<K>(a);
  const size_t smem = (size_t)kTmaStages * st.bytes;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(probe_tma_kernel<K, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int resident = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, probe_tma_kernel<K, WIDE>, kDirectThreads, smem);
  const int64_t tiles = (p.num_rows + kTmaTile - 1) / kTmaTile;
  const int per_sm = std::min(std::max(1, resident), std::max(1, t->params.ctas_per_sm));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count(t->device) * per_sm));
  probe_tma_kernel<K, WIDE><<<grid, kDirectThreads, smem, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, d_n, a, st);
}

bool probe_direct(const sj_table* t, const sj_column& p, const int64_t* d_n, const GatherArgs& g, cudaStream_t s,
                  const Allocator& alloc, unsigned long long* tile_ctr) {
  const sj_join_params& pr = t->params;
  if (pr.probe_kernel == SJ_PROBE_KERNEL_STAGED) return false;
  DirectArgs a;
  if (!direct_args(g, a)) return false;
  const int agg = pr.aggregation;
  const int mode = agg == SJ_AGG_CTA ? 1 : agg == SJ_AGG_WARP_DYNAMIC ? 2 : agg == SJ_AGG_WARP ? 0
                 : p.num_rows >= (1 << 20) ? 1 : 0;
  Scratch ctr;  // released (stream-ordered) after the launch below
  if (mode != 0 || pr.probe_kernel == SJ_PROBE_KERNEL_DIRECT_TMA) {
    if (!tile_ctr) {
      if (ctr.get(alloc, 256, s) != SJ_OK) return false;
      tile_ctr = ctr.as<unsigned long long>();
    }
    if (cudaMemsetAsync(tile_ctr, 0, sizeof(unsigned long long), s) != cudaSuccess) return false;
  }
  a.tile_ctr = tile_ctr;
  a.l2_last = pr.table_l2_priority == SJ_L2_EVICT_LAST;
  // AUTO takes the plain-load kernel: on the large 1:1 join the TMA ring's per-tile CTA barriers
  // cost more than the DRAM latency it hides (measured 1.96 vs 1.73 ms per 64M probe rows)
  bool tma = pr.probe_kernel == SJ_PROBE_KERNEL_DIRECT_TMA && (!a.rec || a.rec_std);
  tma = tma && al16(p.data) && (!a.prid_map || al16(a.prid_map));
  for (int c = 0; c < a.n_pin; ++c) tma = tma && al16(a.pin[c]);
  if (tma) {
    KernelTimer timer("probe_direct", s);
    const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
    if (t->key_type == SJ_INT32) {
      if (wide) launch_tma<int32_t, true>(t, p, d_n, a, s);
      else launch_tma<int32_t, false>(t, p, d_n, a, s);
    } else {
      if (wide) launch_tma<int64_t, true>(t, p, d_n, a, s);
      else launch_tma<int64_t, false>(t, p, d_n, a, s);
    }
    return true;
  }
  const int rpl = pr.rows_per_lane > 0 ? pr.rows_per_lane : 2;
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  KernelTimer timer("probe_direct", s);
  if (t->key_type == SJ_INT32) {
    if (wide) launch_direct<int32_t, true>(t, p, d_n, a, rpl, mode, s);
    else launch_direct<int32_t, false>(t, p, d_n, a, rpl, mode, s);
  } else {
    if (wide) launch_direct<int64_t, true>(t, p, d_n, a, rpl, mode, s);
    else launch_direct<int64_t, false>(t, p, d_n, a, rpl, mode, s);
  }
  return true;
}

bool probe_runs_ok(const sj_table* t, const GatherArgs& g) {
  const sj_join_params& pr = t->params;
  if (pr.probe_kernel == SJ_PROBE_KERNEL_STAGED || pr.probe_kernel == SJ_PROBE_KERNEL_DIRECT_TMA) return false;
  if (pr.aggregation != SJ_AGG_AUTO && pr.aggregation != SJ_AGG_CTA) return false;
  if (pr.rows_per_lane != 0 && pr.rows_per_lane != 2) return false;
  DirectArgs a;
  return direct_args(g, a);
}

template <typename K, bool WIDE, int SP, int SB>
static void launch_runs_shape(const sj_table* t, const void* keys, const RunArgs& ra, const DirectArgs& a,
                              cudaStream_t s) {
  int resident = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, probe_runs_kernel<K, WIDE, SP, SB>, kDirectThreads, 0);
  const int64_t items = (int64_t)ra.P * ((ra.n_tiles + ra.group - 1) / ra.group);
  const int per_sm = std::min(std::max(1, resident), std::max(1, t->params.ctas_per_sm) * 256 / kDirectThreads);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)sm_count(t->device) * per_sm));
  probe_runs_kernel<K, WIDE, SP, SB><<<grid, kDirectThreads, 0, s>>>(table_dev(t), static_cast<const K*>(keys), ra, a);
}

template <typename K, bool WIDE>
static void launch_runs(const sj_table* t, const void* keys, const RunArgs& ra, const DirectArgs& a, cudaStream_t s) {
  int sp, sb;
  fixed_shape(a, sp, sb);
  if (sp == 1 && sb == 2) return launch_runs_shape<K, WIDE, 1, 2>(t, keys, ra, a, s);
  if (sp == 0 && sb == 1) return launch_runs_shape<K, WIDE, 0, 1>(t, keys, ra, a, s);
  launch_runs_shape<K, WIDE, -1, -1>(t, keys, ra, a, s);
}

void probe_runs(const sj_table* t, const void* keys, const RunArgs& ra_in, const GatherArgs& g, cudaStream_t s,
                unsigned long long* tile_ctr) {
  // Tiles per work item: about kRunItemRows rows per item (a tile holds kPartTileRows / P rows of
  // a partition). The CTAs walk some thousand items at once; short items keep those rows a small
  // part of one partition's rows, so the table rows in use stay about one partition's share.
  RunArgs ra = ra_in;
  ra.group = 1;
  while (ra.group < (uint32_t)kMaxRunGroup && (uint64_t)ra.group * kPartTileRows < (uint64_t)kRunItemRows * ra.P)
    ra.group <<= 1;
  DirectArgs a;
  direct_args(g, a);
  cudaMemsetAsync(tile_ctr, 0, sizeof(unsigned long long), s);
  a.tile_ctr = tile_ctr;
  a.l2_last = t->params.table_l2_priority == SJ_L2_EVICT_LAST;
  if (ra.n_tiles == 0) return;
  KernelTimer timer("probe_runs", s);
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  if (t->key_type == SJ_INT32) {
    if (wide) launch_runs<int32_t, true>(t, keys, ra, a, s);
    else launch_runs<int32_t, false>(t, keys, ra, a, s);
  } else {
    if (wide) launch_runs<int64_t, true>(t, keys, ra, a, s);
    else launch_runs<int64_t, false>(t, keys, ra, a, s);
  }
}

}  // namespace sj
