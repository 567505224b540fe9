// Batched INNER joins: thousands of independent small joins of uneven sizes in one persistent
// launch (the BUILD_PROBE / STANDARD calls of the operator, src/op/sirius_physical_hash_join.cpp
// :1614-1688 and :1872, for many partition pairs at once), replayable as a CUDA graph.
//
// Work queue. The plan lists work items: every join's build tiles, then every join's probe tiles
// (join by join, so the few joins in flight keep their tables in L2). A CTA takes the next item
// with one atomicAdd and processes `tile_rows` rows of it:
//   build  insert each valid row into the join's table (multiset open addressing, atomicCAS),
//          then publish the tile (threadfence + atomicAdd on the join's built-tile counter);
//   probe  wait until the join's built counter reaches its build-tile count (a bounded wait:
//          every build item was handed to a running CTA before any probe item, so it ends; on
//          timeout the plan's error word is set), then probe and write the matches.
// Tables. One arena of 32-byte buckets, a power-of-two slice per join sized by its build rows and
// the load factor. int32 keys pack into 64-bit slots as (uint32 key << 32 | row id) — no key range
// pass needed, EMPTY = all ones can never be live because row ids are < 2^31; int64 keys use
// 128-bit {key, row id} slots inserted with atom.cas.b128. Duplicates stay in separate slots and
// a probe scans to the first bucket holding an EMPTY slot, so every match is produced.
// Group width G: G lanes share one probe key and each loads one bucket of a G-bucket window
// (longer probe sequences at high load factors); G = 1 is one lane per key.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

struct BJoin {
  const void* bkey;
  const uint32_t* bvalid;
  int64_t bvoff;
  const void* pkey;
  const uint32_t* pvalid;
  int64_t pvoff;
  PayloadIn bpay;  // data == NULL: no payload
  PayloadIn ppay;
  int32_t* out_prid;
  int32_t* out_brid;
  PayloadOut out_bpay;
  PayloadOut out_ppay;
  int64_t capacity;
  int64_t bucket_off;  // first bucket of this join's table in the arena
  int32_t nb;
  int32_t log2_nb;
  int64_t np;
  int32_t build_tiles;
  int32_t pad;
};

struct BItem {
  int32_t join;
  int32_t tile;
};

struct BatchDev {
  const BJoin* joins;
  const BItem* items;
  int64_t n_items;
  int64_t n_build_items;
  void* arena;
  int32_t tile_rows;
  int32_t n_joins;
  unsigned long long* queue;
  unsigned int* built;
  unsigned long long* counts;
  int32_t* error;
};

constexpr unsigned kWaitLimit = 1u << 24;  // x ~128 ns back-off: gives up after ~2 s

template <typename K>
__device__ __forceinline__ K load_key(const void* base, int64_t i) {
  return __ldg(static_cast<const K*>(base) + i);
}

// ---- table access for one join ------------------------------------------------------------------
// Bucket b of the arena in one 32-byte load through L2 (.cg: the same launch's build items wrote the
// bucket with atomics, so it must not come from a stale L1 line).
__device__ __forceinline__ void load_bucket_cg(const void* arena, uint64_t b, uint64_t (&s)[4]) {
  const unsigned long long* p = reinterpret_cast<const unsigned long long*>(arena) + b * 4;
  asm volatile("ld.global.cg.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(s[0]), "=l"(s[1]), "=l"(s[2]), "=l"(s[3]) : "l"(p));
}

template <typename K>
struct BTable;

template <>
struct BTable<int32_t> {  // 4 x uint64 (key << 32 | rid) per bucket
  static constexpr int kSlots = 4;
  __device__ __forceinline__ static uint64_t pack(int32_t k, int32_t r) {
    return ((uint64_t)(uint32_t)k << 32) | (uint32_t)r;
  }
  __device__ __forceinline__ static bool insert(void* arena, uint64_t b, int32_t k, int32_t r) {
    unsigned long long* p = reinterpret_cast<unsigned long long*>(arena) + b * 4;
    const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
    const ulonglong2 x = __ldcg(q), y = __ldcg(q + 1);
    uint64_t s[4] = {x.x, x.y, y.x, y.y};
    const uint64_t v = pack(k, r);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (s[j] == kEmpty && atomicCAS(p + j, kEmpty, v) == kEmpty) return true;
    }
    return false;
  }
  // matches of key k in bucket b (bits), and whether the bucket has an EMPTY slot
  __device__ __forceinline__ static uint32_t probe(const void* arena, uint64_t b, int32_t k, bool& has_empty,
                                                   int32_t (&rid)[4]) {
    uint64_t s[4];
    load_bucket_cg(arena, b, s);
    uint32_t m = 0;
    has_empty = false;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool e = s[j] == kEmpty;
      has_empty |= e;
      if (!e && (uint32_t)(s[j] >> 32) == (uint32_t)k) m |= 1u << j;
      rid[j] = (int32_t)(uint32_t)s[j];
    }
    return m;
  }
};

template <>
struct BTable<int64_t> {  // 2 x {key, rid} per bucket
  static constexpr int kSlots = 2;
  __device__ __forceinline__ static bool insert(void* arena, uint64_t b, int64_t k, int32_t r) {
    uint64_t* p = reinterpret_cast<uint64_t*>(arena) + b * 4;
    const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
    const ulonglong2 x = __ldcg(q), y = __ldcg(q + 1);
    const uint64_t rid_word[2] = {x.y, y.y};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (rid_word[j] == kEmpty) {
        uint64_t olo, ohi;
        cas128(p + 2 * j, kEmpty, kEmpty, (uint64_t)k, (uint64_t)(uint32_t)r, olo, ohi);
        if (ohi == kEmpty) return true;
      }
    }
    return false;
  }
  __device__ __forceinline__ static uint32_t probe(const void* arena, uint64_t b, int64_t k, bool& has_empty,
                                                   int32_t (&rid)[4]) {
    uint64_t s[4];
    load_bucket_cg(arena, b, s);
    uint32_t m = 0;
    const bool e0 = s[1] == kEmpty, e1 = s[3] == kEmpty;
    has_empty = e0 || e1;
    if (!e0 && (int64_t)s[0] == k) m |= 1u;
    if (!e1 && (int64_t)s[2] == k) m |= 2u;
    rid[0] = (int32_t)s[1];
    rid[1] = (int32_t)s[3];
    rid[2] = rid[3] = 0;
    return m;
  }
};

// The home bucket of a key in its join's table. The batch's tables are built and probed only by
// this file, so int32 keys take a 32-bit mixer: the finalizer of MurmurHash3 (Austin Appleby,
// public domain; a bijection on 32 bits), about a third of the 64-bit mixer's instructions.
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

template <typename K>
__device__ __forceinline__ uint64_t bhome(const BJoin& J, K k) {
  if constexpr (sizeof(K) == 4) return J.log2_nb ? (fmix32((uint32_t)k) >> (32 - J.log2_nb)) : 0;
  else return J.log2_nb ? (mix64(key_u64<K>(k)) >> (64 - J.log2_nb)) : 0;
}

// ---- work items ---------------------------------------------------------------------------------
template <typename K>
__device__ void build_tile(const BatchDev& P, const BJoin& J, int32_t tile) {
  const int64_t lo = (int64_t)tile * P.tile_rows;
  const int64_t hi = min((int64_t)J.nb, lo + P.tile_rows);
  const uint64_t mask = (1ull << J.log2_nb) - 1;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (!bit_valid(J.bvalid, J.bvoff, i)) continue;
    const K k = load_key<K>(J.bkey, i);
    uint64_t b = bhome<K>(J, k);
    bool done = false;
    for (uint64_t step = 0; step <= mask && !done; ++step) {
      done = BTable<K>::insert(P.arena, J.bucket_off + b, k, (int32_t)i);
      b = (b + 1) & mask;
    }
    if (!done) atomicOr(P.error, 2);  // a join's table ran out of slots (cannot happen at LF < 1)
  }
}

template <typename K, int G>
__device__ void probe_tile(const BatchDev& P, const BJoin& J, int32_t join, int32_t tile) {
  constexpr int S = BTable<K>::kSlots;
  const int lane = threadIdx.x & 31;
  const int glane = lane % G;                     // position inside the group
  const int64_t lo = (int64_t)tile * P.tile_rows;
  const int64_t hi = min(J.np, lo + P.tile_rows);
  const uint64_t mask = (1ull << J.log2_nb) - 1;
  const int keys_per_pass = blockDim.x / G;
  const unsigned gmask = (G == 32) ? kFullMask : (((1u << G) - 1) << (lane - glane));
  for (int64_t base = lo; base < hi; base += keys_per_pass) {
    const int64_t i = base + threadIdx.x / G;
    bool live = i < hi && bit_valid(J.pvalid, J.pvoff, i);
    const K k = live ? load_key<K>(J.pkey, i) : (K)0;
    uint64_t b0 = live ? bhome<K>(J, k) : 0;
    for (uint64_t step = 0; __any_sync(kFullMask, live); step += G) {
      uint32_t m = 0;
      bool has_empty = false;
      int32_t rid[4];
      if (live) m = BTable<K>::probe(P.arena, J.bucket_off + ((b0 + glane) & mask), k, has_empty, rid);
      // the group stops at its first bucket with an EMPTY slot; later buckets do not count
      const unsigned eb = __ballot_sync(kFullMask, live && has_empty) & gmask;
      const int stop = eb ? (__ffs(eb) - 1) - (lane - glane) : G;
      if (!live || glane > stop) m = 0;
      const uint32_t cnt = __popc(m);
      const unsigned long long pos0 = warp_reserve(P.counts + join, cnt);
      uint32_t r = 0;
#pragma unroll
      for (int j = 0; j < S; ++j) {
        if (!(m >> j & 1u)) continue;
        const int64_t p = (int64_t)pos0 + r++;
        if (p >= J.capacity) continue;
        if (J.out_prid) J.out_prid[p] = (int32_t)i;
        if (J.out_brid) J.out_brid[p] = rid[j];
        if (J.ppay.data) {
          store_elem(J.out_ppay.data, p, J.ppay.width, load_elem(J.ppay.data, i, J.ppay.width));
          if (J.ppay.valid && bit_valid(J.ppay.valid, J.ppay.voff, i)) set_out_bit(J.out_ppay.valid, p);
        }
        if (J.bpay.data) {
          store_elem(J.out_bpay.data, p, J.bpay.width, load_elem(J.bpay.data, rid[j], J.bpay.width));
          if (J.bpay.valid && bit_valid(J.bpay.valid, J.bpay.voff, rid[j])) set_out_bit(J.out_bpay.valid, p);
        }
      }
      if (eb || step + G > mask) live = false;  // group finished: stop reached or table scanned
      b0 += G;
    }
  }
}

// Group width 1: each lane keeps kBatchR probe rows in flight (rows base + 32 j + lane, so every
// key load is one coalesced warp access). On 4,096 joins with the staged write-out: two rows per
// lane (4 CTAs of 256 per SM, 64 registers) 99.6 ms; one row (6 or 8 CTAs) 131.6 / 141.3 ms; three
// rows (3 CTAs) 123.6 ms; four rows (2 CTAs) 139.2 ms.
// A step probes each row's home bucket. A row stops at its first bucket with an EMPTY slot (its
// matches there still count) or once the whole table has been scanned. The few rows whose home
// bucket is full (about 7 % at load factor 0.35) go to a per-warp list in shared memory with their
// next bucket, and the warp probes that list 32 rows at a time, with every lane busy, whenever it
// holds 32 rows, and at the end of the tile. Walking them in the step instead cost the whole warp
// one more pass over the step's code for a handful of lanes, in almost every step.
// When every row has at most one match in a pass (unique build keys), all loads a match needs are
// in flight before the warp reserves output: the probe payload loads with the key, the build
// payload (by row id) right after the bucket match; hit lanes are ranked with ballots. Otherwise
// (duplicates in one bucket) positions follow (lane, row, slot) order.
constexpr int kBatchR = 2;

// SH = 4 or 8: every join of the plan gathers one probe and one build payload of SH bytes without
// NULLs and writes both row ids (typed loads and stores, no per-store checks); 0: read from J.
template <int SH>
__device__ __forceinline__ uint64_t pay_load(const PayloadIn& in, int64_t i) {
  if constexpr (SH == 8) return __ldg(static_cast<const unsigned long long*>(in.data) + i);
  else if constexpr (SH == 4) return __ldg(static_cast<const unsigned int*>(in.data) + i);
  else return load_elem(in.data, i, in.width);
}

// Staged write-out (compile-time shapes, SH = 4 or 8): all warps probing one join reserve output on
// the join's one counter, and with one atomicAdd per 64-row step that address serialises the
// launch (spreading it over 32 counters, in a timing-only copy, took the 4,096-join sweep from 120
// to 99 ms). So a warp collects its matches in a shared-memory area of kStage rows (probe row id,
// build row id, both payloads) and reserves output once per ~kStage - 64 matches, then writes the
// area out in contiguous runs. No holes: a flush reserves exactly the rows it holds.
constexpr int kStage = 256;
// per-warp list of rows that go on to their next bucket: {probe row, bucket}; it holds fewer than
// 32 rows between passes, plus at most 32 * kBatchR added by one step
constexpr int kMore = 128;

template <int SH>
constexpr int stage_row_bytes() { return 8 + 2 * SH; }

// dynamic shared memory of a CTA of `block` threads for output shape `sh` (group width 1)
static inline size_t stage_smem(int sh, int block) {
  return (size_t)(block / 32) * ((sh ? (size_t)kStage * (8 + 2 * sh) : 0) + (size_t)kMore * 8);
}

template <typename K, int SH>
__device__ void probe_tile_r(const BatchDev& P, const BJoin& J, int32_t join, int32_t tile) {
  constexpr int S = BTable<K>::kSlots;
  constexpr int R = kBatchR;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int nwarps = blockDim.x >> 5;
  const int64_t lo = (int64_t)tile * P.tile_rows;
  const int64_t hi = min(J.np, lo + P.tile_rows);
  const uint64_t mask = (1ull << J.log2_nb) - 1;
  const bool has_pp = SH || J.ppay.data != nullptr, has_bp = SH || J.bpay.data != nullptr;
  const int64_t stride = (int64_t)nwarps * 32 * R;
  // this warp's shared memory: [prid | brid | probe payload | build payload] x kStage (SH != 0),
  // then the list of rows that continue: row[kMore] | bucket[kMore]
  extern __shared__ __align__(16) unsigned char s_dyn[];
  using PW = std::conditional_t<SH == 8, unsigned long long, unsigned int>;
  unsigned char* wbase = s_dyn + (size_t)(threadIdx.x >> 5) * ((SH ? (size_t)kStage * stage_row_bytes<SH>() : 0) +
                                                               (size_t)kMore * 8);
  int32_t* st_prid = reinterpret_cast<int32_t*>(wbase);
  int32_t* st_brid = st_prid + kStage;
  PW* st_pp = reinterpret_cast<PW*>(st_brid + kStage);
  PW* st_bp = st_pp + kStage;
  int32_t* more_row = reinterpret_cast<int32_t*>(wbase + (SH ? (size_t)kStage * stage_row_bytes<SH>() : 0));
  uint32_t* more_b = reinterpret_cast<uint32_t*>(more_row + kMore);
  uint32_t fill = 0;  // rows staged (warp-uniform)
  uint32_t n_more = 0;  // rows in the continue list (warp-uniform)
  auto flush = [&]() {
    __syncwarp();
    unsigned long long pos = 0;
    if (lane == 0) pos = atomicAdd(P.counts + join, (unsigned long long)fill);
    pos = __shfl_sync(kFullMask, pos, 0);
    for (uint32_t e = lane; e < fill; e += 32) {
      const int64_t p = (int64_t)(pos + e);
      if (p >= J.capacity) break;
      __stcs(J.out_prid + p, st_prid[e]);
      __stcs(J.out_brid + p, st_brid[e]);
      __stcs(static_cast<PW*>(J.out_ppay.data) + p, st_pp[e]);
      __stcs(static_cast<PW*>(J.out_bpay.data) + p, st_bp[e]);
    }
    __syncwarp();
    fill = 0;
  };
  // write one match: output position p, probe row i, build row id brow, payloads
  auto put = [&](int64_t p, int64_t i, int32_t brow, uint64_t pval, uint64_t bval) {
    if (p >= J.capacity) return;
    if constexpr (SH != 0) {
      __stcs(J.out_prid + p, (int32_t)i);
      __stcs(J.out_brid + p, brow);
      __stcs(static_cast<PW*>(J.out_ppay.data) + p, (PW)pval);
      __stcs(static_cast<PW*>(J.out_bpay.data) + p, (PW)bval);
      return;
    }
    if (J.out_prid) J.out_prid[p] = (int32_t)i;
    if (J.out_brid) J.out_brid[p] = brow;
    if (has_pp) {
      store_elem(J.out_ppay.data, p, J.ppay.width, pval);
      if (J.ppay.valid && bit_valid(J.ppay.valid, J.ppay.voff, i)) set_out_bit(J.out_ppay.valid, p);
    }
    if (has_bp) {
      store_elem(J.out_bpay.data, p, J.bpay.width, bval);
      if (J.bpay.valid && bit_valid(J.bpay.valid, J.bpay.voff, brow)) set_out_bit(J.out_bpay.valid, p);
    }
  };
  // the matches m[j] (slot bits, row ids rid[j]) of probe rows row[j], j < NR, with probe payloads pv
  auto emit = [&](const uint32_t (&m)[R], const int32_t (&rid)[R][4], const int64_t (&row)[R],
                  const uint64_t (&pv)[R]) {
    bool single = true;  // at most one match per row (always so for unique builds)
#pragma unroll
    for (int j = 0; j < R; ++j) single &= (m[j] & (m[j] - 1u)) == 0;
    if (__all_sync(kFullMask, single)) {
      int32_t brow[R];
      uint64_t bv[R];
      unsigned bal[R];
      uint32_t tot = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        brow[j] = 0;
#pragma unroll
        for (int q = 0; q < S; ++q) brow[j] = (m[j] >> q & 1u) ? rid[j][q] : brow[j];
        bv[j] = m[j] && has_bp ? pay_load<SH>(J.bpay, brow[j]) : 0;
        bal[j] = __ballot_sync(kFullMask, m[j] != 0);
        tot += __popc(bal[j]);
      }
      if (tot == 0) return;
      if constexpr (SH != 0) {
        if (fill + tot > (uint32_t)kStage) flush();
        uint32_t run = fill;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const uint32_t e = run + __popc(bal[j] & below);
          run += __popc(bal[j]);
          if (!m[j]) continue;
          st_prid[e] = (int32_t)row[j];
          st_brid[e] = brow[j];
          st_pp[e] = (PW)pv[j];
          st_bp[e] = (PW)bv[j];
        }
        fill = run;
        if (fill > (uint32_t)(kStage - 32 * R)) flush();  // the next pass could not fit
      } else {
        unsigned long long pos = 0;
        if (lane == 0) pos = atomicAdd(P.counts + join, (unsigned long long)tot);
        pos = __shfl_sync(kFullMask, pos, 0);
#pragma unroll
        for (int j = 0; j < R; ++j) {
          if (m[j]) put((int64_t)(pos + __popc(bal[j] & below)), row[j], brow[j], pv[j], bv[j]);
          pos += __popc(bal[j]);
        }
      }
    } else {
      // duplicates in one bucket: lane-major positions
      uint32_t cnt = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) cnt += __popc(m[j]);
      const unsigned long long pos0 = warp_reserve(P.counts + join, cnt);
      uint32_t r = 0;
#pragma unroll
      for (int j = 0; j < R; ++j)
#pragma unroll
        for (int q = 0; q < S; ++q)
          if (m[j] >> q & 1u)
            put((int64_t)pos0 + r++, row[j], rid[j][q], pv[j], has_bp ? pay_load<SH>(J.bpay, rid[j][q]) : 0);
    }
  };
  // rows whose bucket had no EMPTY slot (cont[j]) join the list with their next bucket
  auto keep_on = [&](const bool (&cont)[R], const int64_t (&row)[R], const uint64_t (&b)[R]) {
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const unsigned bal = __ballot_sync(kFullMask, cont[j]);
      if (cont[j]) {
        const uint32_t e = n_more + __popc(bal & below);
        more_row[e] = (int32_t)row[j];
        more_b[e] = (uint32_t)((b[j] + 1) & mask);
      }
      n_more += __popc(bal);
    }
    __syncwarp();
  };
  // one pass over the last `take` (<= 32) rows of the list, one row per lane
  auto walk_more = [&](uint32_t take) {
    const bool mine = (uint32_t)lane < take;
    int64_t row[R] = {};
    uint64_t b[R] = {}, pv[R] = {};
    uint32_t m[R] = {};
    int32_t rid[R][4] = {};
    bool cont[R] = {};
    if (mine) {
      row[0] = more_row[n_more - take + lane];
      b[0] = more_b[n_more - take + lane];
    }
    __syncwarp();
    n_more -= take;
    if (mine) {
      const K k = load_key<K>(J.pkey, row[0]);
      pv[0] = has_pp ? pay_load<SH>(J.ppay, row[0]) : 0;
      bool has_empty = false;
      m[0] = BTable<K>::probe(P.arena, J.bucket_off + b[0], k, has_empty, rid[0]);
      // buckets probed before this one: (b - home) mod the table size; the whole table is scanned
      // once it reaches the last bucket
      const uint64_t before = (b[0] - bhome<K>(J, k)) & mask;
      cont[0] = !has_empty && before < mask;
    }
    emit(m, rid, row, pv);
    keep_on(cont, row, b);
  };
  // the keys and probe payloads of the warp's next step load while this step probes
  K kn[R];
  uint64_t pn[R];
  auto load_step = [&](int64_t sb) {
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int64_t i = sb + 32 * j + lane;
      kn[j] = i < hi ? load_key<K>(J.pkey, i) : (K)0;
      pn[j] = i < hi && has_pp ? pay_load<SH>(J.ppay, i) : 0;
    }
  };
  load_step(lo + (int64_t)(threadIdx.x >> 5) * 32 * R);
  for (int64_t base = lo + (int64_t)(threadIdx.x >> 5) * 32 * R; base < hi; base += stride) {
    K k[R];
    uint64_t b[R], pv[R];
    int64_t row[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      k[j] = kn[j];
      pv[j] = pn[j];
    }
    if (base + stride < hi) load_step(base + stride);
    uint32_t m[R];
    int32_t rid[R][4];
    bool cont[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      row[j] = base + 32 * j + lane;
      const bool live = row[j] < hi && bit_valid(J.pvalid, J.pvoff, row[j]);
      b[j] = live ? bhome<K>(J, k[j]) : 0;
      m[j] = 0;
      cont[j] = false;
      if (!live) continue;
      bool has_empty = false;
      m[j] = BTable<K>::probe(P.arena, J.bucket_off + b[j], k[j], has_empty, rid[j]);
      cont[j] = !has_empty && mask > 0;
    }
    emit(m, rid, row, pv);
    keep_on(cont, row, b);
    while (n_more >= 32) walk_more(32);
  }
  while (n_more > 0) walk_more(n_more < 32 ? n_more : 32);
  if constexpr (SH != 0) {
    if (fill) flush();
  }
}

__device__ __forceinline__ void wait_built(const BatchDev& P, int32_t join, int32_t need) {
  if (threadIdx.x == 0) {
    if (!wait_counter_at_least(P.built + join, (unsigned)need, kWaitLimit)) atomicOr(P.error, 1);
    __threadfence();
  }
  __syncthreads();
}

// 64 registers at most: four CTAs of 256 threads per SM (the shape-specialised probe needs 66
// otherwise, which leaves three)
template <typename K, int G, int SH>
__global__ void __launch_bounds__(512, 2) batch_persistent_kernel(BatchDev P) {
  __shared__ long long s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(P.queue, 1ull);
    __syncthreads();
    const long long it = s_item;
    __syncthreads();
    if (it >= P.n_items) break;
    const BItem item = P.items[it];
    const BJoin J = P.joins[item.join];
    if (it < P.n_build_items) {
      build_tile<K>(P, J, item.tile);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(P.built + item.join, 1u);
      }
    } else {
      wait_built(P, item.join, J.build_tiles);
      if constexpr (G == 1) probe_tile_r<K, SH>(P, J, item.join, item.tile);
      else probe_tile<K, G>(P, J, item.join, item.tile);
    }
  }
}

// One join per launch (the comparison point): build or probe all tiles of join `j`.
template <typename K>
__global__ void batch_build_one_kernel(BatchDev P, int32_t j) {
  const BJoin J = P.joins[j];
  for (int32_t t = blockIdx.x; t < J.build_tiles; t += gridDim.x) build_tile<K>(P, J, t);
}
template <typename K, int G, int SH>
__global__ void batch_probe_one_kernel(BatchDev P, int32_t j, int32_t probe_tiles) {
  const BJoin J = P.joins[j];
  for (int32_t t = blockIdx.x; t < probe_tiles; t += gridDim.x) {
    if constexpr (G == 1) probe_tile_r<K, SH>(P, J, j, t);
    else probe_tile<K, G>(P, J, j, t);
  }
}

}  // namespace sj

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
struct sj_batch_plan {
  int device = 0;
  sj::Allocator alloc;
  sj_batch_params params{};
  int32_t key_type = SJ_INT32;
  int32_t n_joins = 0;
  int32_t shape = 0;  // compile-time output shape of the probe (4 / 8: see probe_tile_r), or 0
  std::vector<sj::BJoin> host_joins;
  std::vector<int32_t> probe_tiles;
  sj::BatchDev dev{};
  void* joins_mem = nullptr;
  size_t joins_bytes = 0;
  void* items_mem = nullptr;
  size_t items_bytes = 0;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  void* counters = nullptr;  // queue | built[n] | counts[n] | error
  size_t counters_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

namespace sj {

static size_t a256b(size_t b) { return (std::max<size_t>(b, 16) + 255) & ~(size_t)255; }

static sj_status batch_resolve(const sj_batch_params* in, sj_batch_params& p) {
  std::memset(&p, 0, sizeof(p));
  p.block_size = 256;
  p.group_width = 1;
  p.load_factor = 0.5f;
  p.tile_rows = 4096;
  p.ctas_per_sm = 4;
  if (in) {
    if (in->block_size) p.block_size = in->block_size;
    if (in->group_width) p.group_width = in->group_width;
    if (in->load_factor > 0.0f) p.load_factor = in->load_factor;
    if (in->tile_rows) p.tile_rows = in->tile_rows;
    if (in->ctas_per_sm) p.ctas_per_sm = in->ctas_per_sm;
  }
  if (p.block_size != 128 && p.block_size != 256 && p.block_size != 512)
    return set_error(SJ_ERR_INVALID, "batch block_size must be 128, 256 or 512");
  if (p.group_width != 1 && p.group_width != 2 && p.group_width != 4 && p.group_width != 8)
    return set_error(SJ_ERR_INVALID, "batch group_width must be 1, 2, 4 or 8");
  if (!(p.load_factor > 0.0f && p.load_factor < 1.0f)) return set_error(SJ_ERR_INVALID, "load_factor must be in (0, 1)");
  if (p.tile_rows < 64 || p.tile_rows > (1 << 20)) return set_error(SJ_ERR_INVALID, "tile_rows must be in [64, 2^20]");
  if (p.ctas_per_sm < 1 || p.ctas_per_sm > 16) return set_error(SJ_ERR_INVALID, "ctas_per_sm must be in [1, 16]");
  return SJ_OK;
}

// key type x group width x output shape (the compile-time shape only with group width 1)
template <typename F>
static void dispatch_kg(int32_t key_type, int g, int shape, F&& f) {
  using I1 = std::integral_constant<int, 1>;
  auto go = [&](auto k) {
    switch (g) {
      case 1:
        if (shape == 8) f(k, I1{}, std::integral_constant<int, 8>{});
        else if (shape == 4) f(k, I1{}, std::integral_constant<int, 4>{});
        else f(k, I1{}, std::integral_constant<int, 0>{});
        break;
      case 2: f(k, std::integral_constant<int, 2>{}, std::integral_constant<int, 0>{}); break;
      case 4: f(k, std::integral_constant<int, 4>{}, std::integral_constant<int, 0>{}); break;
      default: f(k, std::integral_constant<int, 8>{}, std::integral_constant<int, 0>{}); break;
    }
  };
  if (key_type == SJ_INT32) go(int32_t{});
  else go(int64_t{});
}

static sj_status reset_batch(sj_batch_plan* P, cudaStream_t s) {
  SJ_CUDA_TRY(cudaMemsetAsync(P->arena, 0xff, P->arena_bytes, s));
  SJ_CUDA_TRY(cudaMemsetAsync(P->counters, 0, P->counters_bytes, s));
  return SJ_OK;
}

static int resident_ctas(sj_batch_plan* P) {
  int per_sm = 0;
  const int block = P->params.block_size;
  dispatch_kg(P->key_type, P->params.group_width, P->shape, [&](auto k, auto g, auto sh) {
    auto* kern = batch_persistent_kernel<decltype(k), decltype(g)::value, decltype(sh)::value>;
    const size_t smem = (decltype(g)::value == 1 ? stage_smem(decltype(sh)::value, block) : 0);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem);
  });
  per_sm = std::max(1, std::min(per_sm, P->params.ctas_per_sm));
  return per_sm * sm_count(P->device);
}

}  // namespace sj

using namespace sj;

extern "C" {

SJ_EXPORT sj_status sj_batch_plan_create(const sj_batch_join* joins, int32_t n, const sj_batch_params* params,
                                         const sj_alloc* user_alloc, sj_stream_t stream, sj_batch_plan** out) {
  clear_error();
  if (!out) return set_error(SJ_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (n < 0 || (n > 0 && !joins)) return set_error(SJ_ERR_INVALID, "joins array is NULL");
  sj_batch_params p;
  SJ_TRY(batch_resolve(params, p));
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  sj_batch_plan* P = new sj_batch_plan();
  P->alloc = Allocator(user_alloc);
  cudaGetDevice(&P->device);
  P->params = p;
  P->n_joins = n;
  P->key_type = n > 0 ? joins[0].build_key.type : SJ_INT32;
  auto fail = [&](sj_status st) {
    sj_batch_plan_destroy(P, stream);
    return st;
  };
  std::vector<BItem> build_items, probe_items;
  int64_t buckets = 0;
  const int spb = P->key_type == SJ_INT32 ? 4 : 2;
  for (int32_t j = 0; j < n; ++j) {
    const sj_batch_join& q = joins[j];
    if (sj_status e = validate_column(&q.build_key, "batch build key", true)) return fail(e);
    if (sj_status e = validate_column(&q.probe_key, "batch probe key", true)) return fail(e);
    if (q.build_key.type != P->key_type || q.probe_key.type != P->key_type)
      return fail(set_error(SJ_ERR_INVALID, "every join of a batch uses one key type"));
    if (q.build_key.num_rows > INT32_MAX || q.probe_key.num_rows > INT32_MAX)
      return fail(set_error(SJ_ERR_INVALID, "a batched join exceeds the int32 row-id range"));
    if (q.capacity < 0) return fail(set_error(SJ_ERR_INVALID, "capacity must be >= 0"));
    BJoin J{};
    J.bkey = q.build_key.data;
    J.bvalid = q.build_key.validity;
    J.bvoff = q.build_key.validity_offset;
    J.nb = (int32_t)q.build_key.num_rows;
    J.pkey = q.probe_key.data;
    J.pvalid = q.probe_key.validity;
    J.pvoff = q.probe_key.validity_offset;
    J.np = q.probe_key.num_rows;
    auto payload = [&](const sj_column& c, const sj_mut_column& o, int64_t rows, PayloadIn& in, PayloadOut& po,
                       const char* what) -> sj_status {
      if (!c.data) return SJ_OK;
      SJ_TRY(validate_column(&c, what, false));
      if (c.num_rows != rows) return set_error(SJ_ERR_INVALID, std::string(what) + " row count differs from its keys");
      if (o.type != c.type || (q.capacity > 0 && !o.data))
        return set_error(SJ_ERR_INVALID, std::string(what) + " output missing or of another type");
      if (c.validity && q.capacity > 0 && !o.validity)
        return set_error(SJ_ERR_INVALID, std::string(what) + " has NULLs but its output has no validity");
      in = column_payload(c.data, c.validity, c.validity_offset, type_width(c.type));
      po = PayloadOut{o.data, c.validity ? o.validity : nullptr};
      return SJ_OK;
    };
    if (sj_status e = payload(q.build_payload, q.out_build_payload, J.nb, J.bpay, J.out_bpay, "batch build payload"))
      return fail(e);
    if (sj_status e = payload(q.probe_payload, q.out_probe_payload, J.np, J.ppay, J.out_ppay, "batch probe payload"))
      return fail(e);
    J.out_prid = q.out_probe_rid;
    J.out_brid = q.out_build_rid;
    J.capacity = q.capacity;
    const double slots = std::max(1.0, (double)std::max(J.nb, 1) / p.load_factor);
    int l = 0;
    while ((double)(1ll << l) * spb < slots) ++l;
    J.log2_nb = l;
    J.bucket_off = buckets;
    buckets += 1ll << l;
    J.build_tiles = (int32_t)((J.nb + p.tile_rows - 1) / p.tile_rows);
    const int32_t pt = (int32_t)((J.np + p.tile_rows - 1) / p.tile_rows);
    for (int32_t t = 0; t < J.build_tiles; ++t) build_items.push_back(BItem{j, t});
    for (int32_t t = 0; t < pt; ++t) probe_items.push_back(BItem{j, t});
    P->probe_tiles.push_back(pt);
    P->host_joins.push_back(J);
  }
  // one compile-time output shape when every join gathers both payloads of one width (4 or 8 bytes)
  // without NULLs and writes both row ids
  int shape = -1;
  for (const BJoin& J : P->host_joins) {
    const int w = J.ppay.data && J.bpay.data && J.ppay.width == J.bpay.width && !J.ppay.valid && !J.bpay.valid &&
                          J.out_prid && J.out_brid
                      ? J.ppay.width
                      : 0;
    shape = shape < 0 ? w : (shape == w ? w : 0);
  }
  P->shape = shape == 4 || shape == 8 ? shape : 0;
  // if any join's clear is needed, memset covers all slices; the layout is fixed by the plan
  P->arena_bytes = (size_t)std::max<int64_t>(buckets, 1) * kBucketBytes;
  P->joins_bytes = a256b(sizeof(BJoin) * std::max(n, 1));
  std::vector<BItem> items = build_items;
  items.insert(items.end(), probe_items.begin(), probe_items.end());
  P->items_bytes = a256b(sizeof(BItem) * std::max<size_t>(items.size(), 1));
  P->counters_bytes = a256b(8 + 4 * (size_t)std::max(n, 1) + 8) + a256b(8 * (size_t)std::max(n, 1)) + 256;
  if (sj_status e = P->alloc.allocate(&P->arena, P->arena_bytes, s)) return fail(e);
  if (sj_status e = P->alloc.allocate(&P->joins_mem, P->joins_bytes, s)) return fail(e);
  if (sj_status e = P->alloc.allocate(&P->items_mem, P->items_bytes, s)) return fail(e);
  if (sj_status e = P->alloc.allocate(&P->counters, P->counters_bytes, s)) return fail(e);
  if (n > 0)
    SJ_CUDA_TRY(cudaMemcpyAsync(P->joins_mem, P->host_joins.data(), sizeof(BJoin) * n, cudaMemcpyHostToDevice, s));
  if (!items.empty())
    SJ_CUDA_TRY(cudaMemcpyAsync(P->items_mem, items.data(), sizeof(BItem) * items.size(), cudaMemcpyHostToDevice, s));
  // the host vectors are read by the copies: wait before they go out of scope
  SJ_CUDA_TRY(cudaStreamSynchronize(s));
  char* c = static_cast<char*>(P->counters);
  BatchDev& D = P->dev;
  D.joins = static_cast<const BJoin*>(P->joins_mem);
  D.items = static_cast<const BItem*>(P->items_mem);
  D.n_items = (int64_t)items.size();
  D.n_build_items = (int64_t)build_items.size();
  D.arena = P->arena;
  D.tile_rows = p.tile_rows;
  D.n_joins = n;
  D.queue = reinterpret_cast<unsigned long long*>(c);
  D.built = reinterpret_cast<unsigned int*>(c + 8);
  D.counts = reinterpret_cast<unsigned long long*>(c + a256b(8 + 4 * (size_t)std::max(n, 1) + 8));
  D.error = reinterpret_cast<int32_t*>(c + a256b(8 + 4 * (size_t)std::max(n, 1) + 8) + a256b(8 * (size_t)std::max(n, 1)));
  *out = P;
  return SJ_OK;
}

SJ_EXPORT sj_status sj_batch_plan_launch(sj_batch_plan* P, sj_stream_t stream) {
  clear_error();
  if (!P) return set_error(SJ_ERR_INVALID, "plan is NULL");
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  SJ_TRY(reset_batch(P, s));
  if (P->dev.n_items == 0) return SJ_OK;
  const int grid = resident_ctas(P);
  KernelTimer timer("batch_persistent", s);
  dispatch_kg(P->key_type, P->params.group_width, P->shape, [&](auto k, auto g, auto sh) {
    const size_t smem = (decltype(g)::value == 1 ? stage_smem(decltype(sh)::value, P->params.block_size) : 0);
    batch_persistent_kernel<decltype(k), decltype(g)::value, decltype(sh)::value>
        <<<grid, P->params.block_size, smem, s>>>(P->dev);
  });
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

SJ_EXPORT sj_status sj_batch_plan_replay(sj_batch_plan* P, sj_stream_t stream) {
  clear_error();
  if (!P) return set_error(SJ_ERR_INVALID, "plan is NULL");
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (s == nullptr) return set_error(SJ_ERR_INVALID, "graph replay needs a non-default stream");
  if (!P->graph_exec) {
    SJ_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const bool t = timing_enabled();
    if (t) sj_timing_enable(0);  // no timing events inside the graph
    sj_status st = sj_batch_plan_launch(P, stream);
    if (t) sj_timing_enable(1);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != SJ_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return set_error(SJ_ERR_DEVICE, std::string("graph capture: ") + cudaGetErrorString(e));
    P->graph = g;
    SJ_CUDA_TRY(cudaGraphInstantiate(&P->graph_exec, P->graph, 0));
  }
  KernelTimer timer("batch_graph", s);
  SJ_CUDA_TRY(cudaGraphLaunch(P->graph_exec, s));
  return SJ_OK;
}

SJ_EXPORT sj_status sj_batch_plan_launch_per_join(sj_batch_plan* P, sj_stream_t stream) {
  clear_error();
  if (!P) return set_error(SJ_ERR_INVALID, "plan is NULL");
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  SJ_TRY(reset_batch(P, s));
  const int block = P->params.block_size;
  const int cap = sm_count(P->device) * P->params.ctas_per_sm;
  dispatch_kg(P->key_type, P->params.group_width, P->shape, [&](auto k, auto g, auto sh) {
    const size_t smem = (decltype(g)::value == 1 ? stage_smem(decltype(sh)::value, block) : 0);
    cudaFuncSetAttribute(batch_probe_one_kernel<decltype(k), decltype(g)::value, decltype(sh)::value>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  KernelTimer timer("batch_per_join", s);
  for (int32_t j = 0; j < P->n_joins; ++j) {
    const BJoin& J = P->host_joins[j];
    const int gb = std::max(1, std::min(J.build_tiles, cap));
    const int gp = std::max(1, std::min(P->probe_tiles[j], cap));
    dispatch_kg(P->key_type, P->params.group_width, P->shape, [&](auto k, auto g, auto sh) {
      using K = decltype(k);
      if (J.build_tiles > 0) batch_build_one_kernel<K><<<gb, block, 0, s>>>(P->dev, j);
      if (P->probe_tiles[j] > 0) {
        auto* kern = batch_probe_one_kernel<K, decltype(g)::value, decltype(sh)::value>;
        const size_t smem = (decltype(g)::value == 1 ? stage_smem(decltype(sh)::value, block) : 0);
        kern<<<gp, block, smem, s>>>(P->dev, j, P->probe_tiles[j]);
      }
    });
  }
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

SJ_EXPORT sj_status sj_batch_plan_counts(const sj_batch_plan* P, int64_t* d_counts, int32_t* d_error,
                                         sj_stream_t stream) {
  clear_error();
  if (!P) return set_error(SJ_ERR_INVALID, "plan is NULL");
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (d_counts && P->n_joins > 0)
    SJ_CUDA_TRY(cudaMemcpyAsync(d_counts, P->dev.counts, 8 * (size_t)P->n_joins, cudaMemcpyDeviceToDevice, s));
  if (d_error) SJ_CUDA_TRY(cudaMemcpyAsync(d_error, P->dev.error, 4, cudaMemcpyDeviceToDevice, s));
  return SJ_OK;
}

SJ_EXPORT sj_status sj_batch_plan_destroy(sj_batch_plan* P, sj_stream_t stream) {
  if (!P) return SJ_OK;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (P->graph_exec) cudaGraphExecDestroy(P->graph_exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  P->alloc.release(P->arena, P->arena_bytes, s);
  P->alloc.release(P->joins_mem, P->joins_bytes, s);
  P->alloc.release(P->items_mem, P->items_bytes, s);
  P->alloc.release(P->counters, P->counters_bytes, s);
  delete P;
  return SJ_OK;
}

}  // extern "C"
