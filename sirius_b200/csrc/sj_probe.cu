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
// DISTINCT: probe + gather in one pass
// ------------------------------------------------------------------------------------------------
template <typename K, bool WIDE, bool VEC, bool COUNT_ONLY>
__global__ void __launch_bounds__(256) probe_distinct_kernel(TableDev t, const K* __restrict__ keys,
                                                             const uint32_t* __restrict__ kv, int64_t kvoff,
                                                             int64_t n, GatherArgs g) {
  using Ops = SlotOps<WIDE>;
  const int lane = threadIdx.x & 31;
  const int64_t per_cta = (int64_t)blockDim.x * KPT;
  const int64_t tiles = (n + per_cta - 1) / per_cta;
  unsigned long long counted = 0;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row0 = tile * per_cta + (int64_t)threadIdx.x * KPT;
    K k[KPT];
    load_keys<K>(keys, row0, n, VEC, k);
    uint32_t act = live_rows<K>(t, k, row0, n, kv, kvoff);
    uint32_t b[KPT];
    uint64_t kn[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      b[j] = home_bucket(t, key_u64<K>(k[j]));
      kn[j] = (uint64_t)(long long)k[j] - (uint64_t)t.kmin;
    }
    int32_t rid[KPT];
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
          if (!done && Ops::match(bk[j], q, kn[j], key_u64<K>(k[j]), t.rbits)) {
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
    const unsigned long long pos0 = warp_reserve(g.d_count, cnt);
    int64_t pos[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) pos[j] = (int64_t)pos0 + __popc(hit & ((1u << j) - 1));
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      if ((hit >> j & 1u) && pos[j] < g.capacity) {
        if (g.out_prid) __stcs(g.out_prid + pos[j], (int)(row0 + j));
        if (g.out_brid) __stcs(g.out_brid + pos[j], (int)rid[j]);
      }
    }
    for (int c = 0; c < g.n_pin; ++c) {
      const PayloadIn in = g.pin[c];
      const PayloadOut o = g.pout[c];
      uint64_t v[KPT];
#pragma unroll
      for (int j = 0; j < KPT; ++j)
        if (hit >> j & 1u) v[j] = load_elem_cs(in.data, row0 + j, in.width);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        if ((hit >> j & 1u) && pos[j] < g.capacity) {
          store_elem_cs(o.data, pos[j], in.width, v[j]);
          if (in.valid && bit_valid(in.valid, in.voff, row0 + j)) set_out_bit(o.valid, pos[j]);
        }
      }
    }
    for (int c = 0; c < g.n_bin; ++c) {
      const PayloadIn in = g.bin[c];
      const PayloadOut o = g.bout[c];
      uint64_t v[KPT];
#pragma unroll
      for (int j = 0; j < KPT; ++j)
        if (hit >> j & 1u) v[j] = load_elem(in.data, rid[j], in.width);
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        if ((hit >> j & 1u) && pos[j] < g.capacity) {
          store_elem_cs(o.data, pos[j], in.width, v[j]);
          if (in.valid && bit_valid(in.valid, in.voff, rid[j])) set_out_bit(o.valid, pos[j]);
        }
      }
    }
  }
  if (COUNT_ONLY) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) counted += __shfl_down_sync(kFullMask, counted, d);
    if (lane == 0 && counted) atomicAdd(g.d_count, counted);
  }
}

// ------------------------------------------------------------------------------------------------
// GROUPED pass A: find each probe row's group; compact (row, start, size); sum the output size.
// ------------------------------------------------------------------------------------------------
template <typename K, bool WIDE, bool VEC, bool COMPACT>
__global__ void __launch_bounds__(256) grouped_match_kernel(TableDev t, const K* __restrict__ keys,
                                                            const uint32_t* __restrict__ kv, int64_t kvoff,
                                                            int64_t n, int32_t* m_row, int32_t* m_start,
                                                            int32_t* m_cnt, unsigned long long* d_nent,
                                                            unsigned long long* d_total) {
  using Ops = SlotOps<WIDE>;
  const int lane = threadIdx.x & 31;
  const int64_t per_cta = (int64_t)blockDim.x * KPT;
  const int64_t tiles = (n + per_cta - 1) / per_cta;
  unsigned long long total = 0;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row0 = tile * per_cta + (int64_t)threadIdx.x * KPT;
    K k[KPT];
    load_keys<K>(keys, row0, n, VEC, k);
    uint32_t act = live_rows<K>(t, k, row0, n, kv, kvoff);
    int32_t slot[KPT];
    uint32_t b[KPT];
    uint64_t kn[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      slot[j] = -1;
      b[j] = home_bucket(t, key_u64<K>(k[j]));
      kn[j] = (uint64_t)(long long)k[j] - (uint64_t)t.kmin;
      if (t.null_group >= 0 && row0 + j < n && !bit_valid(kv, kvoff, row0 + j)) slot[j] = t.null_group;
    }
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
          if (!done && Ops::match(bk[j], q, kn[j], key_u64<K>(k[j]), t.rbits)) {
            slot[j] = (int32_t)(b[j] * Ops::kSlots + q);
            done = true;
          }
          done |= Ops::empty(bk[j], q);
        }
        if (done) act &= ~(1u << j);
        else b[j] = next_bucket(b[j], t.segmask);
      }
    }
    int32_t start[KPT], cnt[KPT];
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
      cnt[j] = 0;
      if (slot[j] >= 0) {
        start[j] = __ldg(t.grp_off + slot[j]);
        cnt[j] = __ldg(t.grp_off + slot[j] + 1) - start[j];
        if (cnt[j] > 0) hit |= 1u << j;
        total += (unsigned long long)cnt[j];
      }
    }
    if (COMPACT) {
      const unsigned long long p0 = warp_reserve(d_nent, __popc(hit));
#pragma unroll
      for (int j = 0; j < KPT; ++j) {
        if (hit >> j & 1u) {
          const int64_t p = (int64_t)p0 + __popc(hit & ((1u << j) - 1));
          m_row[p] = (int32_t)(row0 + j);
          m_start[p] = start[j];
          m_cnt[p] = cnt[j];
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
// ------------------------------------------------------------------------------------------------
constexpr int kExpandThreads = 256;
constexpr int kExpandItems = 8;
constexpr int kExpandTile = kExpandThreads * kExpandItems;

__device__ __forceinline__ int64_t upper_index(const int64_t* off, int64_t lo, int64_t hi, int64_t j) {
  // largest e in [lo, hi] with off[e] <= j (off[lo] <= j assumed)
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= j) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kExpandThreads) expand_kernel(const int32_t* __restrict__ m_row,
                                                                const int32_t* __restrict__ m_start,
                                                                const int64_t* __restrict__ m_off,
                                                                const unsigned long long* d_nent,
                                                                const int32_t* __restrict__ grp_rid,
                                                                GatherArgs g) {
  __shared__ int64_t s_off[kExpandTile + 1];
  __shared__ int32_t s_row[kExpandTile + 1];
  __shared__ int32_t s_start[kExpandTile + 1];
  __shared__ int64_t s_e0;
  const int lane = threadIdx.x & 31;
  const int64_t nent = (int64_t)*d_nent;
  if (nent == 0) return;
  const int64_t M = m_off[nent];
  const int64_t cap = M < g.capacity ? M : g.capacity;
  const int64_t ntile = (cap + kExpandTile - 1) / kExpandTile;
  const int64_t per_block = (ntile + gridDim.x - 1) / gridDim.x;
  const int64_t t_lo = (int64_t)blockIdx.x * per_block;
  const int64_t t_hi = t_lo + per_block < ntile ? t_lo + per_block : ntile;
  if (t_lo >= t_hi) return;
  if (threadIdx.x == 0) s_e0 = upper_index(m_off, 0, nent - 1, t_lo * kExpandTile);
  __syncthreads();
  int64_t e0 = s_e0;
  for (int64_t tile = t_lo; tile < t_hi; ++tile) {
    const int64_t j0 = tile * kExpandTile;
    const int64_t j1 = j0 + kExpandTile < cap ? j0 + kExpandTile : cap;
    const int64_t ne = (nent - e0) < (kExpandTile + 1) ? (nent - e0) : (kExpandTile + 1);
    for (int i = threadIdx.x; i < ne; i += kExpandThreads) {
      s_off[i] = m_off[e0 + i];
      s_row[i] = m_row[e0 + i];
      s_start[i] = m_start[e0 + i];
    }
    __syncthreads();
#pragma unroll 1
    for (int m = 0; m < kExpandItems; ++m) {
      const int64_t j = j0 + (int64_t)m * kExpandThreads + threadIdx.x;
      const bool live = j < j1;
      int32_t row = 0, rid = 0;
      if (live) {
        const int64_t e = upper_index(s_off, 0, ne - 1, j);
        row = s_row[e];
        rid = __ldg(grp_rid + s_start[e] + (j - s_off[e]));
        if (g.out_prid) __stcs(g.out_prid + j, row);
        if (g.out_brid) __stcs(g.out_brid + j, rid);
      }
      for (int c = 0; c < g.n_pin; ++c) {
        const PayloadIn in = g.pin[c];
        bool v = false;
        if (live) {
          store_elem_cs(g.pout[c].data, j, in.width, load_elem(in.data, row, in.width));
          v = bit_valid(in.valid, in.voff, row);
        }
        if (in.valid) {
          const unsigned word = __ballot_sync(kFullMask, v);
          if (lane == 0 && j - lane < j1) g.pout[c].valid[(j - lane) >> 5] = word;
        }
      }
      for (int c = 0; c < g.n_bin; ++c) {
        const PayloadIn in = g.bin[c];
        bool v = false;
        if (live) {
          store_elem_cs(g.bout[c].data, j, in.width, load_elem(in.data, rid, in.width));
          v = bit_valid(in.valid, in.voff, rid);
        }
        if (in.valid) {
          const unsigned word = __ballot_sync(kFullMask, v);
          if (lane == 0 && j - lane < j1) g.bout[c].valid[(j - lane) >> 5] = word;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) s_e0 = e0 + upper_index(s_off, 0, ne - 1, j1);
    __syncthreads();
    e0 = s_e0;
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
static void launch_distinct(const sj_table* t, const sj_column& p, const GatherArgs& g, cudaStream_t s) {
  const int block = 256;
  probe_distinct_kernel<K, WIDE, VEC, COUNT_ONLY><<<probe_grid(t, p.num_rows, block), block, 0, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, g);
}

template <bool COUNT_ONLY>
static void dispatch_distinct(const sj_table* t, const sj_column& p, const GatherArgs& g, cudaStream_t s) {
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  const bool vec = aligned16(p.data);
  if (t->key_type == SJ_INT32) {
    if (wide) vec ? launch_distinct<int32_t, true, true, COUNT_ONLY>(t, p, g, s)
                  : launch_distinct<int32_t, true, false, COUNT_ONLY>(t, p, g, s);
    else vec ? launch_distinct<int32_t, false, true, COUNT_ONLY>(t, p, g, s)
             : launch_distinct<int32_t, false, false, COUNT_ONLY>(t, p, g, s);
  } else {
    if (wide) vec ? launch_distinct<int64_t, true, true, COUNT_ONLY>(t, p, g, s)
                  : launch_distinct<int64_t, true, false, COUNT_ONLY>(t, p, g, s);
    else vec ? launch_distinct<int64_t, false, true, COUNT_ONLY>(t, p, g, s)
             : launch_distinct<int64_t, false, false, COUNT_ONLY>(t, p, g, s);
  }
}

template <typename K, bool WIDE, bool VEC, bool COMPACT>
static void launch_match(const sj_table* t, const sj_column& p, int32_t* m_row, int32_t* m_start, int32_t* m_cnt,
                         unsigned long long* d_nent, unsigned long long* d_total, cudaStream_t s) {
  const int block = 256;
  grouped_match_kernel<K, WIDE, VEC, COMPACT><<<probe_grid(t, p.num_rows, block), block, 0, s>>>(
      table_dev(t), static_cast<const K*>(p.data), p.validity, p.validity_offset, p.num_rows, m_row, m_start,
      m_cnt, d_nent, d_total);
}

template <bool COMPACT>
static void dispatch_match(const sj_table* t, const sj_column& p, int32_t* m_row, int32_t* m_start, int32_t* m_cnt,
                           unsigned long long* d_nent, unsigned long long* d_total, cudaStream_t s) {
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  const bool vec = aligned16(p.data);
#define SJ_M(K, W, V) launch_match<K, W, V, COMPACT>(t, p, m_row, m_start, m_cnt, d_nent, d_total, s)
  if (t->key_type == SJ_INT32) {
    if (wide) { if (vec) SJ_M(int32_t, true, true); else SJ_M(int32_t, true, false); }
    else { if (vec) SJ_M(int32_t, false, true); else SJ_M(int32_t, false, false); }
  } else {
    if (wide) { if (vec) SJ_M(int64_t, true, true); else SJ_M(int64_t, true, false); }
    else { if (vec) SJ_M(int64_t, false, true); else SJ_M(int64_t, false, false); }
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
    dispatch_distinct<true>(t, p, g, s);
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
      (gs.n_build_payload && (!gs.build_payload || !gs.out_build_payload)))
    return set_error(SJ_ERR_INVALID, "payload column arrays must not be NULL");
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
    pi.data = in.data;
    pi.valid = in.validity;
    pi.voff = in.validity_offset;
    pi.width = type_width(in.type);
    po.data = out.data;
    po.valid = in.validity ? out.validity : nullptr;
    return SJ_OK;
  };
  for (int c = 0; c < g.n_pin; ++c)
    SJ_TRY(fill(gs.probe_payload[c], gs.out_probe_payload[c], p.num_rows, g.pin[c], g.pout[c], "probe"));
  for (int c = 0; c < g.n_bin; ++c)
    SJ_TRY(fill(gs.build_payload[c], gs.out_build_payload[c], t->build_rows, g.bin[c], g.bout[c], "build"));
  g.out_prid = gs.out_probe_rid;
  g.out_brid = gs.out_build_rid;
  g.capacity = gs.capacity;
  return SJ_OK;
}

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
    dispatch_distinct<false>(t, p, g, s);
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
  device_exclusive_scan<int32_t, int64_t>(m_cnt, m_off, d_nent, 0, tmp, s);
  const int grid = sm_count(t->device) * 4;
  expand_kernel<<<grid, kExpandThreads, 0, s>>>(m_row, m_start, m_off, d_nent, t->grp_rid, g);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
