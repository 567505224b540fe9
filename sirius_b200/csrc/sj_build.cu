// Hash-table build for the sm_100a equi-join (replaces the cudf::hash_join /
// cudf::distinct_hash_join constructors called at src/op/sirius_physical_hash_join.cpp:1614-1620).
//
// Passes (all stream-ordered on the caller's stream):
//   1. stats    min / max of the valid keys, valid and NULL row counts (one read of the keys).
//               The host reads them (sync #1) to pick the slot encoding and the table size.
//   2. insert   insert-or-find: each valid row CASes ((key-kmin) << rid_bits | row) into the first
//               EMPTY slot of its probe sequence unless its key is already present, in which case
//               it only counts a duplicate. The host reads the duplicate count (sync #2).
//   3. grouped  only when duplicates exist (or GROUPED is forced, or NULLs are equal):
//               count rows per slot (warp-aggregated with __match_any_sync), exclusive scan of the
//               counts into per-slot offsets, scatter row ids into one array ordered by group.
//               Duplicated keys then cost one slot each and a probe expands a whole group as a
//               contiguous row-id range, so a key with 10^6 copies is no longer a 10^6-slot cluster.
// A DISTINCT table is the result of pass 2 alone: one slot per build row (the unique-key case of
// distinct_hash_join, load factor 0.5 by default as at :1615).
#include <algorithm>
#include <climits>
#include <cstring>

#include <cmath>
#include <type_traits>

#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_partition.cuh"
#include "sj_scan.cuh"

namespace sj {

struct BuildStats {
  long long kmin;
  long long kmax;
  unsigned long long n_valid;
  unsigned long long n_null;
  unsigned long long n_dup;
  unsigned int full;
  unsigned int max_group;
};

__global__ void stats_init_kernel(BuildStats* st) {
  st->kmin = LLONG_MAX;
  st->kmax = LLONG_MIN;
  st->n_valid = 0;
  st->n_null = 0;
  st->n_dup = 0;
  st->full = 0;
  st->max_group = 0;
}

template <typename K>
__global__ void __launch_bounds__(256) stats_kernel(const K* __restrict__ keys, const uint32_t* kv,
                                                    int64_t kvoff, int64_t n, BuildStats* st) {
  long long mn = LLONG_MAX, mx = LLONG_MIN;
  unsigned long long nv = 0, nn = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (bit_valid(kv, kvoff, i)) {
      const long long k = (long long)keys[i];
      mn = k < mn ? k : mn;
      mx = k > mx ? k : mx;
      ++nv;
    } else {
      ++nn;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    long long a = __shfl_down_sync(kFullMask, mn, d);
    long long b = __shfl_down_sync(kFullMask, mx, d);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
    nv += __shfl_down_sync(kFullMask, nv, d);
    nn += __shfl_down_sync(kFullMask, nn, d);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nv) {
      atomicMin(&st->kmin, mn);
      atomicMax(&st->kmax, mx);
      atomicAdd(&st->n_valid, nv);
    }
    if (nn) atomicAdd(&st->n_null, nn);
  }
}

// Insert-or-find one key. Returns 0 = inserted, 1 = key already present, 2 = segment full.
template <bool WIDE>
__device__ __forceinline__ int insert_or_find(const TableDev& t, uint64_t kb, uint64_t kn, int32_t row,
                                              uint32_t* slot_out) {
  using Ops = SlotOps<WIDE>;
  void* slots = const_cast<void*>(t.slots);
  uint32_t b = home_bucket(t, kb);
  const uint64_t packed = (kn << t.rbits) | (uint64_t)(uint32_t)row;
  for (uint32_t step = 0; step <= t.segmask; ++step) {
    Bucket bk = load_bucket<false>(slots, b);
#pragma unroll
    for (int q = 0; q < Ops::kSlots; ++q) {
      if (Ops::empty(bk, q)) {
        if (!WIDE) {
          unsigned long long* p = reinterpret_cast<unsigned long long*>(slots) + (size_t)b * 4 + q;
          const unsigned long long old = atomicCAS(p, kEmpty, packed);
          if (old == kEmpty) {
            *slot_out = b * Ops::kSlots + q;
            return 0;
          }
          bk.a[q] = old;
        } else {
          uint64_t* p = reinterpret_cast<uint64_t*>(slots) + (size_t)b * 4 + 2 * q;
          uint64_t olo, ohi;
          cas128(p, kEmpty, kEmpty, kb, (uint64_t)(uint32_t)row, olo, ohi);
          if (ohi == kEmpty) {
            *slot_out = b * Ops::kSlots + q;
            return 0;
          }
          bk.a[2 * q] = olo;
          bk.a[2 * q + 1] = ohi;
        }
      }
      if (Ops::match(bk, q, kn, kb, t.rbits)) {
        *slot_out = b * Ops::kSlots + q;
        return 1;
      }
    }
    b = next_bucket(b, t.segmask);
  }
  return 2;
}

// Find the slot of a key known to be in the table (grouped passes). UINT32_MAX if absent.
template <bool WIDE>
__device__ __forceinline__ uint32_t find_slot(const TableDev& t, uint64_t kb, uint64_t kn) {
  using Ops = SlotOps<WIDE>;
  uint32_t b = home_bucket(t, kb);
  for (uint32_t step = 0; step <= t.segmask; ++step) {
    const Bucket bk = load_bucket<true>(t.slots, b);
    bool has_empty = false;
#pragma unroll
    for (int q = 0; q < Ops::kSlots; ++q) {
      if (Ops::match(bk, q, kn, kb, t.rbits)) return b * Ops::kSlots + q;
      has_empty |= Ops::empty(bk, q);
    }
    if (has_empty) break;
    b = next_bucket(b, t.segmask);
  }
  return 0xffffffffu;
}

// bloom != NULL: the build's dynamic filter gets each inserted key's bits in the same pass (the key
// is already in a register; its hash is the one the insert computes).
template <typename K, bool WIDE>
__global__ void __launch_bounds__(256) insert_kernel(TableDev t, const K* __restrict__ keys,
                                                     const uint32_t* kv, int64_t kvoff, int64_t n,
                                                     BuildStats* st, uint32_t* bloom, int bloom_log2) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    int r = -1;
    if (i < n && bit_valid(kv, kvoff, i)) {
      const K k = keys[i];
      const uint64_t kb = key_u64<K>(k);
      const uint64_t kn = (uint64_t)(long long)k - (uint64_t)t.kmin;
      uint32_t s;
      r = insert_or_find<WIDE>(t, kb, kn, (int32_t)i, &s);
      if (bloom) bloom_add(bloom, bloom_log2, kb);
    }
    const unsigned dup = __ballot_sync(kFullMask, r == 1);
    const unsigned full = __ballot_sync(kFullMask, r == 2);
    if (lane == 0) {
      if (dup) atomicAdd(&st->n_dup, (unsigned long long)__popc(dup));
      if (full) atomicOr(&st->full, 1u);
    }
  }
}

// Copy every live slot of `src` into `dst` (a smaller table): the grouped build shrinks the
// table to its distinct keys so that the probe's random reads hit a table sized by distinct keys.
template <bool WIDE>
__global__ void __launch_bounds__(256) reinsert_kernel(TableDev src, uint64_t src_buckets, TableDev dst,
                                                       BuildStats* st) {
  using Ops = SlotOps<WIDE>;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < src_buckets;
       b += (uint64_t)gridDim.x * blockDim.x) {
    const Bucket bk = load_bucket<true>(src.slots, (uint32_t)b);
#pragma unroll
    for (int q = 0; q < Ops::kSlots; ++q) {
      if (Ops::empty(bk, q)) continue;
      uint64_t kb, kn;
      int32_t row;
      if (!WIDE) {
        kn = bk.a[q] >> src.rbits;
        kb = kn + (uint64_t)src.kmin;
        row = (int32_t)(bk.a[q] & ((1ull << src.rbits) - 1));
      } else {
        kb = bk.a[2 * q];
        kn = kb - (uint64_t)src.kmin;
        row = (int32_t)bk.a[2 * q + 1];
      }
      uint32_t s;
      if (insert_or_find<WIDE>(dst, kb, kn, row, &s) == 2) atomicOr(&st->full, 1u);
    }
  }
}

// Grouped pass A: rows per slot. NULL-key rows count into the NULL group when NULLs are equal.
template <typename K, bool WIDE>
__global__ void __launch_bounds__(256) group_count_kernel(TableDev t, const K* __restrict__ keys,
                                                          const uint32_t* kv, int64_t kvoff, int64_t n,
                                                          int32_t* cnt, BuildStats* st) {
  const int lane = threadIdx.x & 31;
  unsigned int local_max = 0;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    int64_t s = -1;
    if (i < n) {
      if (bit_valid(kv, kvoff, i)) {
        const K k = keys[i];
        const uint64_t kb = key_u64<K>(k);
        const uint64_t kn = (uint64_t)(long long)k - (uint64_t)t.kmin;
        const uint32_t f = find_slot<WIDE>(t, kb, kn);
        if (f != 0xffffffffu) s = f;
      } else if (t.null_group >= 0) {
        s = t.null_group;
      }
    }
    const unsigned peers = __match_any_sync(kFullMask, (unsigned long long)s);
    const int leader = __ffs(peers) - 1;
    if (s >= 0 && lane == leader) {
      const int add = __popc(peers);
      const int now = atomicAdd(cnt + s, add) + add;
      local_max = (unsigned)now > local_max ? (unsigned)now : local_max;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    unsigned o = __shfl_down_sync(kFullMask, local_max, d);
    local_max = o > local_max ? o : local_max;
  }
  if (lane == 0 && local_max) atomicMax(&st->max_group, local_max);
}

// Grouped pass B: scatter row ids into their group's range (cursor starts at zero).
template <typename K, bool WIDE>
__global__ void __launch_bounds__(256) group_scatter_kernel(TableDev t, const K* __restrict__ keys,
                                                            const uint32_t* kv, int64_t kvoff, int64_t n,
                                                            const int32_t* __restrict__ off,
                                                            int32_t* cursor, int32_t* grp_rid) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + threadIdx.x;
    int64_t s = -1;
    if (i < n) {
      if (bit_valid(kv, kvoff, i)) {
        const K k = keys[i];
        const uint64_t kb = key_u64<K>(k);
        const uint64_t kn = (uint64_t)(long long)k - (uint64_t)t.kmin;
        const uint32_t f = find_slot<WIDE>(t, kb, kn);
        if (f != 0xffffffffu) s = f;
      } else if (t.null_group >= 0) {
        s = t.null_group;
      }
    }
    const unsigned peers = __match_any_sync(kFullMask, (unsigned long long)s);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (s >= 0 && lane == leader) base = atomicAdd(cursor + s, __popc(peers));
    base = __shfl_sync(kFullMask, base, leader);
    if (s >= 0) {
      const int rank = __popc(peers & ((1u << lane) - 1));
      grp_rid[off[s] + base + rank] = (int32_t)i;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------

static int bit_width_u64(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

// Row store of a GROUPED table, rewritten in group order: dst record i = src record idx[i]
// (records of `stride` bytes, a multiple of 4), so a probe expanding a group reads its members'
// records contiguously instead of through a position list.
__global__ void __launch_bounds__(256) permute_records_kernel(const char* __restrict__ src, char* __restrict__ dst,
                                                              const int32_t* __restrict__ idx, int64_t n,
                                                              int stride) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const char* a = src + (int64_t)__ldg(idx + i) * stride;
    char* b = dst + i * stride;
    if (stride % 16 == 0) {
      for (int o = 0; o < stride; o += 16)
        *reinterpret_cast<uint4*>(b + o) = __ldg(reinterpret_cast<const uint4*>(a + o));
    } else if (stride % 8 == 0) {
      for (int o = 0; o < stride; o += 8)
        *reinterpret_cast<uint2*>(b + o) = __ldg(reinterpret_cast<const uint2*>(a + o));
    } else {
      for (int o = 0; o < stride; o += 4)
        *reinterpret_cast<uint32_t*>(b + o) = __ldg(reinterpret_cast<const uint32_t*>(a + o));
    }
  }
}

// Row ids of the NULL-key rows (warp-aggregated compaction; order unspecified).
__global__ void __launch_bounds__(256) null_rows_kernel(const uint32_t* __restrict__ kv, int64_t kvoff, int64_t n,
                                                        int32_t* out, unsigned long long* count) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n;
       i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + lane;
    const bool is_null = i < n && !bit_valid(kv, kvoff, i);
    const unsigned bal = __ballot_sync(kFullMask, is_null);
    if (!bal) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(count, (unsigned long long)__popc(bal));
    base = __shfl_sync(kFullMask, base, 0);
    if (is_null) out[base + __popc(bal & ((1u << lane) - 1))] = (int32_t)i;
  }
}

static TableDev make_dev(const sj_table* t) {
  TableDev d{};
  d.slots = t->slots;
  d.grp_off = t->grp_off;
  d.grp_rid = t->grp_rid;
  d.kmin = t->kmin;
  d.kmax = t->kmax;
  d.log2_nb = (uint32_t)t->log2_nb;
  d.segmask = (uint32_t)((1ull << t->seg_log2) - 1);
  d.rbits = (uint32_t)t->rid_bits;
  d.null_group = -1;
  if (t->layout == SJ_LAYOUT_GROUPED && t->null_eq == SJ_NULLS_EQUAL && t->null_rows > 0)
    d.null_group = (int32_t)t->num_slots();
  return d;
}

TableDev table_dev(const sj_table* t) { return make_dev(t); }

static int grid_for(int device, const sj_join_params& p, int64_t work_items, int per_cta) {
  const int64_t need = (work_items + per_cta - 1) / per_cta;
  const int64_t cap = (int64_t)sm_count(device) * std::max(1, p.ctas_per_sm) * 2;
  return (int)std::max<int64_t>(1, std::min(need, cap));
}

template <typename K>
static void launch_stats(const sj_column& c, int grid, BuildStats* st, cudaStream_t s) {
  stats_kernel<K><<<grid, 256, 0, s>>>(static_cast<const K*>(c.data), c.validity, c.validity_offset,
                                       c.num_rows, st);
}

template <typename K, bool WIDE>
static void launch_insert(const TableDev& d, const sj_column& c, int grid, BuildStats* st, sj_bloom* bloom,
                          cudaStream_t s) {
  insert_kernel<K, WIDE><<<grid, 256, 0, s>>>(d, static_cast<const K*>(c.data), c.validity,
                                              c.validity_offset, c.num_rows, st, bloom ? bloom->words : nullptr,
                                              bloom ? bloom->log2_blocks : 0);
}

template <typename K, bool WIDE>
static void launch_group(const TableDev& d, const sj_column& c, int grid, int32_t* cnt, int32_t* off,
                         int32_t* grp_rid, bool scatter, BuildStats* st, cudaStream_t s) {
  if (!scatter)
    group_count_kernel<K, WIDE><<<grid, 256, 0, s>>>(d, static_cast<const K*>(c.data), c.validity,
                                                     c.validity_offset, c.num_rows, cnt, st);
  else
    group_scatter_kernel<K, WIDE><<<grid, 256, 0, s>>>(d, static_cast<const K*>(c.data), c.validity,
                                                       c.validity_offset, c.num_rows, off, cnt, grp_rid);
}

static sj_status alloc_slots(sj_table* t, int log2_nb, cudaStream_t s) {
  t->log2_nb = log2_nb;
  t->seg_log2 = log2_nb - std::min(t->pbits, log2_nb);
  t->slots_bytes = ((size_t)1 << log2_nb) * kBucketBytes;
  SJ_TRY(t->alloc.allocate(&t->slots, t->slots_bytes, s));
  SJ_CUDA_TRY(cudaMemsetAsync(t->slots, 0xff, t->slots_bytes, s));
  return SJ_OK;
}

static int log2_buckets_for(int64_t keys, double lf, int slots_per_bucket) {
  const double slots = std::max<double>(1.0, (double)std::max<int64_t>(keys, 1) / lf);
  const int64_t buckets = (int64_t)std::ceil(slots / slots_per_bucket);
  int l = 0;
  while ((1ll << l) < buckets) ++l;
  return l;
}

// Radix bits chosen from the bytes a probe touches at random (table slots + position map +
// attached payloads): none while that fits comfortably in L2, else enough partitions that one
// partition's share is ~16 MB, so the partitions the GPU works on at any moment stay L2-resident.
int auto_partition_bits(size_t random_bytes) {
  const size_t kFitsL2 = 40ull << 20, kPerPartition = 16ull << 20;
  if (random_bytes <= kFitsL2) return 0;
  int b = 0;
  while (((size_t)1 << b) * kPerPartition < random_bytes && b < kMaxPartitionBits) ++b;
  return b;
}

__global__ void bits_to_bytes_kernel(const uint32_t* bits, int64_t off, int64_t n, uint8_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = bit_valid(bits, off, i) ? 1 : 0;
}

template <typename Fn>
static void by_type(int32_t key_type, bool wide, Fn&& fn) {
  if (key_type == SJ_INT32) {
    if (wide) fn(int32_t{}, std::true_type{});
    else fn(int32_t{}, std::false_type{});
  } else {
    if (wide) fn(int64_t{}, std::true_type{});
    else fn(int64_t{}, std::false_type{});
  }
}

sj_status build_table(const sj_column& keys, const sj_column* payload, int32_t n_payload, const sj_join_params& p,
                      const Allocator& alloc, cudaStream_t stream, sj_table** out) {
  SJ_TRY(validate_column(&keys, "build key", true));
  if (keys.num_rows > INT32_MAX)
    return set_error(SJ_ERR_INVALID, "build side exceeds the int32 row-id range");
  if (!(p.load_factor > 0.0f && p.load_factor < 1.0f))
    return set_error(SJ_ERR_INVALID, "load_factor must be in (0, 1)");
  if (p.layout < SJ_LAYOUT_AUTO || p.layout > SJ_LAYOUT_GROUPED)
    return set_error(SJ_ERR_INVALID, "unknown layout");
  if (p.partition_bits < -1 || p.partition_bits > kMaxPartitionBits)
    return set_error(SJ_ERR_INVALID, "partition_bits must be 0 (automatic), -1 (never) or in [1, 10]");
  if (p.probe_kernel < SJ_PROBE_KERNEL_AUTO || p.probe_kernel > SJ_PROBE_KERNEL_DIRECT_TMA)
    return set_error(SJ_ERR_INVALID, "unknown probe_kernel");
  if (p.rows_per_lane != 0 && (p.rows_per_lane < 2 || p.rows_per_lane > 4))
    return set_error(SJ_ERR_INVALID, "rows_per_lane must be 0 (default), 2, 3 or 4");
  if (p.probe_partition_mb < 0 || p.probe_partition_mb > 65536)
    return set_error(SJ_ERR_INVALID, "probe_partition_mb must be in [0, 65536]");
  if (p.table_l2_priority < SJ_L2_AUTO || p.table_l2_priority > SJ_L2_EVICT_LAST)
    return set_error(SJ_ERR_INVALID, "unknown table_l2_priority");
  if (p.bloom_bits_per_key < 0 || p.bloom_bits_per_key > 1024)
    return set_error(SJ_ERR_INVALID, "bloom_bits_per_key must be in [0, 1024]");
  if (n_payload < 0 || n_payload > kMaxPayload || (n_payload > 0 && payload == nullptr))
    return set_error(SJ_ERR_INVALID, "at most 8 attached payload columns");
  for (int c = 0; c < n_payload; ++c) {
    SJ_TRY(validate_column(&payload[c], "attached build payload", false));
    if (payload[c].num_rows != keys.num_rows)
      return set_error(SJ_ERR_INVALID, "attached build payload row count differs from the key column");
  }

  sj_table* t = new sj_table();
  t->alloc = alloc;
  cudaGetDevice(&t->device);
  t->key_type = keys.type;
  t->null_eq = p.null_equality;
  t->params = p;
  t->build_rows = keys.num_rows;
  auto fail = [&](sj_status st) {
    destroy_table(t, stream);
    return st;
  };

  Scratch st_buf;
  if (sj_status e = st_buf.get(alloc, sizeof(BuildStats), stream)) return fail(e);
  BuildStats* st = st_buf.as<BuildStats>();
  stats_init_kernel<<<1, 1, 0, stream>>>(st);
  const int64_t n = keys.num_rows;
  const int grid = grid_for(t->device, p, std::max<int64_t>(n, 1), 256);
  if (n > 0) {
    if (keys.type == SJ_INT32) launch_stats<int32_t>(keys, grid, st, stream);
    else launch_stats<int64_t>(keys, grid, st, stream);
  }
  BuildStats h{};
  if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return fail(set_error(SJ_ERR_DEVICE, std::string("build stats: ") + cudaGetErrorString(cudaGetLastError())));
  t->valid_rows = (int64_t)h.n_valid;
  t->null_rows = (int64_t)h.n_null;
  if (t->valid_rows > 0) {
    t->kmin = h.kmin;
    t->kmax = h.kmax;
  } else {
    t->kmin = 0;
    t->kmax = -1;
  }

  // Slot encoding: packed when (key - kmin) and the row position share 64 bits with the all-ones
  // key field left unused, wide otherwise.
  t->rid_bits = std::max(1, bit_width_u64((uint64_t)std::max<int64_t>(n - 1, 0)));
  const uint64_t range = t->valid_rows > 0 ? (uint64_t)t->kmax - (uint64_t)t->kmin : 0;
  const uint64_t key_field_max = (1ull << (64 - t->rid_bits)) - 1;  // all-ones = EMPTY marker
  const bool packed_fits = range < key_field_max;
  t->slot_kind = (packed_fits && !p.force_wide) ? SJ_SLOT_PACKED64 : SJ_SLOT_WIDE128;
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  const int spb = wide ? 2 : 4;
  int log2_nb = log2_buckets_for(t->valid_rows, p.load_factor, spb);
  if (log2_nb > 31) return fail(set_error(SJ_ERR_INVALID, "table too large"));

  // Partitioning (radix bits) and positions.
  const bool null_group = t->null_eq == SJ_NULLS_EQUAL && t->null_rows > 0;
  size_t pay_row_bytes = 0;
  for (int c = 0; c < n_payload; ++c) pay_row_bytes += (size_t)type_width(payload[c].type);
  // bytes a probe touches at random: slots + one row-store record per valid row (row id,
  // validity bytes, payload fields, rounded up to a power of two)
  size_t rec_bytes = 4 + pay_row_bytes + (size_t)n_payload;
  size_t rec = 4;
  while (rec < rec_bytes) rec <<= 1;
  const size_t random_bytes = ((size_t)1 << log2_nb) * kBucketBytes + (size_t)t->valid_rows * rec;
  int pbits = p.partition_bits == 0 ? auto_partition_bits(random_bytes) : std::max(0, p.partition_bits);
  if (null_group) pbits = 0;  // NULL-key rows stay addressable by row id for the NULL group
  pbits = std::min(pbits, log2_nb);
  t->pbits = pbits;
  t->params.partition_bits = pbits;
  const bool use_pos = !null_group && t->valid_rows > 0 && (pbits > 0 || n_payload > 0);
  if (sj_status e = alloc_slots(t, log2_nb, stream)) return fail(e);

  t->n_attached = n_payload;
  for (int c = 0; c < n_payload; ++c) t->apay_type[c] = payload[c].type;
  const int kw = keys.type == SJ_INT32 ? 4 : 8;
  // key source of the insert / grouped passes: the caller's column, or its partitioned copy
  sj_column src = keys;
  Scratch part_keys, part_scratch;
  if (use_pos) {
    const int64_t nv = t->valid_rows;
    if (sj_status e = part_keys.get(alloc, (size_t)nv * kw, stream)) return fail(e);
    if (sj_status e = part_scratch.get(alloc, partition_scratch_bytes(pbits, t->device), stream)) return fail(e);
    // row-store record layout
    int off = 4;  // build row id
    int voff[kMaxPayload], poff[kMaxPayload];
    for (int c = 0; c < n_payload; ++c) voff[c] = payload[c].validity ? off++ : -1;
    for (int c = 0; c < n_payload; ++c) {
      const int w = type_width(payload[c].type);
      off = (off + w - 1) / w * w;
      poff[c] = off;
      off += w;
    }
    int rec = 4;
    while (rec < off && rec < 64) rec <<= 1;
    if (rec < off) rec = (off + 15) / 16 * 16;
    t->arow_stride = rec;
    t->arow_bytes = (size_t)nv * rec;
    if (sj_status e = alloc.allocate(&t->arow, t->arow_bytes, stream)) return fail(e);
    char* arow = static_cast<char*>(t->arow);
    t->pos_rid = reinterpret_cast<int32_t*>(arow);
    t->pos_stride = rec;
    PartSrc ps{};
    PartDst pd{};
    ps.keys = keys.data;
    ps.kvalid = keys.validity;
    ps.kvoff = keys.validity_offset;
    ps.n = n;
    ps.n_pay = n_payload;
    pd.keys = part_keys.ptr;
    pd.rid = t->pos_rid;
    pd.stride = rec;
    for (int c = 0; c < n_payload; ++c) {
      const int w = type_width(payload[c].type);
      ps.pay[c] = column_payload(payload[c].data, payload[c].validity, payload[c].validity_offset, w);
      t->apay[c] = arow + poff[c];
      t->apay_stride[c] = rec;
      t->apay_valid[c] = voff[c] >= 0 ? reinterpret_cast<uint8_t*>(arow + voff[c]) : nullptr;
      t->apay_vstride[c] = rec;
      pd.pay[c] = t->apay[c];
      pd.valid8[c] = t->apay_valid[c];
    }
    const int64_t *d_total, *d_offs;
    int G;
    if (sj_status e = radix_partition(ps, keys.type, pbits, pd, part_scratch.ptr, t->device, stream, &d_total,
                                      &d_offs, &G))
      return fail(e);
    src = sj_column{part_keys.ptr, nullptr, 0, nv, keys.type, 0};
  } else if (n_payload > 0) {
    // positions are row ids: attach owned row-ordered column copies
    t->apay_owned = true;
    for (int c = 0; c < n_payload; ++c) {
      const int w = type_width(payload[c].type);
      t->apay_bytes[c] = (size_t)std::max<int64_t>(n, 1) * w;
      t->apay_stride[c] = w;
      t->apay_vstride[c] = 1;
      if (sj_status e = alloc.allocate(&t->apay[c], t->apay_bytes[c], stream)) return fail(e);
      if (n > 0) SJ_CUDA_TRY(cudaMemcpyAsync(t->apay[c], payload[c].data, (size_t)n * w, cudaMemcpyDeviceToDevice, stream));
      if (payload[c].validity) {
        t->apay_valid_bytes[c] = (size_t)std::max<int64_t>(n, 1);
        if (sj_status e = alloc.allocate((void**)&t->apay_valid[c], t->apay_valid_bytes[c], stream)) return fail(e);
        if (n > 0)
          bits_to_bytes_kernel<<<grid, 256, 0, stream>>>(payload[c].validity, payload[c].validity_offset, n,
                                                         t->apay_valid[c]);
      }
    }
  }
  const int64_t sn = src.num_rows;
  const int sgrid = grid_for(t->device, p, std::max<int64_t>(sn, 1), 256);

  // the dynamic filter, sized by the build rows as sj_bloom_build sizes it, filled by the insert
  if (p.bloom_bits_per_key > 0)
    if (sj_status e = bloom_create(n, p.bloom_bits_per_key, keys.type, alloc, stream, &t->bloom)) return fail(e);
  TableDev d = make_dev(t);
  if (t->valid_rows > 0) {
    KernelTimer timer("insert", stream);
    by_type(keys.type, wide, [&](auto k, auto w) {
      launch_insert<decltype(k), decltype(w)::value>(d, src, sgrid, st, t->bloom, stream);
    });
  }
  if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return fail(set_error(SJ_ERR_DEVICE, std::string("build insert: ") + cudaGetErrorString(cudaGetLastError())));
  if (h.full) return fail(set_error(SJ_ERR_TABLE_FULL, "a table segment ran out of slots"));
  t->distinct = t->valid_rows - (int64_t)h.n_dup;

  const bool grouped = p.layout == SJ_LAYOUT_GROUPED || h.n_dup > 0 || null_group;
  if (p.layout == SJ_LAYOUT_DISTINCT && grouped)
    return fail(set_error(SJ_ERR_INVALID, "layout DISTINCT requested but the build keys are not unique"));
  t->layout = grouped ? SJ_LAYOUT_GROUPED : SJ_LAYOUT_DISTINCT;
  t->max_group = 1;

  if (grouped) {
    // Shrink to the distinct keys when that saves at least 4x (keeping the partition bits).
    const int want = std::max(log2_buckets_for(t->distinct, p.load_factor, spb), t->pbits);
    if (want + 2 <= t->log2_nb) {
      TableDev old = d;
      void* old_slots = t->slots;
      const size_t old_bytes = t->slots_bytes;
      const uint64_t old_buckets = 1ull << t->log2_nb;
      t->slots = nullptr;
      if (sj_status e = alloc_slots(t, want, stream)) {
        alloc.release(old_slots, old_bytes, stream);
        return fail(e);
      }
      d = make_dev(t);
      const int g2 = grid_for(t->device, p, (int64_t)old_buckets, 256);
      if (wide) reinsert_kernel<true><<<g2, 256, 0, stream>>>(old, old_buckets, d, st);
      else reinsert_kernel<false><<<g2, 256, 0, stream>>>(old, old_buckets, d, st);
      alloc.release(old_slots, old_bytes, stream);
    }
    const int64_t ns = t->num_slots();
    const int64_t ngroups = ns + 1;  // + the NULL group
    Scratch cnt_buf, tmp_buf;
    if (sj_status e = cnt_buf.get(alloc, (size_t)ngroups * sizeof(int32_t), stream)) return fail(e);
    if (sj_status e = tmp_buf.get(alloc, kScanBlocks * sizeof(int64_t), stream)) return fail(e);
    int32_t* cnt = cnt_buf.as<int32_t>();
    SJ_CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)ngroups * sizeof(int32_t), stream));
    t->grp_off_bytes = (size_t)(ngroups + 1) * sizeof(int32_t);
    if (sj_status e = alloc.allocate((void**)&t->grp_off, t->grp_off_bytes, stream)) return fail(e);
    const int64_t grouped_rows = t->valid_rows + (null_group ? t->null_rows : 0);
    t->grp_rid_bytes = (size_t)std::max<int64_t>(grouped_rows, 1) * sizeof(int32_t);
    if (sj_status e = alloc.allocate((void**)&t->grp_rid, t->grp_rid_bytes, stream)) return fail(e);
    d = make_dev(t);
    if (sn > 0)
      by_type(keys.type, wide, [&](auto k, auto w) {
        launch_group<decltype(k), decltype(w)::value>(d, src, sgrid, cnt, nullptr, nullptr, false, st, stream);
      });
    device_exclusive_scan<int32_t, int32_t>(cnt, t->grp_off, nullptr, ngroups, tmp_buf.as<int64_t>(), stream);
    SJ_CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)ngroups * sizeof(int32_t), stream));
    if (sn > 0)
      by_type(keys.type, wide, [&](auto k, auto w) {
        launch_group<decltype(k), decltype(w)::value>(d, src, sgrid, cnt, t->grp_off, t->grp_rid, true, st, stream);
      });
    if (cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return fail(set_error(SJ_ERR_DEVICE, std::string("grouped build: ") + cudaGetErrorString(cudaGetLastError())));
    if (h.full) return fail(set_error(SJ_ERR_TABLE_FULL, "a table segment ran out of slots"));
    t->max_group = (int32_t)std::max<unsigned>(h.max_group, 1u);
    if (t->arow && grouped_rows > 0) {
      // positions become group-order indices: the row store is rewritten in group order and the
      // position list (now the identity) is dropped
      void* arow2 = nullptr;
      if (sj_status e = alloc.allocate(&arow2, t->arow_bytes, stream)) return fail(e);
      const int g3 = grid_for(t->device, p, grouped_rows, 256);
      permute_records_kernel<<<g3, 256, 0, stream>>>(static_cast<const char*>(t->arow), static_cast<char*>(arow2),
                                                     t->grp_rid, grouped_rows, t->arow_stride);
      char* o = static_cast<char*>(t->arow);
      char* nw = static_cast<char*>(arow2);
      t->pos_rid = reinterpret_cast<int32_t*>(nw + (reinterpret_cast<char*>(t->pos_rid) - o));
      for (int c = 0; c < n_payload; ++c) {
        t->apay[c] = nw + (static_cast<char*>(t->apay[c]) - o);
        if (t->apay_valid[c]) t->apay_valid[c] = reinterpret_cast<uint8_t*>(nw + (reinterpret_cast<char*>(t->apay_valid[c]) - o));
      }
      alloc.release(t->arow, t->arow_bytes, stream);
      t->arow = arow2;
      alloc.release(t->grp_rid, t->grp_rid_bytes, stream);
      t->grp_rid = nullptr;
      t->grp_rid_bytes = 0;
    }
  }
  if (t->null_rows > 0 && !null_group) {
    t->null_rid_bytes = (size_t)t->null_rows * sizeof(int32_t);
    if (sj_status e = alloc.allocate((void**)&t->null_rid, t->null_rid_bytes, stream)) return fail(e);
    Scratch cnt_buf;
    if (sj_status e = cnt_buf.get(alloc, sizeof(unsigned long long), stream)) return fail(e);
    SJ_CUDA_TRY(cudaMemsetAsync(cnt_buf.ptr, 0, sizeof(unsigned long long), stream));
    null_rows_kernel<<<grid, 256, 0, stream>>>(keys.validity, keys.validity_offset, n, t->null_rid,
                                               cnt_buf.as<unsigned long long>());
  }
  SJ_CUDA_TRY(cudaGetLastError());
  *out = t;
  return SJ_OK;
}

sj_status destroy_table(sj_table* t, cudaStream_t stream) {
  if (!t) return SJ_OK;
  if (t->slots) t->alloc.release(t->slots, t->slots_bytes, stream);
  if (t->grp_off) t->alloc.release(t->grp_off, t->grp_off_bytes, stream);
  if (t->grp_rid) t->alloc.release(t->grp_rid, t->grp_rid_bytes, stream);
  if (t->arow) t->alloc.release(t->arow, t->arow_bytes, stream);
  if (t->null_rid) t->alloc.release(t->null_rid, t->null_rid_bytes, stream);
  bloom_free(t->bloom, stream);
  if (t->apay_owned) {
    for (int c = 0; c < t->n_attached; ++c) {
      if (t->apay[c]) t->alloc.release(t->apay[c], t->apay_bytes[c], stream);
      if (t->apay_valid[c]) t->alloc.release(t->apay_valid[c], t->apay_valid_bytes[c], stream);
    }
  }
  delete t;
  return SJ_OK;
}

}  // namespace sj

int64_t sj_table::num_slots() const {
  return ((int64_t)1 << log2_nb) * (slot_kind == SJ_SLOT_WIDE128 ? 2 : 4);
}
