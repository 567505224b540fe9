// LEFT, SEMI, ANTI, MARK and FULL joins on a built table: the other join types of the operator's
// BUILD_PROBE path (src/op/sirius_physical_hash_join.cpp:1640-1700 — filtered_join::semi_join /
// anti_join, hash_join::left_join / full_join, distinct_hash_join::left_join — and the MARK result of
// resolve_mark_join_result, :1461-1525).
//
//   SEMI / ANTI  one pass: every probe row looks its key up (a NULL key finds nothing unless NULLs
//                compare equal and the build has NULL keys) and the selected rows are compacted with
//                their probe payloads. A warp stages the selected row ids in shared memory and
//                reserves output once per flush of about 224 rows, then writes rows and payloads in
//                contiguous runs: one atomicAdd per 32-row step on the one output counter serialised
//                the pass (64M rows, 30 % absent: ANTI 2.60 ms, MARK — the same lookups without
//                compaction — 0.85 ms).
//   MARK         one pass, no compaction: mark byte and validity bit of every probe row. Unmatched
//                rows are NULL when their key is NULL, or all of them when the build has a NULL key.
//   LEFT         the INNER probe + gather (probe_gather, any table layout), then the unmatched probe
//                rows appended after the INNER rows on the same counter with build row id
//                SJ_NO_ROW: the rows whose bit is clear in a mask set from the INNER rows' probe row
//                ids (or, when no probe row ids are written or the INNER rows overflowed the
//                capacity, the ANTI lookup); validity of the NULL-padded build payloads is set by
//                range.
//   FULL         LEFT, then the unmatched build rows: the build rows whose bit is clear in a mask
//                set from the INNER rows' build row ids (NULL-key rows included). When no build row
//                ids are written or the INNER rows overflowed the capacity: a pass that flags every
//                table slot (group) some probe row matched, then a DISTINCT table walks its slots, a
//                GROUPED table its group-ordered members (group of member i = the last group starting
//                at or before i), and the NULL-key build rows come from the table's NULL-row list.
#include <algorithm>

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

TableDev table_dev(const sj_table* t);

constexpr int kKindThreads = 256;
constexpr int kKindStage = 256;  // staged row ids per warp (SEMI / ANTI rows, FULL's unmatched build rows)
constexpr int32_t kNoRow = (int32_t)0x80000000;

enum KindMode { kSemi = 0, kAnti = 1, kMark = 2, kFlags = 3, kUnmatched = 4 };

struct KindArgs {
  int32_t* out_prid;
  int32_t* out_brid;  // LEFT/FULL append: written with kNoRow
  int32_t n_pin;
  PayloadIn pin[kMaxPayload];
  PayloadOut pout[kMaxPayload];
  int64_t capacity;
  unsigned long long* d_count;
  uint8_t* mark;
  uint32_t* mark_valid;
  int32_t build_has_null;
  uint8_t* flags;  // kFlags: one byte per slot (+ the NULL group)
  const uint32_t* matched;  // kUnmatched: bit i set when probe row i has an INNER row
  const unsigned long long* inner_rows;  // kUnmatched: INNER rows; past `capacity` the bits are
                                         // incomplete and the rows are looked up instead
};

// Slot of key k in the table (k in range), or -1. Slots fill each bucket in order, so the walk stops
// after the first bucket that has an EMPTY slot.
template <typename K, bool WIDE>
__device__ __forceinline__ int64_t find_slot(const TableDev& t, K k) {
  using Ops = SlotOps<WIDE>;
  const uint64_t kb = key_u64<K>(k);
  uint32_t b = home_bucket(t, kb);
  const uint64_t kmask = ~((1ull << t.rbits) - 1);
  const uint64_t ks = Ops::probe_key((uint64_t)(long long)k - (uint64_t)t.kmin, kb, t.rbits);
  for (uint32_t step = 0; step <= t.segmask; ++step) {
    const Bucket bk = load_bucket<true>(t.slots, b);
    bool open = false;
#pragma unroll
    for (int q = 0; q < Ops::kSlots; ++q) {
      if (Ops::match_s(bk, q, ks, kmask)) return (int64_t)b * Ops::kSlots + q;
      open |= Ops::empty(bk, q);
    }
    if (open) return -1;
    b = next_bucket(b, t.segmask);
  }
  return -1;
}

__device__ __forceinline__ bool group_nonempty(const TableDev& t, int64_t s) {
  return t.grp_off == nullptr || __ldg(t.grp_off + s + 1) > __ldg(t.grp_off + s);
}

// The slot (group) a probe row matches, or -1.
template <typename K, bool WIDE>
__device__ __forceinline__ int64_t lookup(const TableDev& t, K k, bool valid) {
  if (!valid) return t.null_group >= 0 && group_nonempty(t, t.null_group) ? (int64_t)t.null_group : -1;
  if (!in_range(t, k)) return -1;
  const int64_t s = find_slot<K, WIDE>(t, k);
  return s >= 0 && group_nonempty(t, s) ? s : -1;
}

template <typename K, bool WIDE, int MODE>
__global__ void __launch_bounds__(kKindThreads) kind_probe_kernel(TableDev t, const K* __restrict__ keys,
                                                                  const uint32_t* __restrict__ kv, int64_t kvoff,
                                                                  int64_t n, KindArgs a) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ int32_t s_stage[kKindThreads / 32][kKindStage];
  int32_t* st = s_stage[threadIdx.x >> 5];
  uint32_t fill = 0;  // staged rows of this warp (warp-uniform)
  const bool by_bits = MODE == kUnmatched && (int64_t)*a.inner_rows <= a.capacity;
  // FULL flags pass: not needed when the build-row bits of the INNER rows are complete
  if (MODE == kFlags && a.inner_rows && (int64_t)*a.inner_rows <= a.capacity) return;
  // reserve the staged rows' output range with one atomicAdd and write them out in order
  auto flush = [&]() {
    __syncwarp();
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(a.d_count, (unsigned long long)fill);
    base = __shfl_sync(kFullMask, base, 0);
    for (uint32_t e = lane; e < fill; e += 32) {
      const int64_t p = (int64_t)base + e;
      if (p >= a.capacity) break;
      const int64_t i = st[e];
      if (a.out_prid) a.out_prid[p] = (int32_t)i;
      if (a.out_brid) a.out_brid[p] = kNoRow;
      for (int c = 0; c < a.n_pin; ++c) {
        store_elem(a.pout[c].data, p, a.pin[c].width, pl_load(a.pin[c], i));
        if (a.pout[c].valid && payload_valid(a.pin[c], i)) set_out_bit(a.pout[c].valid, p);
      }
    }
    __syncwarp();
    fill = 0;
  };
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n; i0 += stride) {
    const int64_t i = i0 + lane;
    const bool live = i < n;
    int64_t s = -1;
    const bool valid = live && (by_bits || bit_valid(kv, kvoff, i));
    if (by_bits) {
      // no lookup: the INNER rows already told which probe rows matched
      if (live && (__ldg(a.matched + (i >> 5)) >> (i & 31) & 1u)) s = 0;
    } else {
      s = live ? lookup<K, WIDE>(t, __ldg(keys + i), valid) : -1;
    }
    const bool found = s >= 0;
    if (MODE == kMark) {
      if (live) a.mark[i] = found ? 1 : 0;
      if (a.mark_valid) {
        const unsigned w = __ballot_sync(kFullMask, live && (found || (!a.build_has_null && valid)));
        if (lane == 0) a.mark_valid[i0 >> 5] = w;
      }
      continue;
    }
    if (MODE == kFlags) {
      if (found) a.flags[s] = 1;
      continue;
    }
    const bool sel = live && (MODE == kSemi ? found : !found);  // kAnti / kUnmatched: the rest
    const unsigned bal = __ballot_sync(kFullMask, sel);
    if (!bal) continue;
    if (sel) st[fill + __popc(bal & below)] = (int32_t)i;
    fill += __popc(bal);
    if (fill > (uint32_t)(kKindStage - 32)) flush();  // the next step could not fit
  }
  if (MODE == kSemi || MODE == kAnti || MODE == kUnmatched)
    if (fill) flush();
}

struct BuildEmitArgs {
  int32_t* out_prid;
  int32_t* out_brid;
  int32_t n_bin;
  PayloadIn bin[kMaxPayload];
  PayloadOut bout[kMaxPayload];
  const int32_t* pos_rid;  // table position -> build row id (NULL: positions are row ids)
  int32_t pos_stride;
  int64_t capacity;
  unsigned long long* d_count;
  const uint8_t* flags;
  // FULL by build-row bits: when set and the INNER rows fit the capacity, the unmatched build rows
  // are the rows whose bit in `matched` is clear (unmatched_build_rows_kernel); the slot / member /
  // NULL-row walks then do nothing
  const unsigned long long* inner_rows;
  const uint32_t* matched;
};

__device__ __forceinline__ bool full_by_bits(const BuildEmitArgs& a) {
  return a.inner_rows != nullptr && (int64_t)*a.inner_rows <= a.capacity;
}

// Unmatched build rows of a FULL join, staged per warp like the SEMI / ANTI rows: build row ids
// collect in the warp's shared-memory area, and a flush reserves their output range with one
// atomicAdd and writes them (probe row id SJ_NO_ROW, build row id, build payloads) in order.
struct BuildEmitter {
  const BuildEmitArgs& a;
  int32_t* st;        // this warp's kKindStage staged build row ids
  uint32_t fill = 0;  // warp-uniform
  __device__ BuildEmitter(const BuildEmitArgs& args, int32_t* stage) : a(args), st(stage) {}
  __device__ void add(bool sel, int32_t brid) {
    const int lane = threadIdx.x & 31;
    const unsigned bal = __ballot_sync(kFullMask, sel);
    if (!bal) return;
    if (sel) st[fill + __popc(bal & ((1u << lane) - 1u))] = brid;
    fill += __popc(bal);
    if (fill > (uint32_t)(kKindStage - 32)) flush();
  }
  __device__ void flush() {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    unsigned long long base = 0;
    if (lane == 0 && fill) base = atomicAdd(a.d_count, (unsigned long long)fill);
    base = __shfl_sync(kFullMask, base, 0);
    for (uint32_t e = lane; e < fill; e += 32) {
      const int64_t p = (int64_t)base + e;
      if (p >= a.capacity) break;
      const int32_t brid = st[e];
      if (a.out_prid) a.out_prid[p] = kNoRow;
      if (a.out_brid) a.out_brid[p] = brid;
      for (int c = 0; c < a.n_bin; ++c) {
        store_elem(a.bout[c].data, p, a.bin[c].width, pl_load(a.bin[c], brid));
        if (a.bout[c].valid && payload_valid(a.bin[c], brid)) set_out_bit(a.bout[c].valid, p);
      }
    }
    __syncwarp();
    fill = 0;
  }
};

__device__ __forceinline__ int32_t rid_of_pos(const BuildEmitArgs& a, int64_t pos) {
  return a.pos_rid ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(a.pos_rid) +
                                                             pos * a.pos_stride))
                   : (int32_t)pos;
}

// FULL, DISTINCT table: every live slot nobody matched.
template <bool WIDE>
__global__ void __launch_bounds__(kKindThreads) unmatched_slots_kernel(TableDev t, int64_t n_slots, BuildEmitArgs a) {
  using Ops = SlotOps<WIDE>;
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ int32_t s_stage[kKindThreads / 32][kKindStage];
  BuildEmitter em(a, s_stage[threadIdx.x >> 5]);
  if (full_by_bits(a)) return;  // unmatched_build_rows_kernel emits them
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n_slots; i0 += stride) {
    const int64_t i = i0 + lane;
    bool sel = false;
    int32_t brid = 0;
    if (i < n_slots) {
      const Bucket bk = load_bucket<true>(t.slots, (uint32_t)(i / Ops::kSlots));
      const int q = (int)(i % Ops::kSlots);
      if (!Ops::empty(bk, q) && !a.flags[i]) {
        sel = true;
        brid = rid_of_pos(a, Ops::rid(bk, q, t.rbits));
      }
    }
    em.add(sel, brid);
  }
  em.flush();
}

// FULL, GROUPED table: member i (group order) belongs to the last group s with grp_off[s] <= i.
__global__ void __launch_bounds__(kKindThreads) unmatched_members_kernel(TableDev t, int64_t n_members,
                                                                         int64_t n_groups, BuildEmitArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ int32_t s_stage[kKindThreads / 32][kKindStage];
  BuildEmitter em(a, s_stage[threadIdx.x >> 5]);
  if (full_by_bits(a)) return;  // unmatched_build_rows_kernel emits them
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n_members; i0 += stride) {
    const int64_t i = i0 + lane;
    bool sel = false;
    int32_t brid = 0;
    if (i < n_members) {
      int64_t lo = 0, hi = n_groups - 1;  // largest s with grp_off[s] <= i
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(t.grp_off + mid) <= i) lo = mid;
        else hi = mid - 1;
      }
      if (!a.flags[lo]) {
        sel = true;
        brid = rid_of_pos(a, t.grp_rid ? (int64_t)__ldg(t.grp_rid + i) : i);
      }
    }
    em.add(sel, brid);
  }
  em.flush();
}

// FULL: the NULL-key build rows (not in the table when NULLs never match).
__global__ void __launch_bounds__(kKindThreads) null_build_rows_kernel(const int32_t* __restrict__ null_rid,
                                                                       int64_t n_null, BuildEmitArgs a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ int32_t s_stage[kKindThreads / 32][kKindStage];
  BuildEmitter em(a, s_stage[threadIdx.x >> 5]);
  if (full_by_bits(a)) return;  // unmatched_build_rows_kernel emits them
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n_null; i0 += stride) {
    const int64_t i = i0 + (threadIdx.x & 31);
    em.add(i < n_null, i < n_null ? __ldg(null_rid + i) : 0);
  }
  em.flush();
}

// FULL by build-row bits: every build row (NULL keys included) whose bit is clear.
__global__ void __launch_bounds__(kKindThreads) unmatched_build_rows_kernel(const uint32_t* __restrict__ matched,
                                                                            int64_t nb, BuildEmitArgs a) {
  if (!full_by_bits(a)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ int32_t s_stage[kKindThreads / 32][kKindStage];
  BuildEmitter em(a, s_stage[threadIdx.x >> 5]);
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < nb; i0 += stride) {
    const int64_t i = i0 + (threadIdx.x & 31);
    em.add(i < nb && !(__ldg(matched + (i >> 5)) >> (i & 31) & 1u), (int32_t)i);
  }
  em.flush();
}

// Sets validity bits [lo, hi) (bounds read from the device, clamped to cap; lo_p NULL = 0).
__global__ void set_valid_range_kernel(uint32_t* words, const unsigned long long* lo_p, const unsigned long long* hi_p,
                                       int64_t cap) {
  const int64_t lo = lo_p ? std::min<int64_t>((int64_t)*lo_p, cap) : 0;
  const int64_t hi = std::min<int64_t>((int64_t)*hi_p, cap);
  if (hi <= lo) return;
  for (int64_t w = (lo >> 5) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w <= ((hi - 1) >> 5);
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = std::max<int64_t>(lo, w * 32) - w * 32;
    const int64_t b = std::min<int64_t>(hi, w * 32 + 32) - w * 32;
    const unsigned mask = (b - a == 32) ? kFullMask : (((1u << (b - a)) - 1u) << a);
    atomicOr(words + w, mask);
  }
}

__global__ void set_count_kernel(int64_t* d_count, int64_t v) { *d_count = v; }

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
// LEFT / FULL: bit r of `bits` for every probe row r among the first min(*d_n, cap) INNER rows.
__global__ void __launch_bounds__(256) matched_bits_kernel(const int32_t* __restrict__ prid,
                                                           const unsigned long long* d_n, int64_t cap, uint32_t* bits) {
  const int64_t n = (int64_t)*d_n < cap ? (int64_t)*d_n : cap;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)__ldg(prid + i);
    atomicOr(bits + (r >> 5), 1u << (r & 31));
  }
}

static int kind_grid(const sj_table* t, int64_t n) {
  const int64_t need = (n + kKindThreads - 1) / kKindThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sm_count(t->device) * 8));
}

template <int MODE>
static void launch_kind(const sj_table* t, const sj_column& p, const KindArgs& a, cudaStream_t s) {
  const int grid = kind_grid(t, p.num_rows);
  const TableDev d = table_dev(t);
  const bool wide = t->slot_kind == SJ_SLOT_WIDE128;
  KernelTimer timer(MODE == kMark ? "mark" : MODE == kFlags ? "match_flags" : MODE == kSemi ? "semi"
                    : MODE == kUnmatched ? "unmatched_probe" : "anti", s);
  if (t->key_type == SJ_INT32) {
    if (wide) kind_probe_kernel<int32_t, true, MODE><<<grid, kKindThreads, 0, s>>>(d, static_cast<const int32_t*>(p.data), p.validity, p.validity_offset, p.num_rows, a);
    else kind_probe_kernel<int32_t, false, MODE><<<grid, kKindThreads, 0, s>>>(d, static_cast<const int32_t*>(p.data), p.validity, p.validity_offset, p.num_rows, a);
  } else {
    if (wide) kind_probe_kernel<int64_t, true, MODE><<<grid, kKindThreads, 0, s>>>(d, static_cast<const int64_t*>(p.data), p.validity, p.validity_offset, p.num_rows, a);
    else kind_probe_kernel<int64_t, false, MODE><<<grid, kKindThreads, 0, s>>>(d, static_cast<const int64_t*>(p.data), p.validity, p.validity_offset, p.num_rows, a);
  }
}

static sj_status probe_payloads(const sj_column& p, const GatherSpec& gs, KindArgs& a) {
  if (gs.n_probe_payload < 0 || gs.n_probe_payload > kMaxPayload)
    return set_error(SJ_ERR_INVALID, "at most 8 payload columns per side");
  if (gs.n_probe_payload && (!gs.probe_payload || !gs.out_probe_payload))
    return set_error(SJ_ERR_INVALID, "payload column arrays must not be NULL");
  a.n_pin = gs.n_probe_payload;
  for (int c = 0; c < a.n_pin; ++c) {
    const sj_column& in = gs.probe_payload[c];
    const sj_mut_column& out = gs.out_probe_payload[c];
    SJ_TRY(validate_column(&in, "probe payload", false));
    if (in.num_rows != p.num_rows) return set_error(SJ_ERR_INVALID, "probe payload row count differs from its key column");
    if (out.type != in.type) return set_error(SJ_ERR_INVALID, "probe output type differs");
    if (gs.capacity > 0 && !out.data) return set_error(SJ_ERR_INVALID, "probe output data is NULL");
    if (in.validity && gs.capacity > 0 && !out.validity)
      return set_error(SJ_ERR_INVALID, "probe payload has NULLs but its output has no validity");
    a.pin[c] = column_payload(in.data, in.validity, in.validity_offset, type_width(in.type));
    a.pout[c] = PayloadOut{out.data, in.validity ? out.validity : nullptr};
  }
  return SJ_OK;
}

static sj_status zero_validity(const sj_mut_column* outs, int n, int64_t capacity, cudaStream_t s) {
  const size_t bytes = (size_t)((capacity + 31) / 32) * sizeof(uint32_t);
  for (int c = 0; c < n; ++c)
    if (outs[c].validity && bytes) SJ_CUDA_TRY(cudaMemsetAsync(outs[c].validity, 0, bytes, s));
  return SJ_OK;
}

sj_status probe_join(const sj_table* t, int32_t kind, const sj_column& p, const GatherSpec& gs, uint8_t* out_mark,
                     uint32_t* out_mark_valid, const Allocator& alloc, cudaStream_t s, int64_t* d_count) {
  if (kind == SJ_JOIN_INNER) return probe_gather(t, p, gs, alloc, s, d_count);
  if (kind < SJ_JOIN_INNER || kind > SJ_JOIN_FULL) return set_error(SJ_ERR_INVALID, "unknown join kind");
  SJ_TRY(validate_column(&p, "probe key", true));
  if (p.type != t->key_type) return set_error(SJ_ERR_INVALID, "probe key type differs from the build key type");
  if (p.num_rows > INT32_MAX) return set_error(SJ_ERR_INVALID, "probe side exceeds the int32 row-id range");
  if (gs.capacity < 0) return set_error(SJ_ERR_INVALID, "capacity must be >= 0");
  unsigned long long* dc = reinterpret_cast<unsigned long long*>(d_count);
  KindArgs a{};
  a.capacity = gs.capacity;
  a.d_count = dc;

  if (kind == SJ_JOIN_MARK) {
    if (t->null_eq == SJ_NULLS_EQUAL) return set_error(SJ_ERR_INVALID, "MARK joins compare NULLs as unequal");
    if (p.num_rows > 0 && !out_mark) return set_error(SJ_ERR_INVALID, "MARK needs out_mark");
    a.mark = out_mark;
    a.mark_valid = out_mark_valid;
    a.build_has_null = t->null_rows > 0;
    set_count_kernel<<<1, 1, 0, s>>>(d_count, p.num_rows);
    if (p.num_rows > 0) launch_kind<kMark>(t, p, a, s);
    SJ_CUDA_TRY(cudaGetLastError());
    return SJ_OK;
  }
  if (kind == SJ_JOIN_SEMI || kind == SJ_JOIN_ANTI) {
    SJ_TRY(probe_payloads(p, gs, a));
    a.out_prid = gs.out_probe_rid;
    SJ_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(int64_t), s));
    SJ_TRY(zero_validity(gs.out_probe_payload, gs.n_probe_payload, gs.capacity, s));
    if (p.num_rows > 0) {
      if (kind == SJ_JOIN_SEMI) launch_kind<kSemi>(t, p, a, s);
      else launch_kind<kAnti>(t, p, a, s);
    }
    SJ_CUDA_TRY(cudaGetLastError());
    return SJ_OK;
  }

  // LEFT / FULL
  const bool full = kind == SJ_JOIN_FULL;
  const bool attached = gs.n_build_payload > 0 && gs.build_payload == nullptr;
  if (full && attached)
    return set_error(SJ_ERR_INVALID, "FULL joins gather build payloads from caller columns (build_payload != NULL)");
  for (int c = 0; c < gs.n_build_payload; ++c)
    if (gs.capacity > 0 && (!gs.out_build_payload || !gs.out_build_payload[c].validity))
      return set_error(SJ_ERR_INVALID, "LEFT/FULL build payload outputs need validity (NULL padding)");
  for (int c = 0; full && c < gs.n_probe_payload; ++c)
    if (gs.capacity > 0 && (!gs.out_probe_payload || !gs.out_probe_payload[c].validity))
      return set_error(SJ_ERR_INVALID, "FULL probe payload outputs need validity (NULL padding)");
  SJ_TRY(probe_payloads(p, gs, a));
  if (gs.n_build_payload > 0 && !gs.out_build_payload)
    return set_error(SJ_ERR_INVALID, "payload column arrays must not be NULL");
  SJ_TRY(zero_validity(gs.out_build_payload, gs.n_build_payload, gs.capacity, s));
  if (full) SJ_TRY(zero_validity(gs.out_probe_payload, gs.n_probe_payload, gs.capacity, s));
  Scratch marks;  // [0] = INNER rows, [1] = LEFT rows
  SJ_TRY(marks.get(alloc, 2 * sizeof(unsigned long long), s));
  unsigned long long* m = marks.as<unsigned long long>();

  // 1. INNER rows
  SJ_TRY(probe_gather(t, p, gs, alloc, s, d_count));
  SJ_CUDA_TRY(cudaMemcpyAsync(m, d_count, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  // 2. unmatched probe rows, appended: the probe rows no INNER row names (one bit per probe row, set
  // from the INNER rows' probe row ids; 0.94 ms for a second lookup of 64M rows before), or a second
  // lookup when the call writes no probe row ids
  a.out_prid = gs.out_probe_rid;
  a.out_brid = gs.out_build_rid;
  Scratch mbits;
  if (p.num_rows > 0) {
    if (gs.out_probe_rid && gs.capacity > 0) {
      const size_t words = (size_t)((p.num_rows + 31) / 32);
      SJ_TRY(mbits.get(alloc, words * sizeof(uint32_t), s));
      SJ_CUDA_TRY(cudaMemsetAsync(mbits.ptr, 0, words * sizeof(uint32_t), s));
      {
        KernelTimer timer("matched_bits", s);
        matched_bits_kernel<<<kind_grid(t, std::min<int64_t>(gs.capacity, p.num_rows)), 256, 0, s>>>(
            gs.out_probe_rid, m, gs.capacity, mbits.as<uint32_t>());
      }
      a.matched = mbits.as<uint32_t>();
      a.inner_rows = m;
      launch_kind<kUnmatched>(t, p, a, s);
    } else {
      launch_kind<kAnti>(t, p, a, s);
    }
  }
  SJ_CUDA_TRY(cudaMemcpyAsync(m + 1, d_count, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));

  // 3. FULL: unmatched build rows. With build row ids written: the build rows no INNER row names
  // (one bit per build row, set from the INNER rows' build row ids), else — or when the INNER rows
  // overflowed the capacity, decided on the device — the slots (groups) no probe row matched
  Scratch flags, bbits;
  if (full) {
    const int64_t ns = t->num_slots();
    const int64_t nflags = ns + 1;  // + the NULL group
    SJ_TRY(flags.get(alloc, (size_t)nflags, s));
    SJ_CUDA_TRY(cudaMemsetAsync(flags.ptr, 0, (size_t)nflags, s));
    const bool bits_ok = gs.out_build_rid != nullptr && gs.capacity > 0 && t->build_rows > 0;
    if (bits_ok) {
      const size_t words = (size_t)((t->build_rows + 31) / 32);
      SJ_TRY(bbits.get(alloc, words * sizeof(uint32_t), s));
      SJ_CUDA_TRY(cudaMemsetAsync(bbits.ptr, 0, words * sizeof(uint32_t), s));
      KernelTimer timer("matched_build_bits", s);
      matched_bits_kernel<<<kind_grid(t, std::min<int64_t>(gs.capacity, p.num_rows)), 256, 0, s>>>(
          gs.out_build_rid, m, gs.capacity, bbits.as<uint32_t>());
    }
    KindArgs fa{};
    fa.flags = flags.as<uint8_t>();
    fa.capacity = gs.capacity;
    fa.inner_rows = bits_ok ? m : nullptr;  // the flags pass returns at once when the bits apply
    if (p.num_rows > 0) launch_kind<kFlags>(t, p, fa, s);
    BuildEmitArgs e{};
    e.out_prid = gs.out_probe_rid;
    e.out_brid = gs.out_build_rid;
    e.n_bin = gs.n_build_payload;
    for (int c = 0; c < e.n_bin; ++c) {
      const sj_column& in = gs.build_payload[c];
      SJ_TRY(validate_column(&in, "build payload", false));
      if (in.num_rows != t->build_rows) return set_error(SJ_ERR_INVALID, "build payload row count differs from its key column");
      if (gs.out_build_payload[c].type != in.type) return set_error(SJ_ERR_INVALID, "build output type differs");
      e.bin[c] = column_payload(in.data, in.validity, in.validity_offset, type_width(in.type));
      e.bout[c] = PayloadOut{gs.out_build_payload[c].data, in.validity ? gs.out_build_payload[c].validity : nullptr};
    }
    e.pos_rid = t->pos_rid;
    e.pos_stride = t->pos_stride;
    e.capacity = gs.capacity;
    e.d_count = dc;
    e.flags = fa.flags;
    e.inner_rows = bits_ok ? m : nullptr;
    e.matched = bits_ok ? bbits.as<uint32_t>() : nullptr;
    const TableDev d = table_dev(t);
    KernelTimer timer("unmatched_build", s);
    if (bits_ok)
      unmatched_build_rows_kernel<<<kind_grid(t, t->build_rows), kKindThreads, 0, s>>>(e.matched, t->build_rows, e);
    if (t->layout == SJ_LAYOUT_DISTINCT) {
      if (ns > 0) {
        if (t->slot_kind == SJ_SLOT_WIDE128) unmatched_slots_kernel<true><<<kind_grid(t, ns), kKindThreads, 0, s>>>(d, ns, e);
        else unmatched_slots_kernel<false><<<kind_grid(t, ns), kKindThreads, 0, s>>>(d, ns, e);
      }
    } else {
      const int64_t members = t->valid_rows + (d.null_group >= 0 ? t->null_rows : 0);
      if (members > 0)
        unmatched_members_kernel<<<kind_grid(t, members), kKindThreads, 0, s>>>(d, members, ns + 1, e);
    }
    if (t->null_rid && t->null_rows > 0)
      null_build_rows_kernel<<<kind_grid(t, t->null_rows), kKindThreads, 0, s>>>(t->null_rid, t->null_rows, e);
  }

  // 4. validity of payload columns whose inputs have no NULLs (NULL padding by row range)
  const unsigned long long* total = dc;
  auto range = [&](uint32_t* words, const unsigned long long* lo, const unsigned long long* hi) {
    if (!words || gs.capacity == 0) return;
    const int64_t nw = (gs.capacity + 31) / 32;
    const int g = (int)std::max<int64_t>(1, std::min<int64_t>((nw + 255) / 256, (int64_t)sm_count(t->device) * 4));
    set_valid_range_kernel<<<g, 256, 0, s>>>(words, lo, hi, gs.capacity);
  };
  for (int c = 0; c < gs.n_build_payload; ++c) {
    const bool nullable = attached ? t->apay_valid[c] != nullptr : gs.build_payload[c].validity != nullptr;
    if (nullable) continue;
    range(gs.out_build_payload[c].validity, nullptr, m);      // INNER rows
    if (full) range(gs.out_build_payload[c].validity, m + 1, total);  // unmatched build rows
  }
  for (int c = 0; full && c < gs.n_probe_payload; ++c) {
    if (gs.probe_payload[c].validity) continue;
    range(gs.out_probe_payload[c].validity, nullptr, m + 1);  // INNER + unmatched probe rows
  }
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
