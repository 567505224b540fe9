// Composite equi-join keys: 2..4 INT32/INT64 key columns packed into one INT64 key per row, so every
// table layout, probe kernel and join type runs on them unchanged (the reference's multi-column
// conditions, prepare_join_keys, src/op/sirius_physical_hash_join.cpp:1234-1291).
//
// Packing is exact: column c contributes (key_c - min_c) in `bits_c` bits, where min/max come from
// the build side's valid values, so two rows have equal packed keys iff all their key columns are
// equal. NULLs: with NULLs unequal a row with any NULL key column has a NULL packed key (it never
// matches, as in SQL); with NULLs equal (IS NOT DISTINCT FROM on every column) a NULL column takes
// its own code (max - min + 1), so rows match iff they agree column by column, NULL included.
// A probe value outside a column's build range cannot match: its row gets a packed key one past
// every build code. Keys whose ranges need more than 63 bits in total are refused.
#include <algorithm>
#include <climits>
#include <limits>
#include <string>

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

struct KeyCols {
  const void* data[kMaxKeyColumns];
  const uint32_t* valid[kMaxKeyColumns];
  int64_t voff[kMaxKeyColumns];
  int32_t is64[kMaxKeyColumns];
  int32_t n;
};

__device__ __forceinline__ int64_t key_at(const KeyCols& k, int c, int64_t i) {
  return k.is64[c] ? __ldg(static_cast<const long long*>(k.data[c]) + i)
                   : (int64_t)__ldg(static_cast<const int*>(k.data[c]) + i);
}

struct KeyRange {
  long long kmin[kMaxKeyColumns];
  long long kmax[kMaxKeyColumns];
};

__global__ void key_range_init_kernel(KeyRange* r) {
  for (int c = 0; c < kMaxKeyColumns; ++c) {
    r->kmin[c] = LLONG_MAX;
    r->kmax[c] = LLONG_MIN;
  }
}

// per-column min / max of the valid values (warp-reduced, one atomic per warp and column)
__global__ void __launch_bounds__(256) key_range_kernel(KeyCols k, int64_t n, KeyRange* r) {
  const int lane = threadIdx.x & 31;
  for (int c = 0; c < k.n; ++c) {
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      if (!bit_valid(k.valid[c], k.voff[c], i)) continue;
      const long long v = key_at(k, c, i);
      lo = v < lo ? v : lo;
      hi = v > hi ? v : hi;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      const long long olo = __shfl_down_sync(kFullMask, lo, d);
      const long long ohi = __shfl_down_sync(kFullMask, hi, d);
      lo = olo < lo ? olo : lo;
      hi = ohi > hi ? ohi : hi;
    }
    if (lane == 0) {
      if (lo != LLONG_MAX) atomicMin(&r->kmin[c], lo);
      if (hi != LLONG_MIN) atomicMax(&r->kmax[c], hi);
    }
  }
}

// Packs every row; validity words are written whole by one warp per 32 rows.
__global__ void __launch_bounds__(256) key_pack_kernel(KeyCols k, int64_t n, KeyPack kp, long long* out,
                                                       uint32_t* out_valid) {
  const int lane = threadIdx.x & 31;
  const uint64_t miss = kp.bits_total < 63 ? (1ull << kp.bits_total) : 0;
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n;
       i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + lane;
    bool valid = i < n;
    uint64_t code = 0;
    bool out_of_range = false;
    if (i < n) {
      for (int c = 0; c < k.n; ++c) {
        uint64_t v;
        if (!bit_valid(k.valid[c], k.voff[c], i)) {
          if (!kp.nulls_equal) {
            valid = false;
            continue;
          }
          v = kp.null_code[c];
        } else {
          const uint64_t d = (uint64_t)key_at(k, c, i) - (uint64_t)kp.kmin[c];
          if (d >= kp.null_code[c]) out_of_range = true;  // null_code = max - min + 1
          v = d;
        }
        code |= v << kp.shift[c];
      }
      out[i] = (long long)(out_of_range ? miss : code);
    }
    if (out_valid) {
      const unsigned w = __ballot_sync(kFullMask, valid && i < n);
      if (lane == 0) out_valid[i0 >> 5] = w;
    }
  }
}

static KeyCols key_cols(const sj_column* keys, int n_keys) {
  KeyCols k{};
  k.n = n_keys;
  for (int c = 0; c < n_keys; ++c) {
    k.data[c] = keys[c].data;
    k.valid[c] = keys[c].validity;
    k.voff[c] = keys[c].validity_offset;
    k.is64[c] = keys[c].type == SJ_INT64;
  }
  return k;
}

static sj_status check_key_columns(const sj_column* keys, int n_keys) {
  if (n_keys < 2 || n_keys > kMaxKeyColumns) return set_error(SJ_ERR_INVALID, "composite keys have 2 to 4 columns");
  for (int c = 0; c < n_keys; ++c) {
    SJ_TRY(validate_column(&keys[c], "key", true));
    if (keys[c].num_rows != keys[0].num_rows) return set_error(SJ_ERR_INVALID, "key columns differ in row count");
  }
  if (keys[0].num_rows > INT32_MAX) return set_error(SJ_ERR_INVALID, "more rows than the int32 row-id range");
  return SJ_OK;
}

static sj_status pack(const KeyCols& k, int64_t n, const KeyPack& kp, bool any_null, const Allocator& alloc,
                      cudaStream_t s, Scratch& buf, sj_column* packed, int device) {
  const size_t vb = (size_t)(n + 31) / 32 * 4;
  const size_t kb = ((size_t)std::max<int64_t>(n, 1) * 8 + 255) & ~(size_t)255;
  const bool need_valid = any_null && !kp.nulls_equal;
  SJ_TRY(buf.get(alloc, kb + (need_valid ? vb : 0) + 256, s));
  long long* out = buf.as<long long>();
  uint32_t* ov = need_valid ? reinterpret_cast<uint32_t*>(buf.as<char>() + kb) : nullptr;
  if (n > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
    key_pack_kernel<<<grid, 256, 0, s>>>(k, n, kp, out, ov);
    SJ_CUDA_TRY(cudaGetLastError());
  }
  *packed = sj_column{out, ov, 0, n, SJ_INT64, 0};
  return SJ_OK;
}

sj_status pack_build_keys(const sj_column* keys, int n_keys, bool nulls_equal, const Allocator& alloc,
                          cudaStream_t s, KeyPack* kp, Scratch& buf, sj_column* packed) {
  SJ_TRY(check_key_columns(keys, n_keys));
  int device = 0;
  cudaGetDevice(&device);
  const int64_t n = keys[0].num_rows;
  const KeyCols k = key_cols(keys, n_keys);
  Scratch rbuf;
  SJ_TRY(rbuf.get(alloc, sizeof(KeyRange), s));
  KeyRange* dr = rbuf.as<KeyRange>();
  key_range_init_kernel<<<1, 1, 0, s>>>(dr);
  if (n > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
    key_range_kernel<<<grid, 256, 0, s>>>(k, n, dr);
  }
  KeyRange h{};
  if (cudaMemcpyAsync(&h, dr, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
    return set_error(SJ_ERR_DEVICE, std::string("composite key ranges: ") + cudaGetErrorString(cudaGetLastError()));
  *kp = KeyPack{};
  kp->n = n_keys;
  kp->nulls_equal = nulls_equal ? 1 : 0;
  int shift = 0;
  bool any_null = false;
  for (int c = 0; c < n_keys; ++c) {
    any_null |= keys[c].validity != nullptr;
    uint64_t span = 0;  // distinct codes of valid values
    if (h.kmin[c] <= h.kmax[c]) {
      kp->kmin[c] = h.kmin[c];
      span = (uint64_t)h.kmax[c] - (uint64_t)h.kmin[c] + 1;  // 0 = the full 2^64 range
      if (span == 0) return set_error(SJ_ERR_INVALID, "composite key column spans the whole int64 range");
    }
    kp->null_code[c] = span;
    const uint64_t codes = span + (nulls_equal ? 1 : 0);
    int bits = 0;
    while (bits < 64 && (codes > 1 ? ((codes - 1) >> bits) != 0 : false)) ++bits;
    kp->shift[c] = shift;
    shift += bits;
    if (shift > 62) return set_error(SJ_ERR_INVALID, "composite key ranges need more than 63 bits; not packable");
  }
  kp->bits_total = shift;
  return pack(k, n, *kp, any_null, alloc, s, buf, packed, device);
}

sj_status pack_probe_keys(const KeyPack& kp, const sj_column* keys, int n_keys, const Allocator& alloc,
                          cudaStream_t s, Scratch& buf, sj_column* packed) {
  if (n_keys != kp.n) return set_error(SJ_ERR_INVALID, "probe has a different number of key columns than the build");
  SJ_TRY(check_key_columns(keys, n_keys));
  bool any_null = false;
  for (int c = 0; c < n_keys; ++c) any_null |= keys[c].validity != nullptr;
  int device = 0;
  cudaGetDevice(&device);
  return pack(key_cols(keys, n_keys), keys[0].num_rows, kp, any_null, alloc, s, buf, packed, device);
}

// ------------------------------------------------------------------------------------------------
// Single-column probe keys of the other integer type than the table's (the reference casts key
// columns to the join's comparison type, cudf::cast in prepare_join_keys,
// src/op/sirius_physical_hash_join.cpp:1272-1284). int32 into an int64 table widens exactly;
// int64 into an int32 table narrows values in the int32 range exactly and maps the others to
// `miss`, an int32 value outside the table's key range, so they never match (they stay non-NULL:
// LEFT, ANTI and MARK treat them as rows without a match). Validity passes through unchanged.
// ------------------------------------------------------------------------------------------------
template <typename In, typename Out>
__global__ void __launch_bounds__(256) key_cast_kernel(const In* __restrict__ in, int64_t n, Out* out, long long miss) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const long long v = (long long)__ldg(in + i);
    const bool fits = v >= (long long)std::numeric_limits<Out>::min() && v <= (long long)std::numeric_limits<Out>::max();
    out[i] = (Out)(fits ? v : miss);
  }
}

sj_status cast_probe_keys(int32_t table_type, int64_t kmin, int64_t kmax, const sj_column& keys, const Allocator& alloc,
                          cudaStream_t s, Scratch& buf, sj_column* out) {
  const int64_t n = keys.num_rows;
  long long miss = 0;
  if (table_type == SJ_INT32) {  // a value the table cannot hold
    if (kmax < kmin) miss = 0;  // no valid build key: nothing matches anyway
    else if (kmax < INT32_MAX) miss = kmax + 1;
    else if (kmin > INT32_MIN) miss = kmin - 1;
    else return set_error(SJ_ERR_INVALID, "int64 probe keys into an int32 table whose keys span the whole int32 range");
  }
  const size_t w = table_type == SJ_INT32 ? 4 : 8;
  SJ_TRY(buf.get(alloc, (size_t)std::max<int64_t>(n, 1) * w, s));
  *out = keys;
  out->data = buf.ptr;
  out->type = table_type;
  if (n == 0) return SJ_OK;
  int device = 0;
  cudaGetDevice(&device);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
  if (table_type == SJ_INT64)
    key_cast_kernel<int32_t, long long><<<grid, 256, 0, s>>>(static_cast<const int32_t*>(keys.data), n,
                                                             buf.as<long long>(), 0);
  else
    key_cast_kernel<long long, int32_t><<<grid, 256, 0, s>>>(static_cast<const long long*>(keys.data), n,
                                                             buf.as<int32_t>(), miss);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
