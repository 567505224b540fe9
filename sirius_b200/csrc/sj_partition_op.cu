// Hash partitioning of a table (the partition operator's hash_partition,
// src/op/partition/gpu_partition_impl.cpp:29-110, which feeds partitioned joins): rows are
// reordered so that partition p occupies [offsets[p], offsets[p+1]). It runs the join's own
// radix partition (sj_partition.cu: per-CTA histogram, scan, shared-memory counting-sort scatter)
// on a 64-bit partition key:
//   - one key column without NULLs: the key itself (the partition is the top bits of mix64(key),
//     the same function that splits a partitioned hash table into segments);
//   - NULLs or several key columns: a folded key (k0, then mix64(h) ^ k_c per further column), and
//     0 for a row with any NULL key column — mix64(0) = 0, so NULL-key rows all land in partition 0.
// Equal key tuples always land in the same partition, whichever table they come from.
#include <algorithm>
#include <string>

#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_partition.cuh"

namespace sj {

struct FoldCols {
  const void* data[kMaxKeyColumns];
  const uint32_t* valid[kMaxKeyColumns];
  int64_t voff[kMaxKeyColumns];
  int32_t is64[kMaxKeyColumns];
  int32_t n;
};

__global__ void __launch_bounds__(256) fold_keys_kernel(FoldCols k, int64_t n, unsigned long long* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t h = 0;
    bool null = false;
    for (int c = 0; c < k.n; ++c) {
      if (!bit_valid(k.valid[c], k.voff[c], i)) {
        null = true;
        break;
      }
      const uint64_t v = k.is64[c] ? (uint64_t)__ldg(static_cast<const long long*>(k.data[c]) + i)
                                   : (uint64_t)(int64_t)__ldg(static_cast<const int*>(k.data[c]) + i);
      h = c == 0 ? v : (mix64(h) ^ v);
    }
    out[i] = null ? 0ull : h;
  }
}

// validity bytes (one per row) -> cuDF bitmask words
__global__ void __launch_bounds__(256) bytes_to_bits_kernel(const uint8_t* __restrict__ b, int64_t n, uint32_t* w) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n;
       i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + lane;
    const unsigned word = __ballot_sync(kFullMask, i < n && b[i] != 0);
    if (lane == 0) w[i0 >> 5] = word;
  }
}

// partition starts: offsets[p] = off[p * G] (partition-major offsets of the scan), offsets[P] = total
__global__ void partition_starts_kernel(const int64_t* off, const int64_t* total, int P, int G, int64_t* out) {
  for (int p = threadIdx.x; p <= P; p += blockDim.x) out[p] = p < P ? off[(int64_t)p * G] : *total;
}

sj_status hash_partition(const sj_column* keys, int n_keys, const sj_column* cols, int n_cols, int n_parts,
                         const sj_mut_column* out, int64_t* d_offsets, const Allocator& alloc, cudaStream_t s) {
  if (n_keys < 1 || n_keys > kMaxKeyColumns) return set_error(SJ_ERR_INVALID, "1 to 4 key columns");
  if (n_cols < 0 || n_cols > kMaxPayload) return set_error(SJ_ERR_INVALID, "at most 8 columns to partition");
  if (n_parts < 1 || n_parts > (1 << kMaxPartitionBits) || (n_parts & (n_parts - 1)))
    return set_error(SJ_ERR_INVALID, "num_partitions must be a power of two in [1, 1024]");
  if (!d_offsets) return set_error(SJ_ERR_INVALID, "offsets is NULL");
  const int64_t n = keys[0].num_rows;
  for (int c = 0; c < n_keys; ++c) {
    SJ_TRY(validate_column(&keys[c], "key", true));
    if (keys[c].num_rows != n) return set_error(SJ_ERR_INVALID, "key columns differ in row count");
  }
  if (n > INT32_MAX) return set_error(SJ_ERR_INVALID, "more rows than the int32 row-id range");
  for (int c = 0; c < n_cols; ++c) {
    SJ_TRY(validate_column(&cols[c], "column", false));
    if (cols[c].num_rows != n) return set_error(SJ_ERR_INVALID, "columns differ in row count from the keys");
    if (!out || out[c].type != cols[c].type) return set_error(SJ_ERR_INVALID, "output column type differs");
    if (n > 0 && !out[c].data) return set_error(SJ_ERR_INVALID, "output column data is NULL");
    if (cols[c].validity && n > 0 && !out[c].validity)
      return set_error(SJ_ERR_INVALID, "column has NULLs but its output has no validity");
  }
  int pbits = 0;
  while ((1 << pbits) < n_parts) ++pbits;
  int device = 0;
  cudaGetDevice(&device);
  const bool folded = n_keys > 1 || keys[0].validity != nullptr;
  const int kw = folded || keys[0].type == SJ_INT64 ? 8 : 4;
  auto a256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
  size_t bytes = a256((size_t)std::max<int64_t>(n, 1) * kw) * (folded ? 2 : 1)  // folded key + partitioned keys
                 + a256((size_t)std::max<int64_t>(n, 1) * 4)                     // row ids
                 + partition_scratch_bytes(pbits, device);
  for (int c = 0; c < n_cols; ++c) bytes += cols[c].validity ? a256((size_t)std::max<int64_t>(n, 1)) : 0;
  Scratch sc;
  SJ_TRY(sc.get(alloc, bytes, s));
  char* cur = sc.as<char>();
  auto carve = [&](size_t b) {
    char* r = cur;
    cur += a256(b);
    return r;
  };
  const void* key_data = keys[0].data;
  const int key_type = folded ? SJ_INT64 : keys[0].type;
  if (folded) {
    FoldCols f{};
    f.n = n_keys;
    for (int c = 0; c < n_keys; ++c) {
      f.data[c] = keys[c].data;
      f.valid[c] = keys[c].validity;
      f.voff[c] = keys[c].validity_offset;
      f.is64[c] = keys[c].type == SJ_INT64;
    }
    unsigned long long* hk = reinterpret_cast<unsigned long long*>(carve((size_t)std::max<int64_t>(n, 1) * 8));
    if (n > 0) {
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
      fold_keys_kernel<<<grid, 256, 0, s>>>(f, n, hk);
    }
    key_data = hk;
  }
  PartSrc ps{};
  PartDst pd{};
  ps.keys = key_data;
  ps.n = n;
  ps.n_pay = n_cols;
  pd.keys = carve((size_t)std::max<int64_t>(n, 1) * kw);
  pd.rid = reinterpret_cast<int32_t*>(carve((size_t)std::max<int64_t>(n, 1) * 4));
  for (int c = 0; c < n_cols; ++c) {
    ps.pay[c] = column_payload(cols[c].data, cols[c].validity, cols[c].validity_offset, type_width(cols[c].type));
    pd.pay[c] = out[c].data;
    pd.valid8[c] = cols[c].validity ? reinterpret_cast<uint8_t*>(carve((size_t)std::max<int64_t>(n, 1))) : nullptr;
  }
  void* pscratch = carve(partition_scratch_bytes(pbits, device));
  const int64_t *d_total, *d_offs;
  int G;
  SJ_TRY(radix_partition(ps, key_type, pbits, pd, pscratch, device, s, &d_total, &d_offs, &G));
  partition_starts_kernel<<<1, 1024, 0, s>>>(d_offs, d_total, 1 << pbits, G, d_offsets);
  for (int c = 0; c < n_cols; ++c) {
    if (!pd.valid8[c] || n == 0) continue;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
    bytes_to_bits_kernel<<<grid, 256, 0, s>>>(pd.valid8[c], n, out[c].validity);
  }
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
