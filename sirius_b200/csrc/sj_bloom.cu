// Blocked Bloom filter built from the build keys and tested by the probe scan: the join's dynamic
// filter (src/cuda/sirius_dynamic_bloom_filter.cu: ~16 bits per key in 256-bit blocks, a BOOL8
// "may contain" mask per probe row with the probe's NULLs; published by the hash join,
// src/op/sirius_physical_hash_join.cpp:1960-2069).
//
// Layout (bloom_locate, sj_device.cuh): 2^log2_blocks blocks of 8 x 32-bit words (32 bytes = one
// DRAM sector). A key's block is the top bits of mix64(key); a second mix of that hash gives 8
// five-bit numbers, one bit per word. Insert: 8 atomicOr on one sector; test: one 256-bit load and
// 8 bit tests, so a probe row costs one sector read. NULL build keys are not inserted; NULL probe
// rows test false with a NULL mask. The same filter can come out of a table's build, set by its
// insert pass (sj_join_params.bloom_bits_per_key, sj_build.cu), instead of a second pass here.
#include <algorithm>
#include <string>

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

template <typename K>
__global__ void __launch_bounds__(256) bloom_insert_kernel(const K* __restrict__ keys, const uint32_t* kv, int64_t kvoff,
                                                           int64_t n, uint32_t* words, int log2_blocks) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!bit_valid(kv, kvoff, i)) continue;
    bloom_add(words, log2_blocks, key_u64<K>(__ldg(keys + i)));
  }
}

template <typename K>
__global__ void __launch_bounds__(256) bloom_test_kernel(const K* __restrict__ keys, const uint32_t* kv, int64_t kvoff,
                                                         int64_t n, const uint32_t* __restrict__ words, int log2_blocks,
                                                         uint8_t* out, uint32_t* out_valid) {
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; i0 < n;
       i0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = i0 + lane;
    const bool valid = i < n && bit_valid(kv, kvoff, i);
    bool hit = false;
    if (valid) {
      uint64_t block, bits;
      bloom_locate(key_u64<K>(__ldg(keys + i)), log2_blocks, block, bits);
      uint32_t w[8];
      asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
          : "l"(words + block * 8));
      hit = true;
#pragma unroll
      for (int q = 0; q < 8; ++q) hit &= (w[q] >> ((bits >> (5 * q)) & 31)) & 1u;
    }
    if (i < n) out[i] = hit ? 1 : 0;
    if (out_valid) {
      const unsigned word = __ballot_sync(kFullMask, valid);
      if (lane == 0) out_valid[i0 >> 5] = word;
    }
  }
}

static int grid_of(int device, int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(device) * 8));
}

sj_status bloom_create(int64_t n_keys, int32_t bits_per_key, int32_t key_type, const Allocator& alloc, cudaStream_t s,
                       sj_bloom** out) {
  *out = nullptr;
  if (bits_per_key <= 0) bits_per_key = 16;
  if (bits_per_key > 1024) return set_error(SJ_ERR_INVALID, "bits_per_key must be in [1, 1024]");
  sj_bloom* b = new sj_bloom();
  b->alloc = alloc;
  cudaGetDevice(&b->device);
  b->key_type = key_type;
  b->keys = n_keys;
  const uint64_t want_bits = (uint64_t)std::max<int64_t>(n_keys, 1) * (uint64_t)bits_per_key;
  while (b->log2_blocks < 40 && ((uint64_t)256 << b->log2_blocks) < want_bits) ++b->log2_blocks;
  b->bytes = (size_t)32 << b->log2_blocks;
  if (sj_status e = b->alloc.allocate((void**)&b->words, b->bytes, s)) {
    delete b;
    return e;
  }
  if (cudaMemsetAsync(b->words, 0, b->bytes, s) != cudaSuccess) {
    bloom_free(b, s);
    return set_error(SJ_ERR_DEVICE, "bloom filter memset failed");
  }
  *out = b;
  return SJ_OK;
}

void bloom_free(sj_bloom* b, cudaStream_t s) {
  if (!b) return;
  if (b->words) b->alloc.release(b->words, b->bytes, s);
  delete b;
}

}  // namespace sj

using namespace sj;

extern "C" {

SJ_EXPORT sj_status sj_bloom_build(const sj_column* keys, int32_t bits_per_key, const sj_alloc* alloc,
                                   sj_stream_t stream, sj_bloom** out) {
  clear_error();
  if (!out || !keys) return set_error(SJ_ERR_INVALID, "keys and out are required");
  *out = nullptr;
  SJ_TRY(validate_column(keys, "bloom key", true));
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  sj_bloom* b = nullptr;
  SJ_TRY(bloom_create(keys->num_rows, bits_per_key, keys->type, Allocator(alloc), s, &b));
  const int64_t n = keys->num_rows;
  if (n > 0) {
    KernelTimer timer("bloom_build", s);
    if (keys->type == SJ_INT32)
      bloom_insert_kernel<int32_t><<<grid_of(b->device, n), 256, 0, s>>>(
          static_cast<const int32_t*>(keys->data), keys->validity, keys->validity_offset, n, b->words, b->log2_blocks);
    else
      bloom_insert_kernel<int64_t><<<grid_of(b->device, n), 256, 0, s>>>(
          static_cast<const int64_t*>(keys->data), keys->validity, keys->validity_offset, n, b->words, b->log2_blocks);
  }
  if (cudaGetLastError() != cudaSuccess) {
    bloom_free(b, s);
    return set_error(SJ_ERR_DEVICE, "bloom filter build launch failed");
  }
  *out = b;
  return SJ_OK;
}

SJ_EXPORT sj_status sj_bloom_contains(const sj_bloom* bloom, const sj_column* probe_keys, uint8_t* out_mask,
                                      uint32_t* out_validity, sj_stream_t stream) {
  clear_error();
  if (!bloom || !probe_keys) return set_error(SJ_ERR_INVALID, "bloom and probe_keys are required");
  SJ_TRY(validate_column(probe_keys, "probe key", true));
  if (probe_keys->type != bloom->key_type) return set_error(SJ_ERR_INVALID, "probe key type differs from the filter's");
  const int64_t n = probe_keys->num_rows;
  if (n > 0 && !out_mask) return set_error(SJ_ERR_INVALID, "out_mask is NULL");
  if (n == 0) return SJ_OK;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  KernelTimer timer("bloom_test", s);
  if (probe_keys->type == SJ_INT32)
    bloom_test_kernel<int32_t><<<grid_of(bloom->device, n), 256, 0, s>>>(
        static_cast<const int32_t*>(probe_keys->data), probe_keys->validity, probe_keys->validity_offset, n,
        bloom->words, bloom->log2_blocks, out_mask, out_validity);
  else
    bloom_test_kernel<int64_t><<<grid_of(bloom->device, n), 256, 0, s>>>(
        static_cast<const int64_t*>(probe_keys->data), probe_keys->validity, probe_keys->validity_offset, n,
        bloom->words, bloom->log2_blocks, out_mask, out_validity);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

SJ_EXPORT int64_t sj_bloom_bytes(const sj_bloom* bloom) { return bloom ? (int64_t)bloom->bytes : 0; }

SJ_EXPORT sj_status sj_bloom_destroy(sj_bloom* bloom, sj_stream_t stream) {
  bloom_free(bloom, reinterpret_cast<cudaStream_t>(stream));
  return SJ_OK;
}

SJ_EXPORT const sj_bloom* sj_table_bloom(const sj_table* table) { return table ? table->bloom : nullptr; }

}  // extern "C"
