// Device-side building blocks of the sm_100a equi-hash-join: hashing, the slot encodings,
// bucket loads, validity bits, warp-aggregated output reservation and the payload gather.
//
// Table geometry. The open-addressing table is an array of 32-byte buckets (one DRAM sector).
//   PACKED64: a bucket holds 4 slots of uint64 = ((key - key_min) << rid_bits) | row_id.
//             EMPTY = all ones; the key field never reaches all ones (the build checks
//             key_max - key_min + 1 < 2^(64 - rid_bits)), so EMPTY never equals a live slot.
//   WIDE128:  a bucket holds 2 slots of {uint64 key, uint64 row_id}; EMPTY = {~0, ~0}; a slot
//             is live iff row_id != ~0.
// A key's home bucket is the top log2_nb bits of mix64(key); probing walks buckets linearly and
// wraps inside its segment of 2^seg_log2 buckets (the whole table unless partitioned; with radix
// partitioning the top partition bits of the hash select the segment). Inserts fill a bucket's
// slots in order, so occupied slots form a prefix of each bucket and a probe can stop after the
// first bucket that still has an EMPTY slot.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sj {

constexpr uint64_t kEmpty       = ~0ull;
constexpr int kBucketBytes      = 32;
constexpr int kMaxPayload       = 8;
constexpr unsigned kFullMask    = 0xffffffffu;

// splitmix64 finalizer (Steele, Lea & Flood, "Fast Splittable Pseudorandom Number Generators",
// OOPSLA 2014): a bijective 64-bit mixer, so distinct keys never share a full hash.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

template <typename K>
__host__ __device__ __forceinline__ uint64_t key_u64(K k);
template <>
__host__ __device__ __forceinline__ uint64_t key_u64<int32_t>(int32_t k) {
  return (uint64_t)(uint32_t)k;
}
template <>
__host__ __device__ __forceinline__ uint64_t key_u64<int64_t>(int64_t k) {
  return (uint64_t)k;
}

// Per-launch, by-value view of a built table.
struct TableDev {
  const void* slots;
  const int32_t* grp_off;  // GROUPED only
  const int32_t* grp_rid;  // GROUPED only
  int64_t kmin, kmax;      // valid key range; kmax < kmin for an empty table
  uint32_t log2_nb;
  uint32_t segmask;        // (1 << seg_log2) - 1
  uint32_t rbits;
  int32_t null_group;      // slot index of the NULL group (nulls equal) or -1
};

__device__ __forceinline__ uint32_t home_bucket(const TableDev& t, uint64_t kb) {
  return t.log2_nb ? (uint32_t)(mix64(kb) >> (64 - t.log2_nb)) : 0u;
}
__device__ __forceinline__ uint32_t next_bucket(uint32_t b, uint32_t segmask) {
  return (b & ~segmask) | ((b + 1) & segmask);
}

template <typename K>
__device__ __forceinline__ bool in_range(const TableDev& t, K k) {
  return (int64_t)k >= t.kmin && (int64_t)k <= t.kmax;
}

// ---- buckets -----------------------------------------------------------------------------------
struct Bucket {
  uint64_t a[4];  // PACKED64: 4 slots; WIDE128: {key0, rid0, key1, rid1}
};

template <bool NC>
__device__ __forceinline__ Bucket load_bucket(const void* slots, uint32_t b) {
  const ulonglong2* p = reinterpret_cast<const ulonglong2*>(slots) + (size_t)b * 2;
  ulonglong2 x, y;
  if (NC) {
    x = __ldg(p);
    y = __ldg(p + 1);
  } else {
    x = __ldcg(p);
    y = __ldcg(p + 1);
  }
  Bucket r;
  r.a[0] = x.x;
  r.a[1] = x.y;
  r.a[2] = y.x;
  r.a[3] = y.y;
  return r;
}

template <bool WIDE>
struct SlotOps;

template <>
struct SlotOps<false> {
  static constexpr int kSlots = 4;
  __device__ __forceinline__ static bool empty(const Bucket& bk, int q) { return bk.a[q] == kEmpty; }
  __device__ __forceinline__ static bool match(const Bucket& bk, int q, uint64_t kn, uint64_t, uint32_t rbits) {
    return bk.a[q] != kEmpty && (bk.a[q] >> rbits) == kn;
  }
  __device__ __forceinline__ static int32_t rid(const Bucket& bk, int q, uint32_t rbits) {
    return (int32_t)(bk.a[q] & ((1ull << rbits) - 1));
  }
};

template <>
struct SlotOps<true> {
  static constexpr int kSlots = 2;
  __device__ __forceinline__ static bool empty(const Bucket& bk, int q) { return bk.a[2 * q + 1] == kEmpty; }
  __device__ __forceinline__ static bool match(const Bucket& bk, int q, uint64_t, uint64_t kb, uint32_t) {
    return bk.a[2 * q + 1] != kEmpty && bk.a[2 * q] == kb;
  }
  __device__ __forceinline__ static int32_t rid(const Bucket& bk, int q, uint32_t) {
    return (int32_t)bk.a[2 * q + 1];
  }
};

// 128-bit compare-and-swap (PTX atom.cas.b128, sm_90+). Returns the previous 16 bytes.
__device__ __forceinline__ void cas128(void* addr, uint64_t cmp_lo, uint64_t cmp_hi, uint64_t new_lo,
                                       uint64_t new_hi, uint64_t& old_lo, uint64_t& old_hi) {
  asm volatile(
      "{\n\t.reg .b128 c, s, o;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 s, {%4, %5};\n\t"
      "atom.global.cas.b128 o, [%6], c, s;\n\t"
      "mov.b128 {%0, %1}, o;\n\t}"
      : "=l"(old_lo), "=l"(old_hi)
      : "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi), "l"(addr)
      : "memory");
}

// ---- validity bits -----------------------------------------------------------------------------
__device__ __forceinline__ bool bit_valid(const uint32_t* v, int64_t off, int64_t i) {
  if (v == nullptr) return true;
  const int64_t b = off + i;
  return (__ldg(v + (b >> 5)) >> (b & 31)) & 1u;
}

// ---- warp helpers ------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t o = __shfl_up_sync(kFullMask, v, d);
    if (lane >= d) v += o;
  }
  return v;
}

// Warp-aggregated reservation: every lane passes its count; one atomicAdd per warp.
// Returns this lane's first output position. Must be called by all 32 lanes.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* counter, uint32_t cnt) {
  const int lane      = threadIdx.x & 31;
  const uint32_t incl = warp_inclusive_sum(cnt);
  const uint32_t tot  = __shfl_sync(kFullMask, incl, 31);
  unsigned long long base = 0;
  if (tot) {
    if (lane == 0) base = atomicAdd(counter, (unsigned long long)tot);
    base = __shfl_sync(kFullMask, base, 0);
  }
  return base + (incl - cnt);
}

// ---- payload gather --------------------------------------------------------------------------
struct PayloadIn {
  const void* data;
  const uint32_t* valid;
  int64_t voff;
  int32_t width;
  int32_t pad;
};
struct PayloadOut {
  void* data;
  uint32_t* valid;
};

struct GatherArgs {
  int32_t n_pin, n_bin;
  PayloadIn pin[kMaxPayload];
  PayloadIn bin[kMaxPayload];
  PayloadOut pout[kMaxPayload];
  PayloadOut bout[kMaxPayload];
  int32_t* out_prid;
  int32_t* out_brid;
  int64_t capacity;
  unsigned long long* d_count;
};

__device__ __forceinline__ uint64_t load_elem(const void* base, int64_t i, int w) {
  switch (w) {
    case 8: return __ldg(reinterpret_cast<const unsigned long long*>(base) + i);
    case 4: return __ldg(reinterpret_cast<const unsigned int*>(base) + i);
    case 2: return __ldg(reinterpret_cast<const unsigned short*>(base) + i);
    default: return __ldg(reinterpret_cast<const unsigned char*>(base) + i);
  }
}
__device__ __forceinline__ void store_elem(void* base, int64_t i, int w, uint64_t v) {
  switch (w) {
    case 8: reinterpret_cast<unsigned long long*>(base)[i] = v; break;
    case 4: reinterpret_cast<unsigned int*>(base)[i] = (unsigned int)v; break;
    case 2: reinterpret_cast<unsigned short*>(base)[i] = (unsigned short)v; break;
    default: reinterpret_cast<unsigned char*>(base)[i] = (unsigned char)v; break;
  }
}
// Streaming store for output columns that are written once and not re-read by this kernel.
__device__ __forceinline__ void store_elem_cs(void* base, int64_t i, int w, uint64_t v) {
  switch (w) {
    case 8: __stcs(reinterpret_cast<unsigned long long*>(base) + i, (unsigned long long)v); break;
    case 4: __stcs(reinterpret_cast<unsigned int*>(base) + i, (unsigned int)v); break;
    case 2: __stcs(reinterpret_cast<unsigned short*>(base) + i, (unsigned short)v); break;
    default: reinterpret_cast<unsigned char*>(base)[i] = (unsigned char)v; break;
  }
}

__device__ __forceinline__ void set_out_bit(uint32_t* mask, int64_t pos) {
  atomicOr(mask + (pos >> 5), 1u << (pos & 31));
}

}  // namespace sj
