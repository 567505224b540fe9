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
// Keys enter the hash sign-extended to 64 bits, so an int32 key and its (key - key_min) + key_min
// reconstruction (the grouped build's shrink pass) hash identically.
template <>
__host__ __device__ __forceinline__ uint64_t key_u64<int32_t>(int32_t k) {
  return (uint64_t)(int64_t)k;
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

// One bucket = one 32-byte sector. Read-only probes fetch it with a single 256-bit load
// (ld.global.nc.v4.u64, sm_100); the build's insert pass reads it through L2 only (.cg) because
// other threads are CASing the same slots.
template <bool NC>
__device__ __forceinline__ Bucket load_bucket(const void* slots, uint32_t b) {
  Bucket r;
  const unsigned long long* p = reinterpret_cast<const unsigned long long*>(slots) + (size_t)b * 4;
  if (NC) {
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];"
        : "=l"(r.a[0]), "=l"(r.a[1]), "=l"(r.a[2]), "=l"(r.a[3])
        : "l"(p));
  } else {
    const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
    const ulonglong2 x = __ldcg(q), y = __ldcg(q + 1);
    r.a[0] = x.x;
    r.a[1] = x.y;
    r.a[2] = y.x;
    r.a[3] = y.y;
  }
  return r;
}

// L2 policy for table loads that should outlive the probe stream's lines in L2 (PTX createpolicy:
// every access through it is marked evict_last).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// load_bucket<true> with an L2 cache policy.
__device__ __forceinline__ Bucket load_bucket_hint(const void* slots, uint32_t b, uint64_t pol) {
  Bucket r;
  const unsigned long long* p = reinterpret_cast<const unsigned long long*>(slots) + (size_t)b * 4;
  asm("ld.global.nc.L2::cache_hint.v4.u64 {%0, %1, %2, %3}, [%4], %5;"
      : "=l"(r.a[0]), "=l"(r.a[1]), "=l"(r.a[2]), "=l"(r.a[3])
      : "l"(p), "l"(pol));
  return r;
}

// A row-store record of up to 32 bytes in one load (4, 8, 16 or 32 bytes, naturally aligned).
struct Record {
  uint32_t w[8];
};
__device__ __forceinline__ Record load_record(const void* p, int bytes) {
  Record r;
#pragma unroll
  for (int k = 0; k < 8; ++k) r.w[k] = 0;
  if (bytes == 32) {
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3]), "=r"(r.w[4]), "=r"(r.w[5]), "=r"(r.w[6]),
          "=r"(r.w[7])
        : "l"(p));
  } else if (bytes == 16) {
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
    r.w[0] = x.x;
    r.w[1] = x.y;
    r.w[2] = x.z;
    r.w[3] = x.w;
  } else if (bytes == 8) {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
    r.w[0] = x.x;
    r.w[1] = x.y;
  } else {
    r.w[0] = __ldg(reinterpret_cast<const unsigned int*>(p));
  }
  return r;
}
// Field of `width` bytes at byte offset `off` (aligned to its width) of a record, picked with
// predicated moves so the record stays in registers (no dynamic register indexing).
__device__ __forceinline__ uint64_t record_field(const Record& r, int off, int width) {
  const int wi = off >> 2;
  uint32_t lo = 0, hi = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    lo = (k == wi) ? r.w[k] : lo;
    hi = (k == wi + 1) ? r.w[k] : hi;
  }
  if (width == 8) return ((uint64_t)hi << 32) | lo;
  if (width == 4) return lo;
  const uint32_t v = lo >> ((off & 3) * 8);
  return width == 2 ? (v & 0xffffu) : (v & 0xffu);
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
  // Probe form: ks = (key - key_min) << rid_bits, kmask = ~(row-id mask). One masked compare;
  // EMPTY never matches because its key field is all ones and a live key field never is.
  __device__ __forceinline__ static uint64_t probe_key(uint64_t kn, uint64_t, uint32_t rbits) { return kn << rbits; }
  __device__ __forceinline__ static bool match_s(const Bucket& bk, int q, uint64_t ks, uint64_t kmask) {
    return (bk.a[q] & kmask) == ks;
  }
  // DISTINCT tables: a key occupies at most one slot, so the bucket is tested as a whole (32-bit
  // halves: rid_bits <= 31, so the row-id field lies in the low word) and the walk may stop once the
  // bucket's last slot is EMPTY (slots fill in order).
  __device__ __forceinline__ static bool match_distinct(const Bucket& bk, uint64_t ks, uint64_t kmask,
                                                        uint32_t rbits, int32_t& pos) {
    const uint32_t khi = (uint32_t)(ks >> 32), klo = (uint32_t)ks;
    const uint32_t mhi = (uint32_t)(kmask >> 32), mlo = (uint32_t)kmask;
    bool any = false;
    uint32_t sel = 0;
#pragma unroll
    for (int q = 0; q < kSlots; ++q) {
      const uint32_t hi = (uint32_t)(bk.a[q] >> 32), lo = (uint32_t)bk.a[q];
      const bool m = ((hi & mhi) == khi) & ((lo & mlo) == klo);
      sel = m ? lo : sel;
      any |= m;
    }
    pos = (int32_t)(sel & ((1u << rbits) - 1u));
    return any;
  }
  // GROUPED tables (one slot per distinct key): the bucket as a whole, returning the slot index.
  __device__ __forceinline__ static bool match_slot(const Bucket& bk, uint64_t ks, uint64_t kmask, int& slot) {
    const uint32_t khi = (uint32_t)(ks >> 32), klo = (uint32_t)ks;
    const uint32_t mhi = (uint32_t)(kmask >> 32), mlo = (uint32_t)kmask;
    bool any = false;
    int sel = 0;
#pragma unroll
    for (int q = 0; q < kSlots; ++q) {
      const uint32_t hi = (uint32_t)(bk.a[q] >> 32), lo = (uint32_t)bk.a[q];
      const bool m = ((hi & mhi) == khi) & ((lo & mlo) == klo);
      sel = m ? q : sel;
      any |= m;
    }
    slot = sel;
    return any;
  }
  __device__ __forceinline__ static bool open(const Bucket& bk) { return bk.a[kSlots - 1] == kEmpty; }
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
  __device__ __forceinline__ static uint64_t probe_key(uint64_t, uint64_t kb, uint32_t) { return kb; }
  __device__ __forceinline__ static bool match_s(const Bucket& bk, int q, uint64_t kb, uint64_t) {
    return bk.a[2 * q + 1] != kEmpty && bk.a[2 * q] == kb;
  }
  __device__ __forceinline__ static bool match_distinct(const Bucket& bk, uint64_t kb, uint64_t, uint32_t,
                                                        int32_t& pos) {
    const bool m0 = bk.a[1] != kEmpty && bk.a[0] == kb;
    const bool m1 = bk.a[3] != kEmpty && bk.a[2] == kb;
    pos = (int32_t)(m0 ? bk.a[1] : bk.a[3]);
    return m0 | m1;
  }
  __device__ __forceinline__ static bool match_slot(const Bucket& bk, uint64_t kb, uint64_t, int& slot) {
    const bool m0 = bk.a[1] != kEmpty && bk.a[0] == kb;
    const bool m1 = bk.a[3] != kEmpty && bk.a[2] == kb;
    slot = m0 ? 0 : 1;
    return m0 | m1;
  }
  __device__ __forceinline__ static bool open(const Bucket& bk) { return bk.a[3] == kEmpty; }
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

// ---- blocked Bloom filter ----------------------------------------------------------------------
// 2^log2_blocks blocks of 8 x 32-bit words (32 bytes = one DRAM sector). A key's block is the top
// bits of mix64(key) (the table's hash); a second mix of that hash gives 8 five-bit numbers, one
// bit per word.
constexpr uint64_t kBloomSalt = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ void bloom_locate(uint64_t kb, int log2_blocks, uint64_t& block, uint64_t& bits) {
  const uint64_t h = mix64(kb);
  block = log2_blocks ? h >> (64 - log2_blocks) : 0;
  bits = mix64(h + kBloomSalt);  // word w uses bits [5w, 5w + 5)
}

// The key's 8 bits, as 4 64-bit ORs: words 2k and 2k + 1 of the block are the low and high halves
// of its k-th 64-bit word (half the atomic operations of one OR per 32-bit word, same bits).
__device__ __forceinline__ void bloom_add(uint32_t* words, int log2_blocks, uint64_t kb) {
  uint64_t block, bits;
  bloom_locate(kb, log2_blocks, block, bits);
  unsigned long long* b = reinterpret_cast<unsigned long long*>(words + block * 8);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    atomicOr(b + k, (1ull << ((bits >> (10 * k)) & 31)) | (1ull << (32 + ((bits >> (10 * k + 5)) & 31))));
}

// ---- bounded waits -----------------------------------------------------------------------------
// Polls `*counter` (written by other CTAs) until it reaches `need`, sleeping ~128 ns between polls;
// gives up after `polls` polls and returns false. One thread calls it; the caller publishes the
// outcome to its CTA.
__device__ __forceinline__ bool wait_counter_at_least(const unsigned int* counter, unsigned need, unsigned polls) {
  unsigned spins = 0;
  while (*(const volatile unsigned int*)counter < need) {
    if (++spins > polls) return false;
    __nanosleep(128);
  }
  return true;
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
// A payload source: element i lives at data + i * stride (stride == width for a plain column,
// the record size for the table's interleaved row store).
struct PayloadIn {
  const void* data;
  const uint32_t* valid;   // cuDF bitmask (with voff), or NULL
  const uint8_t* valid8;   // validity byte of element i at valid8 + i * vstride, or NULL
  int64_t voff;
  int32_t width;
  int32_t stride;
  int32_t vstride;
  int32_t pad;
};
struct PayloadOut {
  void* data;
  uint32_t* valid;
};

__host__ __device__ inline PayloadIn column_payload(const void* data, const uint32_t* valid, int64_t voff, int w) {
  return PayloadIn{data, valid, nullptr, voff, w, w, 1, 0};
}

__device__ __forceinline__ bool has_validity(const PayloadIn& in) { return in.valid || in.valid8; }
__device__ __forceinline__ bool payload_valid(const PayloadIn& in, int64_t i) {
  if (in.valid8) return __ldg(in.valid8 + i * in.vstride) != 0;
  return bit_valid(in.valid, in.voff, i);
}

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
  const int32_t* prid_map;  // probe array index -> probe row id (partitioned probe), or NULL
  const int32_t* brid_map;  // build row id of table position p at brid_map + p * brid_stride bytes,
  int32_t brid_stride;      //   or NULL when positions are the row ids
  int32_t bin_by_pos;       // build payloads are the table's position-ordered attached copies
  // The table's row store when the attached build payloads live in records of <= 32 bytes: one
  // load per match returns the build row id and every attached field.
  const void* rec;
  int32_t rec_stride;
  int16_t rec_off[kMaxPayload];   // byte offset of attached column c inside a record
  int16_t rec_voff[kMaxPayload];  // byte offset of its validity byte, -1 when it has no NULLs
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

// Strided payload element (plain column or interleaved record field).
__device__ __forceinline__ uint64_t pl_load(const PayloadIn& in, int64_t i) {
  const void* a = static_cast<const char*>(in.data) + i * in.stride;
  switch (in.width) {
    case 8: return __ldg(reinterpret_cast<const unsigned long long*>(a));
    case 4: return __ldg(reinterpret_cast<const unsigned int*>(a));
    case 2: return __ldg(reinterpret_cast<const unsigned short*>(a));
    default: return __ldg(reinterpret_cast<const unsigned char*>(a));
  }
}
__device__ __forceinline__ int32_t brid_of(const GatherArgs& g, int32_t pos) {
  return g.brid_map ? __ldg(reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(g.brid_map) +
                                                               (int64_t)pos * g.brid_stride))
                    : pos;
}

__device__ __forceinline__ uint64_t load_elem_smem(const void* base, int64_t i, int w) {
  switch (w) {
    case 8: return reinterpret_cast<const unsigned long long*>(base)[i];
    case 4: return reinterpret_cast<const unsigned int*>(base)[i];
    case 2: return reinterpret_cast<const unsigned short*>(base)[i];
    default: return reinterpret_cast<const unsigned char*>(base)[i];
  }
}

__device__ __forceinline__ void set_out_bit(uint32_t* mask, int64_t pos) {
  atomicOr(mask + (pos >> 5), 1u << (pos & 31));
}

}  // namespace sj
