// Host-side internals shared by the sj translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "sj/sj_join.h"

namespace sj {

// ---- errors --------------------------------------------------------------------------------
// Every ABI entry point records a message for its thread before returning a failure status.
sj_status set_error(sj_status st, const std::string& msg);
void clear_error();

#define SJ_CUDA_TRY(expr)                                                                     \
  do {                                                                                        \
    cudaError_t sj_e_ = (expr);                                                               \
    if (sj_e_ != cudaSuccess) {                                                               \
      return ::sj::set_error(SJ_ERR_DEVICE, std::string(#expr " failed: ") +                  \
                                              cudaGetErrorString(sj_e_));                     \
    }                                                                                         \
  } while (0)

#define SJ_TRY(expr)                  \
  do {                                \
    sj_status sj_s_ = (expr);         \
    if (sj_s_ != SJ_OK) return sj_s_; \
  } while (0)

// ---- memory ----------------------------------------------------------------------------------
// All device memory goes through the caller's sj_alloc (or cudaMallocAsync when it is NULL).
struct Allocator {
  sj_alloc a{};
  bool use_default = true;
  explicit Allocator(const sj_alloc* user = nullptr);
  // Returns SJ_ERR_OOM (and records a message) when the allocation fails.
  sj_status allocate(void** p, size_t bytes, cudaStream_t s) const;
  void release(void* p, size_t bytes, cudaStream_t s) const;
};

// RAII scratch buffer released on scope exit (stream-ordered).
struct Scratch {
  const Allocator* alloc = nullptr;
  cudaStream_t stream    = nullptr;
  void* ptr              = nullptr;
  size_t bytes           = 0;
  Scratch() = default;
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  sj_status get(const Allocator& a, size_t n, cudaStream_t s) {
    alloc = &a;
    stream = s;
    bytes = n < 16 ? 16 : n;
    return a.allocate(&ptr, bytes, s);
  }
  ~Scratch() {
    if (ptr) alloc->release(ptr, bytes, stream);
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

// ---- opt-in per-kernel timing (sj_timing_enable / sj_timing_collect) ---------------------------
// While enabled, every KernelTimer scope records a CUDA event pair on its stream around the
// launch it wraps; the calling thread collects the durations later. Off by default: no events.
bool timing_enabled();
struct KernelTimer {
  KernelTimer(const char* name, cudaStream_t s);
  ~KernelTimer();
  KernelTimer(const KernelTimer&) = delete;
  KernelTimer& operator=(const KernelTimer&) = delete;
  int idx = -1;
  cudaStream_t stream = nullptr;
};

int sm_count(int device);
int type_width(int32_t t);  // bytes per element, 0 if invalid

// ---- the table -------------------------------------------------------------------------------
}  // namespace sj

namespace sj {
constexpr int kMaxKeyColumns = 4;
// Packing of a composite key (sj_keys.cu): column c's code (key - kmin[c], or null_code[c] for a
// NULL when NULLs compare equal) at bit shift[c]. n <= 1: a single key column, no packing.
struct KeyPack {
  int32_t n;
  int32_t nulls_equal;
  int32_t bits_total;
  int32_t shift[kMaxKeyColumns];
  int64_t kmin[kMaxKeyColumns];
  uint64_t null_code[kMaxKeyColumns];  // = max - min + 1 of the build's valid values
};
}  // namespace sj

struct sj_bloom {
  int device = 0;
  sj::Allocator alloc;
  uint32_t* words = nullptr;
  size_t bytes = 0;
  int32_t log2_blocks = 0;
  int32_t key_type = SJ_INT64;
  int64_t keys = 0;
};

struct sj_table {
  int device = 0;
  sj::Allocator alloc;
  int32_t key_type   = SJ_INT64;
  int32_t layout     = SJ_LAYOUT_DISTINCT;
  int32_t slot_kind  = SJ_SLOT_PACKED64;
  int32_t null_eq    = SJ_NULLS_UNEQUAL;
  int64_t build_rows = 0, valid_rows = 0, null_rows = 0, distinct = 0;
  int64_t kmin = 0, kmax = -1;
  int32_t rid_bits   = 1;
  int32_t log2_nb    = 0;  // log2(#buckets)
  int32_t seg_log2   = 0;  // log2(#buckets per probing segment); == log2_nb unless partitioned
  int32_t pbits      = 0;  // radix bits of the partitioned variant
  int32_t max_group  = 1;
  void* slots        = nullptr;  // #buckets * 32 bytes
  size_t slots_bytes = 0;
  int32_t* grp_off   = nullptr;  // GROUPED: #slots + 2 offsets (group #slots = NULL keys)
  size_t grp_off_bytes = 0;
  int32_t* grp_rid   = nullptr;  // GROUPED: table positions ordered by group; NULL when the row
                                  // store is in group order (position = index in group order)
  size_t grp_rid_bytes = 0;
  // Table positions. A slot's row-id field holds a position; the build row id of position p is
  // the int32 at pos_rid + p * pos_stride bytes (pos_rid NULL: positions are the row ids). With
  // radix partitioning positions follow partition order, so a partition's rows are contiguous.
  int32_t* pos_rid   = nullptr;
  int32_t pos_stride = 4;
  // Row store, one record of arow_stride bytes (a power of two) per position:
  //   [build row id (int32) | one validity byte per nullable attached column | attached payload
  //    fields, each aligned to its width]
  // so a match reads its row id and all its attached payloads from one record.
  void* arow         = nullptr;
  size_t arow_bytes  = 0;
  int32_t arow_stride = 0;
  // Attached build payload columns: field views into the row store, or (when positions are the
  // row ids, i.e. NULLs are equal and the build has NULL keys) owned column copies.
  int32_t n_attached = 0;
  int32_t apay_type[8] = {};
  void* apay[8]      = {};
  int32_t apay_stride[8] = {};
  uint8_t* apay_valid[8] = {};
  int32_t apay_vstride[8] = {};
  bool apay_owned    = false;
  // Row ids of the NULL-key build rows when NULLs never match (they are not in the table; a FULL
  // join emits them as unmatched rows). Built only when the build has NULL keys.
  int32_t* null_rid  = nullptr;
  size_t null_rid_bytes = 0;
  sj_bloom* bloom    = nullptr;  // the dynamic filter set by the insert pass (bloom_bits_per_key > 0)
  size_t apay_bytes[8] = {};
  size_t apay_valid_bytes[8] = {};
  sj_join_params params{};
  sj::KeyPack kpack{};  // composite key packing (kpack.n >= 2) or none
  int64_t num_slots() const;
};

namespace sj {

// ---- kernel launchers (sj_build.cu / sj_probe.cu) ---------------------------------------------
sj_status build_table(const sj_column& keys, const sj_column* payload, int32_t n_payload,
                      const sj_join_params& p, const Allocator& alloc, cudaStream_t stream, sj_table** out);
sj_status destroy_table(sj_table* t, cudaStream_t stream);

// Probes of a radix-partitioned table with at least this many rows are partitioned too.
constexpr int64_t kMinPartitionedProbe = 1 << 16;

struct GatherSpec {
  const sj_column* probe_payload;
  int32_t n_probe_payload;
  const sj_column* build_payload;
  int32_t n_build_payload;
  int32_t* out_probe_rid;
  int32_t* out_build_rid;
  const sj_mut_column* out_probe_payload;
  const sj_mut_column* out_build_payload;
  int64_t capacity;
};

sj_status probe_count(const sj_table* t, const sj_column& probe, const Allocator& alloc,
                      cudaStream_t stream, int64_t* d_count);
sj_status probe_gather(const sj_table* t, const sj_column& probe, const GatherSpec& g,
                       const Allocator& alloc, cudaStream_t stream, int64_t* d_count);

sj_status validate_column(const sj_column* c, const char* what, bool key);

// Composite keys (sj_keys.cu): pack 2..4 key columns into one INT64 column held in `buf`.
sj_status pack_build_keys(const sj_column* keys, int n_keys, bool nulls_equal, const Allocator& alloc,
                          cudaStream_t s, KeyPack* kp, Scratch& buf, sj_column* packed);
// A single-column probe key of the other integer type, converted to the table's type `table_type`
// (int32 -> int64 exactly; int64 -> int32 exactly in range, else a value outside [kmin, kmax]).
sj_status cast_probe_keys(int32_t table_type, int64_t kmin, int64_t kmax, const sj_column& keys, const Allocator& alloc,
                          cudaStream_t s, Scratch& buf, sj_column* out);
sj_status pack_probe_keys(const KeyPack& kp, const sj_column* keys, int n_keys, const Allocator& alloc,
                          cudaStream_t s, Scratch& buf, sj_column* packed);

// Hash partitioning of a table (sj_partition_op.cu).
sj_status hash_partition(const sj_column* keys, int n_keys, const sj_column* cols, int n_cols, int n_parts,
                         const sj_mut_column* out, int64_t* d_offsets, const Allocator& alloc, cudaStream_t s);

// Blocked Bloom filter of n keys at `bits_per_key` (sj_bloom.cu): words allocated and zeroed on `s`.
sj_status bloom_create(int64_t n_keys, int32_t bits_per_key, int32_t key_type, const Allocator& alloc, cudaStream_t s,
                       sj_bloom** out);
void bloom_free(sj_bloom* b, cudaStream_t s);

// LEFT / SEMI / ANTI / MARK / FULL (sj_probe_kinds.cu); INNER delegates to probe_gather.
sj_status probe_join(const sj_table* t, int32_t kind, const sj_column& probe, const GatherSpec& g, uint8_t* out_mark,
                     uint32_t* out_mark_valid, const Allocator& alloc, cudaStream_t stream, int64_t* d_count);

}  // namespace sj
