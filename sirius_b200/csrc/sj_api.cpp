// C ABI entry points of the join (declared in include/sj/sj_join.h). Each one validates its
// arguments, converts C++ failures into sj_status + a per-thread message, and never throws.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "sj_internal.h"

namespace sj {

static thread_local std::string g_last_error;

sj_status set_error(sj_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}
void clear_error() { g_last_error.clear(); }

Allocator::Allocator(const sj_alloc* user) {
  if (user && user->alloc && user->free) {
    a = *user;
    use_default = false;
  }
}

// The default allocator keeps freed blocks in the device's default memory pool (release threshold
// = unlimited) so per-call scratch is recycled instead of returned to the driver at every sync.
static void keep_default_pool(cudaStream_t s) {
  static std::mutex mu;
  static std::vector<char> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  if (done[dev]) return;
  done[dev] = 1;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  (void)s;
}

sj_status Allocator::allocate(void** p, size_t bytes, cudaStream_t s) const {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (use_default) {
    keep_default_pool(s);
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e != cudaSuccess || *p == nullptr) {
      cudaGetLastError();  // clear the non-sticky allocation error
      *p = nullptr;
      return set_error(SJ_ERR_OOM, "cudaMallocAsync of " + std::to_string(bytes) + " bytes failed");
    }
    return SJ_OK;
  }
  *p = a.alloc(a.ctx, bytes, reinterpret_cast<sj_stream_t>(s));
  if (*p == nullptr) return set_error(SJ_ERR_OOM, "allocator callback returned NULL for " + std::to_string(bytes) + " bytes");
  return SJ_OK;
}

void Allocator::release(void* p, size_t bytes, cudaStream_t s) const {
  if (!p) return;
  if (bytes == 0) bytes = 16;
  if (use_default) cudaFreeAsync(p, s);
  else a.free(a.ctx, p, bytes, reinterpret_cast<sj_stream_t>(s));
}

// ---- per-kernel timing --------------------------------------------------------------------
static std::atomic<bool> g_timing{false};
struct TimingRecord {
  const char* name;
  cudaEvent_t a, b;
};
static thread_local std::vector<TimingRecord> t_records;
static thread_local std::vector<cudaEvent_t> t_event_pool;

static cudaEvent_t pooled_event() {
  if (!t_event_pool.empty()) {
    cudaEvent_t e = t_event_pool.back();
    t_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

bool timing_enabled() { return g_timing.load(std::memory_order_relaxed); }

KernelTimer::KernelTimer(const char* name, cudaStream_t s) : stream(s) {
  if (!timing_enabled()) return;
  cudaEvent_t a = pooled_event(), b = pooled_event();
  if (!a || !b) return;
  cudaEventRecord(a, s);
  t_records.push_back(TimingRecord{name, a, b});
  idx = (int)t_records.size() - 1;
}

KernelTimer::~KernelTimer() {
  if (idx >= 0 && idx < (int)t_records.size()) cudaEventRecord(t_records[idx].b, stream);
}

int sm_count(int device) {
  static std::mutex mu;
  static std::vector<int> cache;
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0) device = 0;
  if ((int)cache.size() <= device) cache.resize(device + 1, 0);
  if (cache[device] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
    cache[device] = v;
  }
  return cache[device];
}

int type_width(int32_t t) {
  switch (t) {
    case SJ_INT8:
    case SJ_BOOL8: return 1;
    case SJ_INT16: return 2;
    case SJ_INT32:
    case SJ_FLOAT32:
    case SJ_UINT32: return 4;
    case SJ_INT64:
    case SJ_FLOAT64:
    case SJ_UINT64: return 8;
    default: return 0;
  }
}

sj_status validate_column(const sj_column* c, const char* what, bool key) {
  if (!c) return set_error(SJ_ERR_INVALID, std::string(what) + " column is NULL");
  if (c->num_rows < 0) return set_error(SJ_ERR_INVALID, std::string(what) + " column has negative num_rows");
  if (key) {
    if (c->type != SJ_INT32 && c->type != SJ_INT64)
      return set_error(SJ_ERR_INVALID, std::string(what) + " column must be INT32 or INT64");
  } else if (type_width(c->type) == 0) {
    return set_error(SJ_ERR_INVALID, std::string(what) + " column has an unknown type");
  }
  if (c->num_rows > 0 && c->data == nullptr)
    return set_error(SJ_ERR_INVALID, std::string(what) + " column data is NULL");
  if (c->validity_offset < 0) return set_error(SJ_ERR_INVALID, std::string(what) + " validity_offset < 0");
  const uintptr_t align = (uintptr_t)type_width(c->type);
  if (c->data && ((uintptr_t)c->data % align) != 0)
    return set_error(SJ_ERR_INVALID, std::string(what) + " column data is not aligned to its element size");
  return SJ_OK;
}

static sj_join_params resolve(const sj_join_params* p) {
  sj_join_params r;
  sj_default_params(&r);
  if (!p) return r;
  r.layout = p->layout;
  r.null_equality = p->null_equality;
  if (p->load_factor > 0.0f) r.load_factor = p->load_factor;
  if (p->block_size > 0) r.block_size = p->block_size;
  if (p->group_width > 0) r.group_width = p->group_width;
  r.partition_bits = p->partition_bits;
  r.force_wide = p->force_wide;
  if (p->ctas_per_sm > 0) r.ctas_per_sm = p->ctas_per_sm;
  r.aggregation = p->aggregation;
  r.probe_kernel = p->probe_kernel;
  r.rows_per_lane = p->rows_per_lane;
  r.probe_partition_mb = p->probe_partition_mb;
  r.table_l2_priority = p->table_l2_priority;
  r.bloom_bits_per_key = p->bloom_bits_per_key;
  return r;
}

}  // namespace sj

using namespace sj;

extern "C" {

SJ_EXPORT void sj_default_params(sj_join_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->layout = SJ_LAYOUT_AUTO;
  p->null_equality = SJ_NULLS_UNEQUAL;
  p->load_factor = 0.5f;
  p->block_size = 256;
  p->group_width = 1;
  p->partition_bits = 0;
  p->force_wide = 0;
  p->ctas_per_sm = 4;
}

SJ_EXPORT sj_status sj_build(const sj_column* keys, int32_t num_keys, const sj_join_params* params,
                             const sj_alloc* alloc, sj_stream_t stream, sj_table** out) {
  clear_error();
  if (!out) return set_error(SJ_ERR_INVALID, "out is NULL");
  *out = nullptr;
  return sj_build_ex(keys, num_keys, nullptr, 0, params, alloc, stream, out);
}

// Builds on keys[0], or on the packed composite key of 2..4 columns (the table keeps the packing).
static sj_status build_keys(const sj_column* keys, int32_t num_keys, const sj_column* payload, int32_t num_payload,
                            const sj_join_params& p, const Allocator& a, cudaStream_t s, sj_table** out) {
  if (num_keys == 1) return build_table(keys[0], payload, num_payload, p, a, s, out);
  if (p.bloom_bits_per_key > 0)
    return set_error(SJ_ERR_INVALID, "a build-time dynamic filter needs a single key column");
  KeyPack kp{};
  Scratch buf;
  sj_column packed{};
  SJ_TRY(pack_build_keys(keys, num_keys, p.null_equality == SJ_NULLS_EQUAL, a, s, &kp, buf, &packed));
  SJ_TRY(build_table(packed, payload, num_payload, p, a, s, out));
  (*out)->kpack = kp;
  return SJ_OK;
}

// The probe's key column: keys[0], or the composite key packed as the table's build was.
static sj_status probe_keys_of(const sj_table* t, const sj_column* keys, int32_t num_keys, const Allocator& a,
                               cudaStream_t s, Scratch& buf, sj_column* out) {
  if (t->kpack.n > 1) return pack_probe_keys(t->kpack, keys, num_keys, a, s, buf, out);
  if (num_keys != 1) return set_error(SJ_ERR_INVALID, "the table was built on one key column");
  if ((keys[0].type == SJ_INT32 || keys[0].type == SJ_INT64) && keys[0].type != t->key_type &&
      (t->key_type == SJ_INT32 || t->key_type == SJ_INT64)) {
    SJ_TRY(validate_column(&keys[0], "probe key", true));
    return cast_probe_keys(t->key_type, t->kmin, t->kmax, keys[0], a, s, buf, out);
  }
  *out = keys[0];
  return SJ_OK;
}

SJ_EXPORT sj_status sj_build_ex(const sj_column* keys, int32_t num_keys, const sj_column* payload,
                                int32_t num_payload, const sj_join_params* params, const sj_alloc* alloc,
                                sj_stream_t stream, sj_table** out) {
  clear_error();
  if (!out) return set_error(SJ_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (num_keys < 1 || num_keys > kMaxKeyColumns) return set_error(SJ_ERR_INVALID, "1 to 4 key columns");
  if (!keys) return set_error(SJ_ERR_INVALID, "keys is NULL");
  try {
    const sj_join_params p = resolve(params);
    const Allocator a(alloc);
    return build_keys(keys, num_keys, payload, num_payload, p, a, reinterpret_cast<cudaStream_t>(stream), out);
  } catch (const std::bad_alloc&) {
    return set_error(SJ_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}

SJ_EXPORT sj_status sj_table_destroy(sj_table* table, sj_stream_t stream) {
  clear_error();
  return destroy_table(table, reinterpret_cast<cudaStream_t>(stream));
}

SJ_EXPORT sj_status sj_table_get_info(const sj_table* t, sj_table_info* info) {
  clear_error();
  if (!t || !info) return set_error(SJ_ERR_INVALID, "table or info is NULL");
  std::memset(info, 0, sizeof(*info));
  info->build_rows = t->build_rows;
  info->valid_rows = t->valid_rows;
  info->null_rows = t->null_rows;
  info->distinct_keys = t->distinct;
  info->num_slots = t->num_slots();
  size_t bytes = t->slots_bytes + t->grp_off_bytes + t->grp_rid_bytes + t->arow_bytes + t->null_rid_bytes;
  if (t->apay_owned)
    for (int c = 0; c < t->n_attached; ++c) bytes += t->apay_bytes[c] + t->apay_valid_bytes[c];
  info->device_bytes = (int64_t)bytes;
  info->key_min = t->valid_rows ? t->kmin : 0;
  info->key_max = t->valid_rows ? t->kmax : -1;
  info->layout = t->layout;
  info->slot_kind = t->slot_kind;
  info->rid_bits = t->rid_bits;
  info->key_type = t->key_type;
  info->partition_bits = t->pbits;
  info->max_group = t->max_group;
  return SJ_OK;
}

SJ_EXPORT sj_status sj_probe_count(const sj_table* table, const sj_column* probe_keys, int32_t num_keys,
                                   const sj_alloc* alloc, sj_stream_t stream, int64_t* d_count) {
  clear_error();
  if (!table || !probe_keys || !d_count) return set_error(SJ_ERR_INVALID, "table, probe_keys and d_count are required");
  try {
    const Allocator a(alloc);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    Scratch buf;
    sj_column key{};
    SJ_TRY(probe_keys_of(table, probe_keys, num_keys, a, s, buf, &key));
    return probe_count(table, key, a, s, d_count);
  } catch (const std::exception& e) {
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}

SJ_EXPORT sj_status sj_probe_gather(const sj_table* table, const sj_column* probe_keys, int32_t num_keys,
                                    const sj_column* probe_payload, int32_t num_probe_payload,
                                    const sj_column* build_payload, int32_t num_build_payload,
                                    int32_t* out_probe_rid, int32_t* out_build_rid,
                                    const sj_mut_column* out_probe_payload, const sj_mut_column* out_build_payload,
                                    int64_t capacity, const sj_alloc* alloc, sj_stream_t stream, int64_t* d_count) {
  clear_error();
  if (!table || !probe_keys || !d_count) return set_error(SJ_ERR_INVALID, "table, probe_keys and d_count are required");
  GatherSpec g{probe_payload, num_probe_payload, build_payload, num_build_payload, out_probe_rid,
               out_build_rid, out_probe_payload, out_build_payload, capacity};
  try {
    const Allocator a(alloc);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    Scratch buf;
    sj_column key{};
    SJ_TRY(probe_keys_of(table, probe_keys, num_keys, a, s, buf, &key));
    return probe_gather(table, key, g, a, s, d_count);
  } catch (const std::exception& e) {
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}

SJ_EXPORT sj_status sj_probe_join(const sj_table* table, sj_join_kind kind, const sj_column* probe_keys,
                                  int32_t num_keys, const sj_column* probe_payload, int32_t num_probe_payload,
                                  const sj_column* build_payload, int32_t num_build_payload, int32_t* out_probe_rid,
                                  int32_t* out_build_rid, const sj_mut_column* out_probe_payload,
                                  const sj_mut_column* out_build_payload, int64_t capacity, uint8_t* out_mark,
                                  uint32_t* out_mark_validity, const sj_alloc* alloc, sj_stream_t stream,
                                  int64_t* d_count) {
  clear_error();
  if (!table || !probe_keys || !d_count) return set_error(SJ_ERR_INVALID, "table, probe_keys and d_count are required");
  GatherSpec g{probe_payload, num_probe_payload, build_payload, num_build_payload, out_probe_rid,
               out_build_rid, out_probe_payload, out_build_payload, capacity};
  try {
    const Allocator a(alloc);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    Scratch buf;
    sj_column key{};
    SJ_TRY(probe_keys_of(table, probe_keys, num_keys, a, s, buf, &key));
    return probe_join(table, (int32_t)kind, key, g, out_mark, out_mark_validity, a, s, d_count);
  } catch (const std::exception& e) {
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}

SJ_EXPORT sj_status sj_hash_partition(const sj_column* keys, int32_t num_keys, const sj_column* columns,
                                      int32_t num_columns, int32_t num_partitions, const sj_mut_column* out_columns,
                                      int64_t* d_offsets, const sj_alloc* alloc, sj_stream_t stream) {
  clear_error();
  if (!keys || (num_columns > 0 && !columns)) return set_error(SJ_ERR_INVALID, "keys and columns are required");
  try {
    return hash_partition(keys, num_keys, columns, num_columns, num_partitions, out_columns, d_offsets,
                          Allocator(alloc), reinterpret_cast<cudaStream_t>(stream));
  } catch (const std::exception& e) {
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}

SJ_EXPORT sj_status sj_inner_join(const sj_column* build_keys, const sj_column* probe_keys, int32_t num_keys,
                                  const sj_column* probe_payload, int32_t num_probe_payload,
                                  const sj_column* build_payload, int32_t num_build_payload, int32_t* out_probe_rid,
                                  int32_t* out_build_rid, const sj_mut_column* out_probe_payload,
                                  const sj_mut_column* out_build_payload, int64_t capacity,
                                  const sj_join_params* params, const sj_alloc* alloc, sj_stream_t stream,
                                  int64_t* d_count) {
  clear_error();
  sj_table* t = nullptr;
  sj_status st = sj_build(build_keys, num_keys, params, alloc, stream, &t);
  if (st != SJ_OK) return st;
  st = sj_probe_gather(t, probe_keys, num_keys, probe_payload, num_probe_payload, build_payload,
                       num_build_payload, out_probe_rid, out_build_rid, out_probe_payload, out_build_payload,
                       capacity, alloc, stream, d_count);
  const std::string msg = sj_last_error();
  destroy_table(t, reinterpret_cast<cudaStream_t>(stream));
  if (st != SJ_OK) set_error(st, msg);
  return st;
}

SJ_EXPORT const char* sj_status_string(sj_status s) {
  switch (s) {
    case SJ_OK: return "SJ_OK";
    case SJ_ERR_OOM: return "SJ_ERR_OOM";
    case SJ_ERR_TABLE_FULL: return "SJ_ERR_TABLE_FULL";
    case SJ_ERR_INVALID: return "SJ_ERR_INVALID";
    case SJ_ERR_DEVICE: return "SJ_ERR_DEVICE";
    case SJ_ERR_TIMEOUT: return "SJ_ERR_TIMEOUT";
    case SJ_ERR_CAPACITY: return "SJ_ERR_CAPACITY";
    case SJ_ERR_BUSY: return "SJ_ERR_BUSY";
  }
  return "SJ_ERR_UNKNOWN";
}

SJ_EXPORT const char* sj_last_error(void) { return g_last_error.c_str(); }

SJ_EXPORT void sj_timing_enable(int32_t on) {
  // events for the calling thread's timed launches, made here rather than inside a timed region
  if (on)
    while (t_event_pool.size() < 512) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess) break;
      t_event_pool.push_back(e);
    }
  g_timing.store(on != 0);
}

SJ_EXPORT int32_t sj_timing_collect(sj_kernel_time* out, int32_t capacity) {
  const int32_t n = (int32_t)t_records.size();
  for (int32_t i = 0; i < n; ++i) {
    TimingRecord& r = t_records[i];
    float ms = -1.0f;
    if (cudaEventSynchronize(r.b) == cudaSuccess) cudaEventElapsedTime(&ms, r.a, r.b);
    if (out && i < capacity) {
      out[i].name = r.name;
      out[i].ms = ms;
    }
    t_event_pool.push_back(r.a);
    t_event_pool.push_back(r.b);
  }
  t_records.clear();
  return n;
}

SJ_EXPORT int32_t sj_version(void) { return 100; }

}  // extern "C"
