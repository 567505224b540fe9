// sj_inner_join_noalloc: the one-shot INNER join for callers that cannot allocate device memory.
//
// Who needs it: code that runs under a device-memory budget it must not exceed or grow (for
// example a task whose reservation from Sirius's memory manager is already fully committed, where
// any allocation attempt would be refused and turned into an out-of-memory reschedule), code on a
// latency-critical host thread that must not wait in the driver's allocator (cudaMalloc can
// synchronize the whole device), and hosts whose device allocator belongs to another component
// and may not be called from this library. For them this entry point takes every byte of scratch
// (the hash table, its build statistics, the grouped-probe match list) from one statically
// allocated device array instead of cudaMalloc / cudaMallocAsync / an allocator callback.
//
// Limits and rules:
//   - The arena is kNoAllocArenaBytes = 64 MiB per GPU, declared below as a file-scope
//     `static __device__` array. The driver commits it when it loads this file's device code: at
//     the first call on a device under lazy module loading (CUDA_MODULE_LOADING=LAZY, the default
//     since CUDA 12.2), or when the library's device code is loaded under EAGER. A caller whose
//     device memory is fully committed later should make one warm-up call while the 64 MiB is still
//     free. From then on every GPU that ran the entry point holds the arena until the process exits.
//   - A call whose worst-case need exceeds the arena is rejected with SJ_ERR_INVALID before any
//     GPU work (the exact need is in the message). At load factor 0.5: 2^19 build rows with up to
//     1.9M probe rows, or 2^20 build rows with up to 600K probe rows.
//   - Radix partitioning and attached payloads are not used (the table is built unpartitioned).
//   - All calls share the arena and leave their data in it; each call re-initialises everything it
//     reads (slots, counters, offsets) before use, so stale contents never leak into a result.
//     Calls that overlap on the GPU race on the arena: issue them on one stream, or synchronise.
//   - The arena's device address is looked up with cudaGetSymbolAddress the first time the entry
//     point runs on a device (with that device current); make that first call before any stream
//     capture begins on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sj_internal.h"

namespace sj {

constexpr size_t kNoAllocArenaBytes = 64ull << 20;

// The arena. In host code `g_noalloc_arena` only names the symbol; its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_arena[kNoAllocArenaBytes];

static std::mutex g_noalloc_mu;
static std::vector<void*> g_noalloc_base;  // per device: the arena's device address

static sj_status noalloc_arena(void** out) {
  int dev = 0;
  SJ_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if ((int)g_noalloc_base.size() <= dev) g_noalloc_base.resize(dev + 1, nullptr);
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_arena);
    if (e != cudaSuccess || p == nullptr)
      return set_error(SJ_ERR_DEVICE, std::string("cudaGetSymbolAddress of the static arena failed: ") +
                                          cudaGetErrorString(e));
    g_noalloc_base[dev] = p;
  }
  *out = g_noalloc_base[dev];
  return SJ_OK;
}

// Bump allocator over the arena for one call: frees are no-ops, the next call starts over.
struct Bump {
  char* base;
  size_t cap;
  size_t used;
};

static void* bump_alloc(void* ctx, size_t bytes, sj_stream_t) {
  Bump* b = static_cast<Bump*>(ctx);
  const size_t off = (b->used + 255) & ~(size_t)255;
  if (off > b->cap || bytes > b->cap - off) return nullptr;
  b->used = off + bytes;
  return b->base + off;
}

static void bump_free(void*, void*, size_t, sj_stream_t) {}

static size_t a256(size_t b) { return (std::max<size_t>(b, 16) + 255) & ~(size_t)255; }

// Buckets of a table of `keys` keys with `spb` slots per bucket at load factor lf: the same
// power-of-two geometry build_table chooses.
static size_t buckets_for(int64_t keys, double lf, int spb) {
  const double slots = std::max(1.0, (double)std::max<int64_t>(keys, 1) / lf);
  const size_t want = (size_t)std::ceil(slots / spb);
  size_t b = 1;
  while (b < want) b <<= 1;
  return b;
}

// Worst case over slot encodings and layouts of what build + probe take from the allocator. The
// bump allocator never reuses memory within a call, so every request counts, temporaries included.
static size_t noalloc_need(int64_t n_build, int64_t n_probe, double lf) {
  const size_t nb = (size_t)std::max<int64_t>(n_build, 1), np = (size_t)std::max<int64_t>(n_probe, 1);
  // Both slot encodings have the same slot count (wide: 2 per bucket; packed: 4 per bucket in half
  // as many buckets); wide slots take the most bytes.
  const size_t wide_buckets = buckets_for((int64_t)nb, lf, 2);
  const size_t slot_bytes = wide_buckets * 32;
  const size_t nslots = wide_buckets * 2;
  size_t need = a256(sizeof(long long) * 6) + a256(slot_bytes);  // build statistics, slots
  // grouped layout: counts + offsets over every slot, or a shrink to at most a quarter of the
  // buckets (the copy, then counts + offsets over its slots), whichever is larger
  const size_t groups_full = a256((nslots + 1) * 4) + a256((nslots + 2) * 4);
  const size_t groups_shrunk = a256(slot_bytes / 4) + a256((nslots / 4 + 1) * 4) + a256((nslots / 4 + 2) * 4);
  need += std::max(groups_full, groups_shrunk) + a256(1024 * 8);  // + the scan's block sums
  // group members and NULL-key row ids (together at most one per build row), the NULL-row counter
  need += a256(nb * 4) + 256 + a256(8);
  // probe: the grouped match list in one request (a DISTINCT probe takes a 256-byte tile counter)
  need += a256(3 * a256(np * 4) + a256((np + 1) * 8) + 1024 * 8 + 256);
  return need;
}

}  // namespace sj

using namespace sj;

extern "C" SJ_EXPORT sj_status sj_inner_join_noalloc(
    const sj_column* build_keys, const sj_column* probe_keys, int32_t num_keys, const sj_column* probe_payload,
    int32_t num_probe_payload, const sj_column* build_payload, int32_t num_build_payload, int32_t* out_probe_rid,
    int32_t* out_build_rid, const sj_mut_column* out_probe_payload, const sj_mut_column* out_build_payload,
    int64_t capacity, const sj_join_params* params, sj_stream_t stream, int64_t* d_count) {
  clear_error();
  if (num_keys != 1) return set_error(SJ_ERR_INVALID, "exactly one key column is supported");
  if (!build_keys || !probe_keys || !d_count)
    return set_error(SJ_ERR_INVALID, "build_keys, probe_keys and d_count are required");
  sj_join_params p;
  sj_default_params(&p);
  // every field is honoured except partition_bits (always -1 here), probe_partition_mb, which only
  // applies to partitioned tables, and bloom_bits_per_key (the table is discarded at the end of the
  // call); zero fields take their defaults, as in sj_build
  if (params) {
    const sj_join_params defaults = p;
    p = *params;
    if (!(p.load_factor > 0.0f)) p.load_factor = defaults.load_factor;
    if (p.block_size <= 0) p.block_size = defaults.block_size;
    if (p.group_width <= 0) p.group_width = defaults.group_width;
    if (p.ctas_per_sm <= 0) p.ctas_per_sm = defaults.ctas_per_sm;
  }
  p.partition_bits = -1;  // unpartitioned: no row store, no partition buffers
  p.probe_partition_mb = 0;
  p.bloom_bits_per_key = 0;  // no dynamic filter: it would outlive the call
  if (!(p.load_factor > 0.0f && p.load_factor < 1.0f)) return set_error(SJ_ERR_INVALID, "load_factor must be in (0, 1)");
  const size_t need = noalloc_need(build_keys->num_rows, probe_keys->num_rows, p.load_factor);
  if (need > kNoAllocArenaBytes)
    return set_error(SJ_ERR_INVALID, "sj_inner_join_noalloc: " + std::to_string(build_keys->num_rows) +
                                         " build rows and " + std::to_string(probe_keys->num_rows) +
                                         " probe rows need up to " + std::to_string(need) +
                                         " bytes of scratch; the static arena holds " +
                                         std::to_string(kNoAllocArenaBytes) + " bytes");
  void* base = nullptr;
  SJ_TRY(noalloc_arena(&base));
  Bump bump{static_cast<char*>(base), kNoAllocArenaBytes, 0};
  const sj_alloc a{&bump, bump_alloc, bump_free};
  const Allocator alloc(&a);
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  sj_table* t = nullptr;
  try {
    SJ_TRY(build_table(build_keys[0], nullptr, 0, p, alloc, s, &t));
    const GatherSpec g{probe_payload, num_probe_payload, build_payload, num_build_payload, out_probe_rid,
                       out_build_rid, out_probe_payload, out_build_payload, capacity};
    const sj_status st = probe_gather(t, probe_keys[0], g, alloc, s, d_count);
    const std::string msg = sj_last_error();
    destroy_table(t, s);
    if (st != SJ_OK) return set_error(st, msg);
    return SJ_OK;
  } catch (const std::exception& e) {
    if (t) destroy_table(t, s);
    return set_error(SJ_ERR_DEVICE, e.what());
  }
}
