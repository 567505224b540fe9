// The serving loop: device-resident tables and a stream of probe requests.
//
// This generalises the reference's BUILD_PROBE pattern — a table built once per partition slot
// and then probed by many tasks concurrently on their own streams
// (src/op/sirius_physical_hash_join.cpp:1585-1624, :893-1030) — into a request server with
// admission control in the manner of Sirius's exec::admission_control (a fixed budget that
// requests reserve before they run, src/include/exec/admission_control.hpp:39-104):
//   - submit() only queues the request (FIFO) and returns;
//   - a worker thread admits queued requests onto free slots (one CUDA stream each) as long as
//     their device bytes (outputs + probe scratch) fit the remaining budget; a request that does
//     not fit may be passed by later, smaller ones, at most `max_skip` times, after which it blocks
//     the queue until memory frees up (no starvation);
//   - an admitted request runs on its slot's stream (probe + gather into outputs drawn from the
//     server's own stream-ordered memory pool) while others run on theirs, so requests that
//     arrive while earlier ones are on the GPU start as soon as a slot and memory free up and
//     their work overlaps on the device;
//   - small requests (fewer rows than a partitioned probe takes) are batched continuously: while
//     the batch stream is idle, the worker admits every queued small request that fits (up to 256)
//     as ONE launch of the multi-request probe kernel (sj_serve_batch.cu) on its own stream — one
//     descriptor upload, one kernel, one count copy and one host callback for all of them — while
//     large requests keep running on the slot streams; requests that arrive meanwhile form the
//     next batch;
//   - a host callback after the request's last GPU operation stamps its completion time; the
//     worker then returns its scratch charge and hands it to poll(); release() frees its outputs
//     (the caller must have finished reading them, e.g. synchronized its own stream).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sj_internal.h"
#include "sj_partition.cuh"
#include "sj_serve_batch.h"

namespace sj {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SrvTable {
  sj_table* t = nullptr;
  int32_t n_payload = 0;
  int32_t type[8] = {};
};

struct SrvReq;

struct SrvSlot {
  cudaStream_t stream = nullptr;
  SrvReq* req = nullptr;
  int64_t* d_count = nullptr;  // device
  int64_t* h_count = nullptr;  // pinned host
};

struct SrvReq {
  sj_server* server = nullptr;
  uint64_t id = 0;
  int32_t table = 0;
  SrvTable tab;  // copied at submit: the worker never reads the server's table list unlocked
  sj_column key{};
  double t_submit = 0, t_admit = 0;
  std::atomic<double> t_done{0};
  std::atomic<int> done{0};
  int64_t count = 0;
  size_t out_bytes = 0, scratch_bytes = 0;
  int32_t* prid = nullptr;
  int32_t* brid = nullptr;
  void* bpay[8] = {};
  uint32_t* bval[8] = {};
  int slot = -1;   // slot stream, or -1 in the batch
  int skipped = 0;
  bool batchable = false;
  sj_status status = SJ_OK;
};

}  // namespace sj

struct sj_server {
  sj_server_config cfg{};
  int device = 0;
  cudaMemPool_t pool = nullptr;
  cudaStream_t release_stream = nullptr;  // frees of released outputs: never waits on a request
  std::vector<sj::SrvTable> tables;
  std::vector<sj::SrvSlot> slots;
  std::deque<sj::SrvReq*> pending;
  size_t pending_small = 0;  // queued requests that may join a batch
  std::deque<sj::SrvReq*> finished;
  std::unordered_map<uint64_t, sj::SrvReq*> polled;
  size_t in_use = 0;
  // the batch of small requests: its stream, the requests in flight and their device descriptors
  // and counts (pinned host copies)
  cudaStream_t batch_stream = nullptr;
  std::vector<sj::SrvReq*> batch;
  bool batch_busy = false;
  std::atomic<int> batch_done{0};
  sj::ServeReq* h_reqs = nullptr;
  sj::ServeReq* d_reqs = nullptr;
  unsigned long long* d_counts = nullptr;
  int64_t* h_counts = nullptr;
  unsigned* d_item_ctr = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
};

namespace sj {

// sj_alloc over the server's pool (stream-ordered)
static void* pool_alloc(void* ctx, size_t bytes, sj_stream_t s) {
  sj_server* S = static_cast<sj_server*>(ctx);
  void* p = nullptr;
  if (cudaMallocFromPoolAsync(&p, bytes, S->pool, reinterpret_cast<cudaStream_t>(s)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
static void pool_free(void*, void* p, size_t, sj_stream_t s) { cudaFreeAsync(p, reinterpret_cast<cudaStream_t>(s)); }

static size_t a256(size_t b) { return (std::max<size_t>(b, 16) + 255) & ~(size_t)255; }

// Device bytes a request holds: outputs until release, probe scratch until completion.
static void size_request(const sj_server* S, SrvReq* r) {
  const SrvTable& T = r->tab;
  const int64_t n = r->key.num_rows;
  size_t out = 2 * a256((size_t)n * 4);
  for (int c = 0; c < T.n_payload; ++c) {
    out += a256((size_t)n * type_width(T.type[c]));
    if (T.t->apay_valid[c]) out += a256((size_t)(n + 31) / 32 * 4);
  }
  r->out_bytes = out;
  const int kw = T.t->key_type == SJ_INT32 ? 4 : 8;
  // a partitioned probe: partitioned keys + row ids + the partition histogram / offsets
  // a partitioned probe: partitioned keys + row ids + the partition scratch (global offsets, or the
  // run tables of the tile-local partition: 2 x int32 per tile and partition)
  const size_t runs = 2 * a256((size_t)((n + kPartTileRows - 1) / kPartTileRows) * ((size_t)4 << T.t->pbits));
  r->scratch_bytes = 256 + (T.t->pbits > 0 && n >= kMinPartitionedProbe
                               ? a256((size_t)n * kw) + a256((size_t)n * 4) + 256 +
                                     std::max(partition_scratch_bytes(T.t->pbits, S->device), runs)
                               : 0);
}

static void CUDART_CB on_request_done(void* p) {
  SrvReq* r = static_cast<SrvReq*>(p);
  sj_server* S = r->server;
  // under the lock: once the worker sees `done` the server may be destroyed, so this callback
  // touches nothing after unlocking
  std::lock_guard<std::mutex> lk(S->mu);
  r->t_done.store(now_s());
  r->done.store(1);
  S->cv_work.notify_one();
}

// Enqueue one admitted request on its slot's stream (called without the lock held).
static void run_request(sj_server* S, SrvReq* r) {
  SrvSlot& slot = S->slots[r->slot];
  cudaStream_t s = slot.stream;
  const SrvTable& T = r->tab;
  const int64_t n = r->key.num_rows;
  const sj_alloc a{S, pool_alloc, pool_free};
  const Allocator alloc(&a);
  sj_status st = SJ_OK;
  auto take = [&](void** p, size_t bytes) {
    if (st == SJ_OK) st = alloc.allocate(p, a256(bytes), s);
  };
  take((void**)&r->prid, (size_t)n * 4);
  take((void**)&r->brid, (size_t)n * 4);
  sj_mut_column outs[8];
  for (int c = 0; c < T.n_payload; ++c) {
    take(&r->bpay[c], (size_t)n * type_width(T.type[c]));
    outs[c] = sj_mut_column{r->bpay[c], nullptr, T.type[c], 0};
    if (T.t->apay_valid[c]) {
      take((void**)&r->bval[c], (size_t)(n + 31) / 32 * 4);
      outs[c].validity = r->bval[c];
    }
  }
  if (st == SJ_OK) {
    const GatherSpec g{nullptr, 0, nullptr, T.n_payload, r->prid, r->brid, nullptr, outs, n};
    st = probe_gather(T.t, r->key, g, alloc, s, slot.d_count);
  }
  if (st == SJ_OK && cudaMemcpyAsync(slot.h_count, slot.d_count, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    st = SJ_ERR_DEVICE;
  r->status = st;
  if (st != SJ_OK || cudaLaunchHostFunc(s, on_request_done, r) != cudaSuccess) {
    if (r->status == SJ_OK) r->status = SJ_ERR_DEVICE;
    cudaStreamSynchronize(s);
    r->t_done.store(now_s());
    r->done.store(1);
  }
}

static void CUDART_CB on_batch_done(void* p) {
  sj_server* S = static_cast<sj_server*>(p);
  std::lock_guard<std::mutex> lk(S->mu);
  const double t = now_s();
  for (SrvReq* r : S->batch) r->t_done.store(t);
  S->batch_done.store(1);
  S->cv_work.notify_one();
}

// Enqueue the admitted batch of small requests on the batch stream (called without the lock held).
static void run_batch(sj_server* S) {
  cudaStream_t s = S->batch_stream;
  const sj_alloc a{S, pool_alloc, pool_free};
  const Allocator alloc(&a);
  int n = 0;
  for (size_t i = 0; i < S->batch.size(); ++i) {
    SrvReq* r = S->batch[i];
    const SrvTable& T = r->tab;
    const int64_t rows = r->key.num_rows;
    sj_status st = alloc.allocate((void**)&r->prid, a256((size_t)rows * 4), s);
    if (st == SJ_OK) st = alloc.allocate((void**)&r->brid, a256((size_t)rows * 4), s);
    for (int c = 0; c < T.n_payload && st == SJ_OK; ++c) st = alloc.allocate(&r->bpay[c], a256((size_t)rows * 8), s);
    r->status = st;
    if (st != SJ_OK) continue;  // reported by the completion pass; its outputs are freed there
    S->h_reqs[n] = serve_request(T.t, r->key, r->prid, r->brid, r->bpay, S->d_counts + i);
    ++n;
  }
  sj_status st = SJ_OK;
  if (cudaMemsetAsync(S->d_counts, 0, sizeof(unsigned long long) * S->batch.size(), s) != cudaSuccess)
    st = SJ_ERR_DEVICE;
  if (st == SJ_OK && n > 0) st = serve_batch_launch(S->h_reqs, n, S->d_reqs, S->d_item_ctr, S->device, s);
  if (st == SJ_OK && cudaMemcpyAsync(S->h_counts, S->d_counts, 8 * S->batch.size(), cudaMemcpyDeviceToHost, s) !=
                         cudaSuccess)
    st = SJ_ERR_DEVICE;
  if (st != SJ_OK)
    for (SrvReq* r : S->batch)
      if (r->status == SJ_OK) r->status = st;
  if (st != SJ_OK || cudaLaunchHostFunc(s, on_batch_done, S) != cudaSuccess) {
    cudaStreamSynchronize(s);
    std::lock_guard<std::mutex> lk(S->mu);
    const double t = now_s();
    for (SrvReq* r : S->batch) {
      if (r->status == SJ_OK) r->status = SJ_ERR_DEVICE;
      r->t_done.store(t);
    }
    S->batch_done.store(1);
  }
}

static void free_outputs(sj_server* S, SrvReq* r, cudaStream_t s) {
  auto give = [&](void* p) {
    if (p) cudaFreeAsync(p, s);
  };
  give(r->prid);
  give(r->brid);
  const SrvTable& T = r->tab;
  for (int c = 0; c < T.n_payload; ++c) {
    give(r->bpay[c]);
    give(r->bval[c]);
  }
  r->prid = r->brid = nullptr;
  std::fill(std::begin(r->bpay), std::end(r->bpay), nullptr);
  std::fill(std::begin(r->bval), std::end(r->bval), nullptr);
}

static void worker_loop(sj_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    // completions
    bool busy = false;
    for (SrvSlot& sl : S->slots) {
      if (!sl.req) continue;
      if (!sl.req->done.load()) {
        busy = true;
        continue;
      }
      SrvReq* r = sl.req;
      r->count = r->status == SJ_OK ? *sl.h_count : 0;
      S->in_use -= r->scratch_bytes;  // outputs stay charged until release
      if (r->status != SJ_OK) {
        free_outputs(S, r, sl.stream);
        S->in_use -= r->out_bytes;
        r->out_bytes = 0;
      }
      sl.req = nullptr;
      S->finished.push_back(r);
      S->cv_done.notify_all();
    }
    if (S->batch_busy) {
      if (!S->batch_done.load()) {
        busy = true;
      } else {
        for (size_t i = 0; i < S->batch.size(); ++i) {
          SrvReq* r = S->batch[i];
          r->count = r->status == SJ_OK ? S->h_counts[i] : 0;
          S->in_use -= r->scratch_bytes;
          if (r->status != SJ_OK) {
            free_outputs(S, r, S->batch_stream);
            S->in_use -= r->out_bytes;
            r->out_bytes = 0;
          }
          S->finished.push_back(r);
        }
        S->batch.clear();
        S->batch_busy = false;
        S->batch_done.store(0);
        S->cv_done.notify_all();
      }
    }
    // admission: FIFO; smaller requests may pass a head that does not fit, boundedly
    std::vector<SrvReq*> admit, ahead;  // ahead: queued requests passed over in this sweep
    const bool batch_open = S->cfg.batch_small >= 0 && !S->batch_busy;
    bool slots_full = false;  // a queued request found no free slot: later ones may only join the batch
    for (auto it = S->pending.begin(); it != S->pending.end();) {
      SrvReq* r = *it;
      // a small request joins the batch being formed while the batch stream is idle (passing large
      // requests that wait for a slot: its work is a few microseconds); any other request needs a
      // free slot stream, in queue order
      const bool to_batch = batch_open && r->batchable && S->batch.size() < (size_t)kServeMaxBatch;
      int free_slot = -1;
      if (!to_batch) {
        // with every slot busy, only batchable requests can still be admitted in this sweep
        const bool may_batch = batch_open && S->pending_small > 0 && S->batch.size() < (size_t)kServeMaxBatch;
        if (slots_full) {
          if (!may_batch) break;
          ++it;
          continue;
        }
        for (size_t i = 0; i < S->slots.size(); ++i)
          if (!S->slots[i].req) {
            free_slot = (int)i;
            break;
          }
        if (free_slot < 0) {
          slots_full = true;
          if (!may_batch) break;
          ++it;
          continue;
        }
      }
      const size_t need = r->out_bytes + r->scratch_bytes;
      if (S->in_use + need <= (size_t)S->cfg.memory_budget_bytes) {
        S->in_use += need;
        r->t_admit = now_s();
        if (to_batch) {
          r->slot = -1;
          S->batch.push_back(r);
        } else {
          r->slot = free_slot;
          S->slots[free_slot].req = r;
          admit.push_back(r);
        }
        if (r->batchable) --S->pending_small;
        it = S->pending.erase(it);
        busy = true;
        for (SrvReq* q : ahead) ++q->skipped;
      } else {
        if (r->skipped >= S->cfg.max_skip) break;  // passed often enough: nothing may pass it now
        ahead.push_back(r);
        ++it;
      }
    }
    const bool launch_batch = batch_open && !S->batch.empty();
    if (launch_batch) S->batch_busy = true;
    if (!admit.empty() || launch_batch) {
      lk.unlock();
      for (SrvReq* r : admit) run_request(S, r);
      if (launch_batch) run_batch(S);  // S->batch is only changed by this thread
      lk.lock();
      continue;
    }
    if (S->stop && !busy) {
      // Nothing runs and nothing more can be admitted (outputs still held by polled requests):
      // the requests left in the queue are cancelled.
      for (SrvReq* r : S->pending) {
        r->status = SJ_ERR_BUSY;
        S->finished.push_back(r);
      }
      S->pending.clear();
      S->pending_small = 0;
      break;
    }
    S->cv_work.wait_for(lk, std::chrono::microseconds(200));
  }
}

}  // namespace sj

using namespace sj;

extern "C" {

SJ_EXPORT sj_status sj_server_create(const sj_server_config* config, sj_server** out) {
  clear_error();
  if (!out) return set_error(SJ_ERR_INVALID, "out is NULL");
  *out = nullptr;
  sj_server* S = new sj_server();
  S->cfg.slots = 4;
  S->cfg.max_skip = 8;
  S->cfg.memory_budget_bytes = 120ll << 30;
  if (config) {
    if (config->slots > 0) S->cfg.slots = config->slots;
    if (config->max_skip > 0) S->cfg.max_skip = config->max_skip;
    if (config->memory_budget_bytes > 0) S->cfg.memory_budget_bytes = config->memory_budget_bytes;
    if (config->reserve_bytes > 0) S->cfg.reserve_bytes = std::min(config->reserve_bytes, S->cfg.memory_budget_bytes);
    S->cfg.batch_small = config->batch_small;
  }
  if (S->cfg.slots > 64) {
    delete S;
    return set_error(SJ_ERR_INVALID, "at most 64 slots");
  }
  cudaGetDevice(&S->device);
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = S->device;
  if (cudaMemPoolCreate(&S->pool, &props) != cudaSuccess) {
    delete S;
    return set_error(SJ_ERR_DEVICE, "cudaMemPoolCreate failed");
  }
  uint64_t thr = ~0ull;
  cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  // No hidden cross-stream waits: a request's allocation must not reuse a block whose free is
  // still queued behind another slot's request (that would make it wait for that request).
  int no = 0;
  cudaMemPoolSetAttribute(S->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  if (cudaStreamCreateWithFlags(&S->release_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaMemPoolDestroy(S->pool);
    delete S;
    return set_error(SJ_ERR_DEVICE, "creating the server's streams failed");
  }
  if (S->cfg.reserve_bytes > 0) {
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, (size_t)S->cfg.reserve_bytes, S->pool, S->release_stream) != cudaSuccess) {
      cudaGetLastError();
      cudaStreamDestroy(S->release_stream);
      cudaMemPoolDestroy(S->pool);
      delete S;
      return set_error(SJ_ERR_OOM, "cannot reserve the server's memory up front");
    }
    cudaFreeAsync(p, S->release_stream);
    cudaStreamSynchronize(S->release_stream);
  }
  if (cudaStreamCreateWithFlags(&S->batch_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost((void**)&S->h_reqs, sizeof(ServeReq) * kServeMaxBatch) != cudaSuccess ||
      cudaMalloc((void**)&S->d_reqs, sizeof(ServeReq) * kServeMaxBatch) != cudaSuccess ||
      cudaMalloc((void**)&S->d_counts, sizeof(unsigned long long) * kServeMaxBatch) != cudaSuccess ||
      cudaMallocHost((void**)&S->h_counts, sizeof(int64_t) * kServeMaxBatch) != cudaSuccess ||
      cudaMalloc((void**)&S->d_item_ctr, 256) != cudaSuccess) {
    sj_server_destroy(S);
    return set_error(SJ_ERR_DEVICE, "creating the server's batch stream failed");
  }
  S->slots.resize(S->cfg.slots);
  for (SrvSlot& sl : S->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&sl.d_count, 8) != cudaSuccess || cudaMallocHost((void**)&sl.h_count, 8) != cudaSuccess) {
      sj_server_destroy(S);
      return set_error(SJ_ERR_DEVICE, "creating the server's streams failed");
    }
  }
  S->worker = std::thread(worker_loop, S);
  *out = S;
  return SJ_OK;
}

SJ_EXPORT sj_status sj_server_add_table(sj_server* S, const sj_column* key, const sj_column* payload,
                                        int32_t num_payload, const sj_join_params* params, int32_t* table_id) {
  clear_error();
  if (!S || !key || !table_id) return set_error(SJ_ERR_INVALID, "server, key and table_id are required");
  if (num_payload < 0 || num_payload > 8) return set_error(SJ_ERR_INVALID, "at most 8 attached payload columns");
  sj_join_params p;
  sj_default_params(&p);
  if (params) p = *params;
  if (!(p.load_factor > 0.0f && p.load_factor < 1.0f)) p.load_factor = 0.5f;
  if (p.ctas_per_sm <= 0) p.ctas_per_sm = 4;
  p.layout = SJ_LAYOUT_DISTINCT;
  p.null_equality = SJ_NULLS_UNEQUAL;
  sj_table* t = nullptr;
  cudaStream_t s = nullptr;
  SJ_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const sj_status st = build_table(*key, payload, num_payload, p, Allocator(nullptr), s, &t);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (st != SJ_OK) return st;
  SrvTable T;
  T.t = t;
  T.n_payload = num_payload;
  for (int c = 0; c < num_payload; ++c) T.type[c] = payload[c].type;
  std::lock_guard<std::mutex> lk(S->mu);
  S->tables.push_back(T);
  *table_id = (int32_t)S->tables.size() - 1;
  return SJ_OK;
}

SJ_EXPORT sj_status sj_server_submit(sj_server* S, int32_t table_id, const sj_column* probe_key, uint64_t id) {
  clear_error();
  if (!S || !probe_key) return set_error(SJ_ERR_INVALID, "server and probe_key are required");
  SrvReq* r = new SrvReq();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (table_id < 0 || table_id >= (int32_t)S->tables.size()) {
      delete r;
      return set_error(SJ_ERR_INVALID, "unknown table id");
    }
    if (probe_key->type != S->tables[table_id].t->key_type || probe_key->num_rows < 0 ||
        probe_key->num_rows > INT32_MAX) {
      delete r;
      return set_error(SJ_ERR_INVALID, "probe key type differs from the table's, or bad row count");
    }
    r->server = S;
    r->id = id;
    r->table = table_id;
    r->tab = S->tables[table_id];
    r->key = *probe_key;
    r->batchable = serve_batchable(r->tab.t, probe_key->num_rows);
    size_request(S, r);
    if (r->out_bytes + r->scratch_bytes > (size_t)S->cfg.memory_budget_bytes) {
      delete r;
      return set_error(SJ_ERR_BUSY, "request needs more device memory than the whole budget");
    }
    r->t_submit = now_s();
    S->pending.push_back(r);
    if (r->batchable) ++S->pending_small;
  }
  S->cv_work.notify_one();
  return SJ_OK;
}

SJ_EXPORT int32_t sj_server_poll(sj_server* S, sj_request_result* out, int32_t capacity, int32_t wait_ms) {
  clear_error();
  if (!S || (capacity > 0 && !out)) return -(int32_t)set_error(SJ_ERR_INVALID, "server and out are required");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->finished.empty() && wait_ms > 0)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->finished.empty(); });
  int32_t n = 0;
  while (n < capacity && !S->finished.empty()) {
    SrvReq* r = S->finished.front();
    S->finished.pop_front();
    sj_request_result& o = out[n++];
    std::memset(&o, 0, sizeof(o));
    o.request_id = r->id;
    o.status = r->status;
    o.table_id = r->table;
    o.count = r->count;
    o.probe_rows = r->key.num_rows;
    o.probe_rid = r->prid;
    o.build_rid = r->brid;
    for (int c = 0; c < 8; ++c) {
      o.build_payload[c] = r->bpay[c];
      o.build_validity[c] = r->bval[c];
    }
    o.t_submit = r->t_submit;
    o.t_admit = r->t_admit;
    o.t_done = r->t_done.load();
    S->polled[r->id] = r;
  }
  return n;
}

SJ_EXPORT sj_status sj_server_release(sj_server* S, uint64_t id) {
  clear_error();
  if (!S) return set_error(SJ_ERR_INVALID, "server is NULL");
  SrvReq* r = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->polled.find(id);
    if (it == S->polled.end()) return set_error(SJ_ERR_INVALID, "unknown or unpolled request id");
    r = it->second;
    S->polled.erase(it);
    free_outputs(S, r, S->release_stream);
    S->in_use -= r->out_bytes;
  }
  delete r;
  S->cv_work.notify_one();
  return SJ_OK;
}

SJ_EXPORT sj_status sj_server_destroy(sj_server* S) {
  if (!S) return SJ_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->device);
  cudaStream_t s0 = S->release_stream;
  for (auto& kv : S->polled) {
    free_outputs(S, kv.second, s0);
    delete kv.second;
  }
  for (SrvReq* r : S->finished) {
    free_outputs(S, r, s0);
    delete r;
  }
  for (SrvSlot& sl : S->slots)
    if (sl.stream) cudaStreamSynchronize(sl.stream);
  if (S->batch_stream) {
    cudaStreamSynchronize(S->batch_stream);
    cudaStreamDestroy(S->batch_stream);
  }
  if (S->h_reqs) cudaFreeHost(S->h_reqs);
  if (S->d_reqs) cudaFree(S->d_reqs);
  if (S->d_counts) cudaFree(S->d_counts);
  if (S->h_counts) cudaFreeHost(S->h_counts);
  if (S->d_item_ctr) cudaFree(S->d_item_ctr);
  for (SrvSlot& sl : S->slots) {
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.d_count) cudaFree(sl.d_count);
    if (sl.h_count) cudaFreeHost(sl.h_count);
  }
  for (SrvTable& T : S->tables) destroy_table(T.t, nullptr);
  cudaDeviceSynchronize();
  if (S->release_stream) cudaStreamDestroy(S->release_stream);
  if (S->pool) cudaMemPoolDestroy(S->pool);
  delete S;
  return SJ_OK;
}

}  // extern "C"
