// One-shot INNER join from HOST buffers (sj_inner_join_host): the operator's whole join when its
// batches live in host memory (the reference moves batches between host and device memory spaces
// before a GPU operator runs, and reads results back after it; src/op/sirius_physical_hash_join.cpp
// :1527-1955 runs on device-resident batches in between).
//
// The build side is copied in and built (sj_build_ex, the build payloads attached to the table).
// The probe side then streams through in chunks of `chunk_rows` rows over two copy streams, with
// two device slots per direction:
//   h2d stream:  chunk i+2's keys, validity words and payloads into input slot i % 2
//   `stream`:    sj_probe_gather of chunk i into output slot i % 2, probe row ids rebased
//   d2h stream:  chunk i's `count` output rows to the host outputs at the running offset
// PCIe is full duplex, so the uploads, the probes and the downloads overlap; a step costs about
// max(upload, download) instead of their sum. The host reads each chunk's count (one event wait
// per chunk) to place the next chunk's rows. Outputs follow sj_probe_gather: rows past `capacity`
// are not written, and *out_count is the full match count.
#include <algorithm>
#include <string>

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

// Adds `base` to the first min(*d_n, cap) entries (probe row ids of a chunk -> of the whole probe).
__global__ void __launch_bounds__(256) rebase_rows_kernel(int32_t* p, const int64_t* d_n, int64_t cap, int32_t base) {
  const int64_t n = *d_n < cap ? *d_n : cap;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] += base;
}

namespace {

constexpr int64_t kDefaultChunkRows = 1ll << 23;

struct HostJoin {
  Allocator alloc;
  cudaStream_t s = nullptr, h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_build_in = nullptr, in_ready[2] = {}, in_free[2] = {}, done[2] = {}, out_free[2] = {};
  int64_t* h_cnt = nullptr;  // pinned, 2 words
  sj_table* table = nullptr;
  struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
  };
  Buf bufs[64];
  int n_bufs = 0;

  explicit HostJoin(const sj_alloc* a) : alloc(a) {}
  sj_status get(void** p, size_t bytes) {
    if (n_bufs == 64) return set_error(SJ_ERR_INVALID, "host join: too many device buffers");
    bytes = (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
    SJ_TRY(alloc.allocate(p, bytes, s));
    bufs[n_bufs++] = Buf{*p, bytes};
    return SJ_OK;
  }
  void put(void* p) {  // stream-ordered release on `s` of a buffer taken with get()
    for (int i = 0; i < n_bufs; ++i)
      if (bufs[i].p == p) {
        alloc.release(p, bufs[i].bytes, s);
        bufs[i] = bufs[--n_bufs];
        return;
      }
  }
  sj_status init(cudaStream_t user) {
    s = user;
    if (cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_build_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost((void**)&h_cnt, 2 * sizeof(int64_t)) != cudaSuccess)
      return set_error(SJ_ERR_DEVICE, "host join: creating streams, events or pinned counts failed");
    for (int k = 0; k < 2; ++k)
      if (cudaEventCreateWithFlags(&in_ready[k], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&in_free[k], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&out_free[k], cudaEventDisableTiming) != cudaSuccess)
        return set_error(SJ_ERR_DEVICE, "host join: creating events failed");
    return SJ_OK;
  }
  ~HostJoin() {
    // every stream drained before a buffer goes back to the allocator
    if (h2d) cudaStreamSynchronize(h2d);
    if (d2h) cudaStreamSynchronize(d2h);
    cudaStreamSynchronize(s);
    if (table) destroy_table(table, s);
    while (n_bufs > 0) put(bufs[n_bufs - 1].p);
    cudaStreamSynchronize(s);
    if (h_cnt) cudaFreeHost(h_cnt);
    for (cudaEvent_t e : {ev_build_in, in_ready[0], in_ready[1], in_free[0], in_free[1], done[0], done[1],
                          out_free[0], out_free[1]})
      if (e) cudaEventDestroy(e);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }
};

sj_status check_host_col(const sj_column& c, const char* what, bool key) {
  if (c.type != SJ_INT32 && c.type != SJ_INT64 && (key || type_width(c.type) == 0))
    return set_error(SJ_ERR_INVALID, std::string(what) + ": unsupported type");
  if (c.num_rows < 0 || c.num_rows > INT32_MAX) return set_error(SJ_ERR_INVALID, std::string(what) + ": bad row count");
  if (c.num_rows > 0 && !c.data) return set_error(SJ_ERR_INVALID, std::string(what) + ": data is NULL");
  if (c.validity_offset < 0) return set_error(SJ_ERR_INVALID, std::string(what) + ": negative validity offset");
  if (!key && c.validity)
    return set_error(SJ_ERR_INVALID, std::string(what) + ": payload columns with NULLs are not supported from host memory");
  return SJ_OK;
}

// Validity words of rows [r0, r0 + m) of a host column: the words to copy and the bit offset of
// row r0 in the first of them.
struct WordRange {
  const uint32_t* src;
  int64_t words;
  int64_t bit_off;
};
WordRange word_range(const sj_column& c, int64_t r0, int64_t m) {
  const int64_t first = c.validity_offset + r0;
  return WordRange{c.validity + first / 32, (first % 32 + m + 31) / 32, first % 32};
}

}  // namespace
}  // namespace sj

using namespace sj;

extern "C" {

SJ_EXPORT sj_status sj_inner_join_host(const sj_column* build_keys, const sj_column* probe_keys, int32_t num_keys,
                                       const sj_column* probe_payload, int32_t num_probe_payload,
                                       const sj_column* build_payload, int32_t num_build_payload,
                                       int32_t* out_probe_rid, int32_t* out_build_rid,
                                       const sj_mut_column* out_probe_payload, const sj_mut_column* out_build_payload,
                                       int64_t capacity, int64_t chunk_rows, const sj_join_params* params,
                                       const sj_alloc* alloc, sj_stream_t stream, int64_t* out_count) {
  clear_error();
  if (!build_keys || !probe_keys || !out_count) return set_error(SJ_ERR_INVALID, "keys and out_count are required");
  if (num_keys < 1 || num_keys > kMaxKeyColumns) return set_error(SJ_ERR_INVALID, "1 to 4 key columns");
  if (num_probe_payload < 0 || num_probe_payload > kMaxPayload || num_build_payload < 0 ||
      num_build_payload > kMaxPayload)
    return set_error(SJ_ERR_INVALID, "at most 8 payload columns per side");
  if ((num_probe_payload > 0 && !probe_payload) || (num_build_payload > 0 && !build_payload))
    return set_error(SJ_ERR_INVALID, "payload column list is NULL");
  if (capacity < 0 || chunk_rows < 0) return set_error(SJ_ERR_INVALID, "negative capacity or chunk_rows");
  *out_count = 0;
  const int64_t nb = build_keys[0].num_rows, np = probe_keys[0].num_rows;
  for (int c = 0; c < num_keys; ++c) {
    SJ_TRY(check_host_col(build_keys[c], "build key", true));
    SJ_TRY(check_host_col(probe_keys[c], "probe key", true));
    if (build_keys[c].num_rows != nb || probe_keys[c].num_rows != np)
      return set_error(SJ_ERR_INVALID, "key columns differ in row count");
    if (probe_keys[c].type != build_keys[c].type) return set_error(SJ_ERR_INVALID, "probe and build key types differ");
  }
  for (int c = 0; c < num_probe_payload; ++c) {
    SJ_TRY(check_host_col(probe_payload[c], "probe payload", false));
    if (probe_payload[c].num_rows != np) return set_error(SJ_ERR_INVALID, "probe payload row count differs");
    if (capacity > 0 && (!out_probe_payload || !out_probe_payload[c].data ||
                         out_probe_payload[c].type != probe_payload[c].type))
      return set_error(SJ_ERR_INVALID, "probe payload output missing or of another type");
  }
  for (int c = 0; c < num_build_payload; ++c) {
    SJ_TRY(check_host_col(build_payload[c], "build payload", false));
    if (build_payload[c].num_rows != nb) return set_error(SJ_ERR_INVALID, "build payload row count differs");
    if (capacity > 0 && (!out_build_payload || !out_build_payload[c].data ||
                         out_build_payload[c].type != build_payload[c].type))
      return set_error(SJ_ERR_INVALID, "build payload output missing or of another type");
  }
  const cudaStream_t us = reinterpret_cast<cudaStream_t>(stream);
  int device = 0;
  cudaGetDevice(&device);
  HostJoin J(alloc);
  SJ_TRY(J.init(us));

  // ---- build side: copy in, build with the payloads attached ----
  sj_column dbk[kMaxKeyColumns], dbp[kMaxPayload];
  for (int c = 0; c < num_keys; ++c) {
    const sj_column& h = build_keys[c];
    const size_t w = type_width(h.type);
    dbk[c] = sj_column{nullptr, nullptr, 0, nb, h.type, 0};
    void* d;
    SJ_TRY(J.get(&d, (size_t)nb * w));
    dbk[c].data = d;
    if (nb > 0) SJ_CUDA_TRY(cudaMemcpyAsync(d, h.data, (size_t)nb * w, cudaMemcpyHostToDevice, us));
    if (h.validity) {
      const WordRange wr = word_range(h, 0, nb);
      void* v;
      SJ_TRY(J.get(&v, (size_t)wr.words * 4));
      if (wr.words > 0) SJ_CUDA_TRY(cudaMemcpyAsync(v, wr.src, (size_t)wr.words * 4, cudaMemcpyHostToDevice, us));
      dbk[c].validity = static_cast<const uint32_t*>(v);
      dbk[c].validity_offset = wr.bit_off;
    }
  }
  for (int c = 0; c < num_build_payload; ++c) {
    const sj_column& h = build_payload[c];
    const size_t w = type_width(h.type);
    void* d;
    SJ_TRY(J.get(&d, (size_t)nb * w));
    if (nb > 0) SJ_CUDA_TRY(cudaMemcpyAsync(d, h.data, (size_t)nb * w, cudaMemcpyHostToDevice, us));
    dbp[c] = sj_column{d, nullptr, 0, nb, h.type, 0};
  }

  // ---- probe-side slots ----
  int64_t chunk = chunk_rows > 0 ? chunk_rows : kDefaultChunkRows;
  chunk = std::min<int64_t>(chunk, std::max<int64_t>(np, 1));
  chunk = (chunk + 31) / 32 * 32;  // chunk starts stay at one bit offset within the validity words
  const int64_t n_chunks = (np + chunk - 1) / chunk;
  void* in_key[2][kMaxKeyColumns] = {};
  uint32_t* in_val[2][kMaxKeyColumns] = {};
  void* in_pay[2][kMaxPayload] = {};
  for (int k = 0; k < 2 && k < n_chunks; ++k) {
    for (int c = 0; c < num_keys; ++c) {
      SJ_TRY(J.get(&in_key[k][c], (size_t)chunk * type_width(probe_keys[c].type)));
      if (probe_keys[c].validity) SJ_TRY(J.get((void**)&in_val[k][c], (size_t)(chunk / 32 + 2) * 4));
    }
    for (int c = 0; c < num_probe_payload; ++c)
      SJ_TRY(J.get(&in_pay[k][c], (size_t)chunk * type_width(probe_payload[c].type)));
  }
  SJ_CUDA_TRY(cudaEventRecord(J.ev_build_in, us));  // build copies queued, slots allocated
  SJ_CUDA_TRY(cudaStreamWaitEvent(J.h2d, J.ev_build_in, 0));

  auto upload = [&](int64_t i) -> sj_status {  // chunk i into input slot i % 2, on h2d
    const int k = (int)(i & 1);
    const int64_t r0 = i * chunk, m = std::min(chunk, np - r0);
    if (i >= 2) SJ_CUDA_TRY(cudaStreamWaitEvent(J.h2d, J.in_free[k], 0));
    for (int c = 0; c < num_keys; ++c) {
      const sj_column& h = probe_keys[c];
      const size_t w = type_width(h.type);
      SJ_CUDA_TRY(cudaMemcpyAsync(in_key[k][c], static_cast<const char*>(h.data) + (size_t)r0 * w, (size_t)m * w,
                                  cudaMemcpyHostToDevice, J.h2d));
      if (h.validity) {
        const WordRange wr = word_range(h, r0, m);
        SJ_CUDA_TRY(cudaMemcpyAsync(in_val[k][c], wr.src, (size_t)wr.words * 4, cudaMemcpyHostToDevice, J.h2d));
      }
    }
    for (int c = 0; c < num_probe_payload; ++c) {
      const size_t w = type_width(probe_payload[c].type);
      SJ_CUDA_TRY(cudaMemcpyAsync(in_pay[k][c], static_cast<const char*>(probe_payload[c].data) + (size_t)r0 * w,
                                  (size_t)m * w, cudaMemcpyHostToDevice, J.h2d));
    }
    SJ_CUDA_TRY(cudaEventRecord(J.in_ready[k], J.h2d));
    return SJ_OK;
  };
  for (int64_t i = 0; i < std::min<int64_t>(n_chunks, 2); ++i) SJ_TRY(upload(i));

  SJ_TRY(sj_build_ex(dbk, num_keys, num_build_payload ? dbp : nullptr, num_build_payload, params, alloc, stream,
                     &J.table));
  for (int c = 0; c < num_keys; ++c) {  // the table holds what the probes need
    J.put(const_cast<void*>(dbk[c].data));
    if (dbk[c].validity) J.put(const_cast<uint32_t*>(dbk[c].validity));
  }
  for (int c = 0; c < num_build_payload; ++c) J.put(const_cast<void*>(dbp[c].data));
  sj_table_info info{};
  SJ_TRY(sj_table_get_info(J.table, &info));
  const bool distinct = info.layout == SJ_LAYOUT_DISTINCT;

  // ---- output slots: a DISTINCT table gives at most one match per probe row ----
  const bool want_prid = out_probe_rid != nullptr, want_brid = out_build_rid != nullptr;
  int64_t out_cap[2] = {0, 0};
  int32_t* o_prid[2] = {};
  int32_t* o_brid[2] = {};
  void* o_ppay[2][kMaxPayload] = {};
  void* o_bpay[2][kMaxPayload] = {};
  int64_t* d_cnt = nullptr;
  SJ_TRY(J.get((void**)&d_cnt, 2 * sizeof(int64_t)));
  auto size_slot = [&](int k, int64_t rows) -> sj_status {  // (re)allocate output slot k for `rows`
    if (rows <= out_cap[k]) return SJ_OK;
    rows = std::max<int64_t>(rows, out_cap[k] + out_cap[k] / 2);
    if (o_prid[k]) J.put(o_prid[k]);
    if (o_brid[k]) J.put(o_brid[k]);
    for (int c = 0; c < num_probe_payload; ++c)
      if (o_ppay[k][c]) J.put(o_ppay[k][c]);
    for (int c = 0; c < num_build_payload; ++c)
      if (o_bpay[k][c]) J.put(o_bpay[k][c]);
    if (want_prid) SJ_TRY(J.get((void**)&o_prid[k], (size_t)rows * 4));
    if (want_brid) SJ_TRY(J.get((void**)&o_brid[k], (size_t)rows * 4));
    for (int c = 0; c < num_probe_payload; ++c)
      SJ_TRY(J.get(&o_ppay[k][c], (size_t)rows * type_width(probe_payload[c].type)));
    for (int c = 0; c < num_build_payload; ++c)
      SJ_TRY(J.get(&o_bpay[k][c], (size_t)rows * type_width(build_payload[c].type)));
    out_cap[k] = rows;
    return SJ_OK;
  };
  if (distinct)
    for (int k = 0; k < 2 && k < n_chunks; ++k) SJ_TRY(size_slot(k, chunk));

  // ---- the probe stream ----
  int64_t total = 0;
  for (int64_t i = 0; i < n_chunks; ++i) {
    const int k = (int)(i & 1);
    const int64_t r0 = i * chunk, m = std::min(chunk, np - r0);
    sj_column pk[kMaxKeyColumns], pp[kMaxPayload];
    for (int c = 0; c < num_keys; ++c) {
      pk[c] = sj_column{in_key[k][c], nullptr, 0, m, probe_keys[c].type, 0};
      if (probe_keys[c].validity) {
        pk[c].validity = in_val[k][c];
        pk[c].validity_offset = word_range(probe_keys[c], r0, m).bit_off;
      }
    }
    for (int c = 0; c < num_probe_payload; ++c) pp[c] = sj_column{in_pay[k][c], nullptr, 0, m, probe_payload[c].type, 0};
    SJ_CUDA_TRY(cudaStreamWaitEvent(us, J.in_ready[k], 0));
    if (i >= 2) SJ_CUDA_TRY(cudaStreamWaitEvent(us, J.out_free[k], 0));  // slot k's rows downloaded
    int64_t slot_cap = chunk;
    if (!distinct) {  // a GROUPED table: size the slot from the exact count
      SJ_TRY(sj_probe_count(J.table, pk, num_keys, alloc, stream, d_cnt + k));
      SJ_CUDA_TRY(cudaMemcpyAsync(J.h_cnt + k, d_cnt + k, 8, cudaMemcpyDeviceToHost, us));
      SJ_CUDA_TRY(cudaStreamSynchronize(us));
      SJ_TRY(size_slot(k, std::max<int64_t>(J.h_cnt[k], 1)));
      slot_cap = J.h_cnt[k];
    }
    sj_mut_column op[kMaxPayload], ob[kMaxPayload];
    for (int c = 0; c < num_probe_payload; ++c) op[c] = sj_mut_column{o_ppay[k][c], nullptr, probe_payload[c].type, 0};
    for (int c = 0; c < num_build_payload; ++c) ob[c] = sj_mut_column{o_bpay[k][c], nullptr, build_payload[c].type, 0};
    SJ_TRY(sj_probe_gather(J.table, pk, num_keys, num_probe_payload ? pp : nullptr, num_probe_payload, nullptr,
                           num_build_payload, o_prid[k], o_brid[k], num_probe_payload ? op : nullptr,
                           num_build_payload ? ob : nullptr, slot_cap, alloc, stream, d_cnt + k));
    if (want_prid && r0 > 0 && slot_cap > 0)
      rebase_rows_kernel<<<(int)std::min<int64_t>((slot_cap + 255) / 256, (int64_t)sm_count(device) * 8), 256, 0, us>>>(
          o_prid[k], d_cnt + k, slot_cap, (int32_t)r0);
    SJ_CUDA_TRY(cudaGetLastError());
    SJ_CUDA_TRY(cudaEventRecord(J.in_free[k], us));
    SJ_CUDA_TRY(cudaMemcpyAsync(J.h_cnt + k, d_cnt + k, 8, cudaMemcpyDeviceToHost, us));
    SJ_CUDA_TRY(cudaEventRecord(J.done[k], us));
    if (i + 2 < n_chunks) SJ_TRY(upload(i + 2));
    // this chunk's rows go to the host once its count is known
    SJ_CUDA_TRY(cudaEventSynchronize(J.done[k]));
    const int64_t cnt = J.h_cnt[k];
    if (cnt < 0) return set_error(SJ_ERR_TIMEOUT, "host join: a bounded device wait ran out");
    if (cnt > slot_cap) return set_error(SJ_ERR_DEVICE, "host join: chunk output exceeds its slot");
    const int64_t put = total < capacity ? std::min(cnt, capacity - total) : 0;
    SJ_CUDA_TRY(cudaStreamWaitEvent(J.d2h, J.done[k], 0));
    auto down = [&](void* host, const void* dev, size_t w) -> sj_status {
      if (put > 0 && host)
        SJ_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(host) + (size_t)total * w, dev, (size_t)put * w,
                                    cudaMemcpyDeviceToHost, J.d2h));
      return SJ_OK;
    };
    SJ_TRY(down(out_probe_rid, o_prid[k], 4));
    SJ_TRY(down(out_build_rid, o_brid[k], 4));
    for (int c = 0; c < num_probe_payload; ++c)
      SJ_TRY(down(out_probe_payload[c].data, o_ppay[k][c], type_width(probe_payload[c].type)));
    for (int c = 0; c < num_build_payload; ++c)
      SJ_TRY(down(out_build_payload[c].data, o_bpay[k][c], type_width(build_payload[c].type)));
    SJ_CUDA_TRY(cudaEventRecord(J.out_free[k], J.d2h));
    total += cnt;
  }
  SJ_CUDA_TRY(cudaStreamSynchronize(J.d2h));
  SJ_CUDA_TRY(cudaStreamSynchronize(us));
  *out_count = total;
  return SJ_OK;
}

}  // extern "C"
