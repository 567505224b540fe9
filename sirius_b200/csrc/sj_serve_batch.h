// Continuous batching of small served requests (sj_serve_batch.cu): one kernel launch probes many
// requests, each against its own resident table, into its own outputs.
#pragma once

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

constexpr int kServeMaxBatch = 256;  // requests per batch launch
constexpr int kServeMaxFields = 3;   // attached 8-byte build fields a batched request gathers

// One request of a batch (copied to the device as is).
struct ServeReq {
  TableDev t;
  const void* keys;
  const uint32_t* kvalid;
  int64_t kvoff;
  int64_t n;
  const char* rec;     // row store (build row id at byte 0, field c at 8 + 8c), or the position ->
  int32_t rec_stride;  //   row id map; NULL: positions are the build row ids
  int32_t n_fields;
  int32_t key64;
  int32_t wide;
  int32_t* out_prid;
  int32_t* out_brid;
  void* out_field[kServeMaxFields];
  unsigned long long* count;  // zeroed before the launch
  int64_t capacity;
  uint32_t first_item;        // set by serve_batch_launch
  uint32_t pad;
};

// True when a probe of `probe_rows` rows into DISTINCT table `t` can join a batch: fewer rows than
// a partitioned probe takes, and attached payloads that are 8-byte fields without NULLs (at most 3).
bool serve_batchable(const sj_table* t, int64_t probe_rows);

// The descriptor of one request (outputs: probe row ids, build row ids, the attached fields).
ServeReq serve_request(const sj_table* t, const sj_column& key, int32_t* prid, int32_t* brid, void* const* fields,
                       unsigned long long* count);

// Numbers the work items, copies h_reqs[0, n_req) to d_reqs and launches the batch on `s`.
sj_status serve_batch_launch(ServeReq* h_reqs, int n_req, ServeReq* d_reqs, unsigned* d_item_ctr, int device,
                             cudaStream_t s);

}  // namespace sj
