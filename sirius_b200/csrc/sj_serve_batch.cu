// Continuous batching of small served probe requests: every small request admitted together runs
// in ONE kernel launch over the resident tables, instead of one launch (plus a count copy and a
// host callback) per request.
//
// A batch is a list of request descriptors, each naming its own resident table (by value: the
// TableDev view plus its row store), its probe keys and its own outputs and match counter. Work
// items are 256-row slices of the requests, numbered request after request; a warp takes the next
// item from a counter, finds its request with a binary search over the requests' first items
// (held in shared memory), and probes the slice in steps of 32 x R rows exactly as the direct
// DISTINCT probe does: lane l handles rows base + 32 j + l, one bucket walk per row, one row-store
// load per match (build row id and the attached 8-byte fields), and the step's matches are ranked
// with ballots and reserved with one atomicAdd on that request's counter.
// Served tables are DISTINCT (unique keys), so a request never has more matches than probe rows.
#include <algorithm>

#include "sj_device.cuh"
#include "sj_internal.h"
#include "sj_serve_batch.h"

namespace sj {

TableDev table_dev(const sj_table* t);

constexpr int kItemRows = 256;  // rows per work item: a 30K-row request spreads over ~120 warps
constexpr int kServeThreads = 256;
constexpr int kServeR = 2;

template <bool WIDE>
__device__ __forceinline__ void serve_step(const ServeReq& q, int64_t base) {
  using Ops = SlotOps<WIDE>;
  constexpr int R = kServeR;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const uint64_t kmask = ~((1ull << q.t.rbits) - 1);
  uint32_t act = 0;
  uint32_t b[R];
  uint64_t ks[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int64_t r = base + 32 * j + lane;
    int64_t k = 0;
    bool live = r < q.n && bit_valid(q.kvalid, q.kvoff, r);
    if (live) k = q.key64 ? __ldcs(static_cast<const long long*>(q.keys) + r)
                          : (int64_t)__ldcs(static_cast<const int*>(q.keys) + r);
    live = live && k >= q.t.kmin && k <= q.t.kmax;
    if (live) act |= 1u << j;
    b[j] = home_bucket(q.t, (uint64_t)k);
    ks[j] = Ops::probe_key((uint64_t)k - (uint64_t)q.t.kmin, (uint64_t)k, q.t.rbits);
  }
  int32_t pos[R];
  uint32_t hit = 0;
#pragma unroll
  for (int j = 0; j < R; ++j) pos[j] = 0;
  for (uint32_t step = 0; act && step <= q.t.segmask; ++step) {
    Bucket bk[R];
#pragma unroll
    for (int j = 0; j < R; ++j)
      if (act >> j & 1u) bk[j] = load_bucket<true>(q.t.slots, b[j]);
#pragma unroll
    for (int j = 0; j < R; ++j) {
      if (!(act >> j & 1u)) continue;
      int32_t pj;
      const bool m = Ops::match_distinct(bk[j], ks[j], kmask, q.t.rbits, pj);
      if (m) {
        pos[j] = pj;
        hit |= 1u << j;
      }
      if (m || Ops::open(bk[j])) act &= ~(1u << j);
      else b[j] = next_bucket(b[j], q.t.segmask);
    }
  }
  // build row id and attached fields: one row-store record per match (positions are the row ids
  // when the table keeps no row store)
  int32_t brid[R];
  uint64_t f[kServeMaxFields][R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    brid[j] = pos[j];
#pragma unroll
    for (int c = 0; c < kServeMaxFields; ++c) f[c][j] = 0;
    if (!(hit >> j & 1u) || !q.rec) continue;
    const Record rec = load_record(q.rec + (size_t)(uint32_t)pos[j] * q.rec_stride, q.rec_stride);
    brid[j] = (int32_t)rec.w[0];
#pragma unroll
    for (int c = 0; c < kServeMaxFields; ++c)
      if (c < q.n_fields) f[c][j] = ((uint64_t)rec.w[3 + 2 * c] << 32) | rec.w[2 + 2 * c];
  }
  unsigned bal[R];
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    bal[j] = __ballot_sync(kFullMask, hit >> j & 1u);
    tot += __popc(bal[j]);
  }
  if (tot == 0) return;
  unsigned long long p0 = 0;
  if (lane == 0) p0 = atomicAdd(q.count, (unsigned long long)tot);
  p0 = __shfl_sync(kFullMask, p0, 0);
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int64_t p = (int64_t)p0 + __popc(bal[j] & below);
    p0 += __popc(bal[j]);
    if (!(hit >> j & 1u) || p >= q.capacity) continue;
    if (q.out_prid) __stcs(q.out_prid + p, (int32_t)(base + 32 * j + lane));
    if (q.out_brid) __stcs(q.out_brid + p, brid[j]);
#pragma unroll
    for (int c = 0; c < kServeMaxFields; ++c)
      if (c < q.n_fields) __stcs(reinterpret_cast<unsigned long long*>(q.out_field[c]) + p, (unsigned long long)f[c][j]);
  }
}

__global__ void __launch_bounds__(kServeThreads) serve_batch_kernel(const ServeReq* __restrict__ reqs, int n_req,
                                                                    uint32_t n_items, unsigned* item_ctr) {
  __shared__ uint32_t s_first[kServeMaxBatch];
  for (int i = threadIdx.x; i < n_req; i += blockDim.x) s_first[i] = reqs[i].first_item;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(item_ctr, 1u);
    it = __shfl_sync(kFullMask, it, 0);
    if (it >= n_items) break;
    int lo = 0, hi = n_req - 1;  // the last request whose first item is <= it
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_first[mid] <= it) lo = mid;
      else hi = mid - 1;
    }
    const ServeReq& q = reqs[lo];
    const int64_t row0 = (int64_t)(it - s_first[lo]) * kItemRows;
    const int64_t row1 = row0 + kItemRows < q.n ? row0 + kItemRows : q.n;
    for (int64_t base = row0; base < row1; base += 32 * kServeR) {
      if (q.wide) serve_step<true>(q, base);
      else serve_step<false>(q, base);
    }
  }
}

bool serve_batchable(const sj_table* t, int64_t probe_rows) {
  if (t->layout != SJ_LAYOUT_DISTINCT || probe_rows <= 0 || probe_rows >= kMinPartitionedProbe) return false;
  if (t->n_attached > kServeMaxFields) return false;
  if (t->n_attached == 0) return true;
  // attached fields: 8-byte values without NULLs at bytes 8, 16, 24 of a row-store record
  if (!t->arow || t->arow_stride > 32) return false;
  for (int c = 0; c < t->n_attached; ++c) {
    if (type_width(t->apay_type[c]) != 8 || t->apay_valid[c]) return false;
    if (static_cast<const char*>(t->apay[c]) - static_cast<const char*>(t->arow) != 8 + 8 * c) return false;
  }
  return true;
}

ServeReq serve_request(const sj_table* t, const sj_column& key, int32_t* prid, int32_t* brid, void* const* fields,
                       unsigned long long* count) {
  ServeReq q{};
  q.t = table_dev(t);
  q.keys = key.data;
  q.kvalid = key.validity;
  q.kvoff = key.validity_offset;
  q.n = key.num_rows;
  q.key64 = t->key_type == SJ_INT64;
  q.wide = t->slot_kind == SJ_SLOT_WIDE128;
  if (t->arow) {
    q.rec = static_cast<const char*>(t->arow);
    q.rec_stride = t->arow_stride;
  } else if (t->pos_rid) {
    q.rec = reinterpret_cast<const char*>(t->pos_rid);
    q.rec_stride = t->pos_stride;
  }
  q.n_fields = t->n_attached;
  q.out_prid = prid;
  q.out_brid = brid;
  for (int c = 0; c < t->n_attached; ++c) q.out_field[c] = fields[c];
  q.count = count;
  q.capacity = key.num_rows;
  return q;
}

sj_status serve_batch_launch(ServeReq* h_reqs, int n_req, ServeReq* d_reqs, unsigned* d_item_ctr, int device,
                             cudaStream_t s) {
  if (n_req <= 0 || n_req > kServeMaxBatch) return set_error(SJ_ERR_INVALID, "bad serve batch size");
  uint32_t items = 0;
  for (int i = 0; i < n_req; ++i) {
    h_reqs[i].first_item = items;
    items += (uint32_t)((h_reqs[i].n + kItemRows - 1) / kItemRows);
  }
  SJ_CUDA_TRY(cudaMemcpyAsync(d_reqs, h_reqs, sizeof(ServeReq) * n_req, cudaMemcpyHostToDevice, s));
  SJ_CUDA_TRY(cudaMemsetAsync(d_item_ctr, 0, sizeof(unsigned), s));
  const int warps = kServeThreads / 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((items + warps - 1) / warps, (int64_t)sm_count(device) * 8));
  KernelTimer timer("serve_batch", s);
  serve_batch_kernel<<<grid, kServeThreads, 0, s>>>(d_reqs, n_req, items, d_item_ctr);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}

}  // namespace sj
