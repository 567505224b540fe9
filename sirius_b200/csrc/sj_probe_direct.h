// The direct write-out DISTINCT probe (sj_probe_direct.cu): its argument block and entry point.
#pragma once

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

constexpr int kDirectMaxProbePayload = 2;
constexpr int kDirectMaxBuildPayload = 3;

struct DirectArgs {
  int32_t* out_prid;
  int32_t* out_brid;
  const int32_t* prid_map;  // probe array index -> probe row id (partitioned probe), or NULL
  const int32_t* brid_map;  // table position -> build row id at brid_map + pos * brid_stride bytes
  int32_t brid_stride;
  int32_t bin_by_pos;       // build payload element index: table position (1) or build row id (0)
  const void* rec;          // row store (record = [row id | fields]) or NULL
  int32_t rec_stride;
  int32_t rec_std;          // fields are 8-byte at offsets 8, 16, 24 (else rec_off / bin_w)
  int16_t rec_off[kDirectMaxBuildPayload];
  int32_t n_pin, n_bin;
  const void* pin[kDirectMaxProbePayload];
  int32_t pin_w[kDirectMaxProbePayload];
  void* pout[kDirectMaxProbePayload];
  const void* bin[kDirectMaxBuildPayload];
  int32_t bin_stride[kDirectMaxBuildPayload];
  int32_t bin_w[kDirectMaxBuildPayload];
  void* bout[kDirectMaxBuildPayload];
  int64_t capacity;
  unsigned long long* d_count;
  unsigned long long* tile_ctr;  // zeroed device word: dynamic tile order of CTA-reserving launches
  int32_t l2_last;               // table slot and record loads marked L2 evict_last
};

// Partition runs of a tile-local partition (local_partition): rows of partition p in tile i are
// [run_off[i * P + p], + run_cnt[i * P + p]).
struct RunArgs {
  const int32_t* run_off;
  const int32_t* run_cnt;
  uint32_t n_tiles;
  uint32_t P;
  uint32_t group;  // tiles per work item (a power of two <= 16); set by probe_runs
};

// Fills `a` from a general gather description; false when the output shape needs the staged
// kernel (NULL payloads, 1/2-byte payloads, too many columns, other record layouts).
bool direct_args(const GatherArgs& g, DirectArgs& a);

// Launches the direct probe of DISTINCT table `t` when the shape allows and the table's
// parameters do not ask for the staged kernel; returns false (nothing launched) otherwise.
// `tile_ctr`: a device word the launch may use as its tile counter (zeroed here, on `s`); when NULL
// and a counter is needed, one is drawn from `alloc`.
bool probe_direct(const sj_table* t, const sj_column& p, const int64_t* d_n, const GatherArgs& g, cudaStream_t s,
                  const Allocator& alloc, unsigned long long* tile_ctr);

// True when probe_runs serves this gather (DIRECT write-out shape, CTA reservation).
bool probe_runs_ok(const sj_table* t, const GatherArgs& g);

// Probe of tile-local partition runs: `keys`, the partition row ids and payloads in `g` are the
// partitioned arrays; work items (partition, group of tiles) are taken partition-major from
// `tile_ctr` (zeroed here). Requires probe_runs_ok.
void probe_runs(const sj_table* t, const void* keys, const RunArgs& ra, const GatherArgs& g, cudaStream_t s,
                unsigned long long* tile_ctr);

}  // namespace sj
