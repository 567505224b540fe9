// Radix partitioning shared by the build and the probe (implemented in sj_partition.cu).
#pragma once

#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

constexpr int kMaxPartitionBits = 10;

struct PartSrc {
  const void* keys;
  const uint32_t* kvalid;
  int64_t kvoff;
  int64_t n;
  int32_t n_pay;
  PayloadIn pay[kMaxPayload];
};

// Outputs. stride == 0: rid / pay[c] / valid8[c] are plain arrays. stride > 0: they point at
// their fields inside one record array of `stride` bytes per row (the table's row store).
struct PartDst {
  void* keys;
  int32_t* rid;
  void* pay[kMaxPayload];
  uint8_t* valid8[kMaxPayload];
  int32_t stride;
};

size_t partition_scratch_bytes(int pbits, int device);
// Tile-local variant (one pass, no histogram): each kTile-row tile (2048) is sorted by partition
// in place; run_off / run_cnt[tile * 2^pbits + p] give partition p's rows of every tile. Only for
// plain outputs with at most 2 payloads of 4/8 bytes without NULLs. NULL-key rows are dropped.
constexpr int kPartTileRows = 2048;
sj_status local_partition(const PartSrc& src, int key_type, int pbits, const PartDst& dst, int32_t* run_off,
                          int32_t* run_cnt, int device, cudaStream_t s);
bool partition_plain_shape(const PartSrc& src, const PartDst& dst);

sj_status radix_partition(const PartSrc& src, int key_type, int pbits, const PartDst& dst, void* scratch,
                          int device, cudaStream_t s, const int64_t** d_total_out, const int64_t** d_offs_out,
                          int* grid_out);

}  // namespace sj
