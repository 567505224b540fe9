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
sj_status radix_partition(const PartSrc& src, int key_type, int pbits, const PartDst& dst, void* scratch,
                          int device, cudaStream_t s, const int64_t** d_total_out, const int64_t** d_offs_out,
                          int* grid_out);

}  // namespace sj
