// Diagnostics: the library's bounded device waits, run on conditions that never come true, so a
// test can see them give up, report the timeout and return with the GPU context still usable.
//   1. the batched join's wait for a join's build tiles (wait_counter_at_least, as
//      batch_persistent_kernel uses it) on a counter that nothing increments;
//   2. the TMA probe ring's wait for a stage's bulk copies (mbar_wait_bounded, as probe_tma_kernel
//      uses it) on an initialised mbarrier that nothing arrives on and no copy completes.
// Neither wait has anything in flight when it gives up, so the kernel simply returns.
#include "sj_bulk.cuh"
#include "sj_device.cuh"
#include "sj_internal.h"

namespace sj {

__global__ void bounded_wait_probe_kernel(int32_t* status, uint32_t polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  const unsigned int* never = reinterpret_cast<const unsigned int*>(status + 2);  // zeroed by the host
  status[0] = wait_counter_at_least(never, 1u, polls) ? 0 : 1;
  mbar_init(&bar, 1);
  mbar_init_fence();
  status[1] = mbar_wait_bounded(&bar, 0, polls) ? 0 : 1;
}

}  // namespace sj

using namespace sj;

extern "C" SJ_EXPORT sj_status sj_debug_wait_timeout(int32_t polls, sj_stream_t stream, int32_t* d_status) {
  clear_error();
  if (!d_status) return set_error(SJ_ERR_INVALID, "d_status is NULL");
  if (polls < 1 || polls > (1 << 20)) return set_error(SJ_ERR_INVALID, "polls must be in [1, 2^20]");
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  SJ_CUDA_TRY(cudaMemsetAsync(d_status, 0, 3 * sizeof(int32_t), s));
  bounded_wait_probe_kernel<<<1, 32, 0, s>>>(d_status, (uint32_t)polls);
  SJ_CUDA_TRY(cudaGetLastError());
  return SJ_OK;
}
