// The stand-in device resource of the adapter test (see standin_runtime.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

#include "cudf/types.hpp"
#include "rmm/resource_ref.hpp"

namespace standin {

// cudaMallocAsync / cudaFreeAsync with a ledger: live allocations and bytes, the number of
// allocation calls, and an optional refusal of call number fail_at (1-based; 0 = never).
struct ledger_resource final : rmm::mr::device_memory_resource {
  int64_t calls = 0, fail_at = 0, live = 0, live_bytes = 0;
  void* allocate_async(std::size_t bytes, std::size_t alignment, rmm::cuda_stream_view stream) override;
  void deallocate_async(void* p, std::size_t bytes, std::size_t alignment, rmm::cuda_stream_view stream) noexcept override;
};

ledger_resource& current();
int width_of(cudf::data_type t);

}  // namespace standin
