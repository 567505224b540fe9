// Stand-in: rmm::device_async_resource_ref (allocate_async / deallocate_async) and the
// out-of-memory exception type.
#pragma once
#include <cstddef>
#include <stdexcept>
#include "rmm/cuda_stream_view.hpp"
namespace rmm {
class device_async_resource_ref {
 public:
  void* allocate_async(std::size_t bytes, std::size_t alignment, cuda_stream_view stream);
  void deallocate_async(void* p, std::size_t bytes, std::size_t alignment, cuda_stream_view stream) noexcept;
};
struct bad_alloc : std::bad_alloc {
  explicit bad_alloc(const char*) {}
};
struct out_of_memory : bad_alloc {
  explicit out_of_memory(const char* m) : bad_alloc(m) {}
};
namespace mr {
device_async_resource_ref get_current_device_resource_ref();
}
}  // namespace rmm
