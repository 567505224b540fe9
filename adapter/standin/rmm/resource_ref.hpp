// Stand-in: rmm::device_async_resource_ref (a non-owning reference to a stream-ordered device
// memory resource: allocate_async / deallocate_async) and the out-of-memory exception type.
#pragma once
#include <cstddef>
#include <new>
#include <stdexcept>
#include "rmm/cuda_stream_view.hpp"
namespace rmm {
namespace mr {
// What a resource reference points at (the real one is a cuda::mr async resource).
class device_memory_resource {
 public:
  virtual ~device_memory_resource() = default;
  virtual void* allocate_async(std::size_t bytes, std::size_t alignment, cuda_stream_view stream) = 0;
  virtual void deallocate_async(void* p, std::size_t bytes, std::size_t alignment,
                                cuda_stream_view stream) noexcept = 0;
};
}  // namespace mr
class device_async_resource_ref {
 public:
  device_async_resource_ref(mr::device_memory_resource& r) : r_(&r) {}  // NOLINT: implicit, as RMM's
  void* allocate_async(std::size_t bytes, std::size_t alignment, cuda_stream_view stream) {
    return r_->allocate_async(bytes, alignment, stream);
  }
  void deallocate_async(void* p, std::size_t bytes, std::size_t alignment, cuda_stream_view stream) noexcept {
    r_->deallocate_async(p, bytes, alignment, stream);
  }

 private:
  mr::device_memory_resource* r_;
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
