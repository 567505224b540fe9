// Stand-in: rmm::device_buffer, stream-ordered device memory from a resource.
#pragma once
#include <cstddef>
#include <optional>
#include <utility>
#include "rmm/resource_ref.hpp"
namespace rmm {
class device_buffer {
 public:
  device_buffer() = default;
  device_buffer(std::size_t size, cuda_stream_view stream,
                device_async_resource_ref mr = mr::get_current_device_resource_ref())
    : size_(size), stream_(stream), mr_(mr) {
    if (size_) data_ = mr.allocate_async(size_, 256, stream);
  }
  device_buffer(device_buffer&& o) noexcept
    : data_(std::exchange(o.data_, nullptr)), size_(std::exchange(o.size_, 0)), stream_(o.stream_), mr_(o.mr_) {}
  device_buffer(device_buffer const&)            = delete;
  device_buffer& operator=(device_buffer const&) = delete;
  device_buffer& operator=(device_buffer&&)      = delete;
  ~device_buffer() {
    if (data_ && mr_) mr_->deallocate_async(data_, size_, 256, stream_);
  }
  void* data() noexcept { return data_; }
  [[nodiscard]] void const* data() const noexcept { return data_; }
  [[nodiscard]] std::size_t size() const noexcept { return size_; }

 private:
  void* data_{nullptr};
  std::size_t size_{0};
  cuda_stream_view stream_{};
  std::optional<device_async_resource_ref> mr_{};
};
}  // namespace rmm
