// Stand-in: rmm::device_buffer.
#pragma once
#include <cstddef>
#include "rmm/resource_ref.hpp"
namespace rmm {
class device_buffer {
 public:
  device_buffer();
  device_buffer(std::size_t size, cuda_stream_view stream,
                device_async_resource_ref mr = mr::get_current_device_resource_ref());
  device_buffer(device_buffer&&) noexcept;
  ~device_buffer();
  void* data() noexcept;
  [[nodiscard]] std::size_t size() const noexcept;
  void resize(std::size_t new_size, cuda_stream_view stream);
  void shrink_to_fit(cuda_stream_view stream);
};
}  // namespace rmm
