// Stand-in: cudf::column, owning its data and null mask (device buffers).
#pragma once
#include <memory>
#include <utility>
#include "cudf/column/column_view.hpp"
#include "rmm/cuda_stream_view.hpp"
#include "rmm/device_buffer.hpp"
#include "rmm/resource_ref.hpp"
namespace cudf {
class column {
 public:
  column(data_type dtype, size_type size, rmm::device_buffer&& data, rmm::device_buffer&& null_mask,
         size_type null_count)
    : type_(dtype), size_(size), data_(std::move(data)), mask_(std::move(null_mask)), null_count_(null_count) {}
  // deep copy of a view
  column(column_view view, rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr);
  [[nodiscard]] column_view view() const {
    return column_view(type_, size_, data_.data(),
                       mask_.size() ? static_cast<bitmask_type const*>(mask_.data()) : nullptr, null_count_);
  }
  [[nodiscard]] size_type size() const noexcept { return size_; }
  [[nodiscard]] size_type null_count() const noexcept { return null_count_; }
  [[nodiscard]] data_type type() const noexcept { return type_; }

 private:
  data_type type_;
  size_type size_;
  rmm::device_buffer data_;
  rmm::device_buffer mask_;
  size_type null_count_;
};
}  // namespace cudf
