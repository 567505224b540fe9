// Stand-in: cudf::column_view, with the constructor and accessors the adapter and its test use.
#pragma once
#include "cudf/types.hpp"
namespace cudf {
class column_view {
 public:
  column_view() = default;
  column_view(data_type type, size_type size, void const* data, bitmask_type const* null_mask,
              size_type null_count, size_type offset = 0)
    : type_(type), size_(size), data_(data), mask_(null_mask), null_count_(null_count), offset_(offset) {}
  [[nodiscard]] data_type type() const noexcept { return type_; }
  [[nodiscard]] size_type size() const noexcept { return size_; }
  [[nodiscard]] size_type offset() const noexcept { return offset_; }
  [[nodiscard]] bool nullable() const noexcept { return mask_ != nullptr; }
  [[nodiscard]] size_type null_count() const { return null_count_; }
  [[nodiscard]] bitmask_type const* null_mask() const noexcept { return mask_; }
  template <typename T = void>
  [[nodiscard]] T const* head() const noexcept { return static_cast<T const*>(data_); }

 private:
  data_type type_{type_id::EMPTY};
  size_type size_{0};
  void const* data_{nullptr};
  bitmask_type const* mask_{nullptr};
  size_type null_count_{0};
  size_type offset_{0};
};
}  // namespace cudf
