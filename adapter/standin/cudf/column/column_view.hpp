// Stand-in: cudf::column_view accessors used by the adapter.
#pragma once
#include "cudf/types.hpp"
namespace cudf {
class column_view {
 public:
  [[nodiscard]] data_type type() const noexcept;
  [[nodiscard]] size_type size() const noexcept;
  [[nodiscard]] size_type offset() const noexcept;
  [[nodiscard]] bool nullable() const noexcept;
  [[nodiscard]] size_type null_count() const;
  [[nodiscard]] bitmask_type const* null_mask() const noexcept;
  template <typename T = void>
  [[nodiscard]] T const* head() const noexcept;
};
}  // namespace cudf
