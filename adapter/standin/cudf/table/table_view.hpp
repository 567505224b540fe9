// Stand-in: cudf::table_view accessors used by the adapter.
#pragma once
#include <vector>
#include "cudf/column/column_view.hpp"
namespace cudf {
class table_view {
 public:
  [[nodiscard]] size_type num_columns() const noexcept;
  [[nodiscard]] size_type num_rows() const noexcept;
  [[nodiscard]] column_view const& column(size_type i) const;
  [[nodiscard]] table_view select(std::vector<size_type> const& idx) const;
};
}  // namespace cudf
