// Stand-in: cudf::table_view, a list of column views.
#pragma once
#include <vector>
#include "cudf/column/column_view.hpp"
namespace cudf {
class table_view {
 public:
  table_view() = default;
  explicit table_view(std::vector<column_view> const& cols) : cols_(cols) {}
  [[nodiscard]] size_type num_columns() const noexcept { return static_cast<size_type>(cols_.size()); }
  [[nodiscard]] size_type num_rows() const noexcept { return cols_.empty() ? 0 : cols_[0].size(); }
  [[nodiscard]] column_view const& column(size_type i) const { return cols_.at(static_cast<size_t>(i)); }
  [[nodiscard]] table_view select(std::vector<size_type> const& idx) const {
    std::vector<column_view> out;
    for (size_type i : idx) out.push_back(column(i));
    return table_view(out);
  }

 private:
  std::vector<column_view> cols_;
};
}  // namespace cudf
