// Stand-in: cudf::table, owning its columns.
#pragma once
#include <memory>
#include <utility>
#include <vector>
#include "cudf/column/column.hpp"
#include "cudf/table/table_view.hpp"
namespace cudf {
class table {
 public:
  table(std::vector<std::unique_ptr<column>>&& columns, rmm::cuda_stream_view)
    : cols_(std::move(columns)) {}
  [[nodiscard]] size_type num_columns() const noexcept { return static_cast<size_type>(cols_.size()); }
  [[nodiscard]] size_type num_rows() const noexcept { return cols_.empty() ? 0 : cols_[0]->size(); }
  [[nodiscard]] column const& get_column(size_type i) const { return *cols_.at(static_cast<size_t>(i)); }
  std::vector<std::unique_ptr<column>> release() { return std::move(cols_); }
  [[nodiscard]] table_view view() const {
    std::vector<column_view> v;
    for (auto const& c : cols_) v.push_back(c->view());
    return table_view(v);
  }

 private:
  std::vector<std::unique_ptr<column>> cols_;
};
}  // namespace cudf
