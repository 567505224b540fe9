// Stand-in: the cudf::table constructor the adapter uses.
#pragma once
#include <memory>
#include <vector>
#include "cudf/column/column.hpp"
namespace cudf {
class table {
 public:
  table(std::vector<std::unique_ptr<column>>&& columns, rmm::cuda_stream_view stream);
};
}  // namespace cudf
