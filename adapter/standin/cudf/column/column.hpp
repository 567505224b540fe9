// Stand-in: the cudf::column constructor the adapter uses.
#pragma once
#include <memory>
#include "cudf/column/column_view.hpp"
#include "rmm/device_buffer.hpp"
namespace cudf {
class column {
 public:
  column(data_type dtype, size_type size, rmm::device_buffer&& data, rmm::device_buffer&& null_mask,
         size_type null_count);
};
}  // namespace cudf
