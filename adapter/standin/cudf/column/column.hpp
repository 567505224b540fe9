// Stand-in: the cudf::column constructors the adapter uses.
#pragma once
#include <memory>
#include "cudf/column/column_view.hpp"
#include "rmm/cuda_stream_view.hpp"
#include "rmm/device_buffer.hpp"
#include "rmm/resource_ref.hpp"
namespace cudf {
class column {
 public:
  column(data_type dtype, size_type size, rmm::device_buffer&& data, rmm::device_buffer&& null_mask,
         size_type null_count);
  // deep copy of a view
  column(column_view view, rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr);
};
}  // namespace cudf
