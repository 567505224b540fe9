// Stand-in: cudf::null_count over a bitmask range.
#pragma once
#include "cudf/types.hpp"
#include "rmm/cuda_stream_view.hpp"
namespace cudf {
size_type null_count(bitmask_type const* bitmask, size_type start, size_type stop, rmm::cuda_stream_view stream);
}  // namespace cudf
