// Out-of-line parts of the stand-in cuDF / RMM names (adapter/standin), so the Sirius adapter can
// run in a test: a stream-ordered device resource over cudaMallocAsync that keeps a ledger of its
// live allocations and can refuse the Nth one (as a fully committed memory reservation refuses),
// null counts, column deep copies and stream synchronisation.
#include "standin_runtime.hpp"

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "cudf/column/column.hpp"
#include "cudf/null_mask.hpp"
#include "rmm/cuda_stream_view.hpp"
#include "rmm/device_buffer.hpp"
#include "rmm/resource_ref.hpp"

extern "C" cudaError_t cudaMemcpy(void* dst, const void* src, size_t count, enum cudaMemcpyKind kind);

namespace standin {

void* ledger_resource::allocate_async(std::size_t bytes, std::size_t, rmm::cuda_stream_view stream) {
  ++calls;
  if (fail_at > 0 && calls == fail_at) throw rmm::out_of_memory("standin: allocation refused");
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, stream.value()) != cudaSuccess || p == nullptr)
    throw rmm::out_of_memory("standin: cudaMallocAsync failed");
  live += 1;
  live_bytes += static_cast<int64_t>(bytes);
  return p;
}

void ledger_resource::deallocate_async(void* p, std::size_t bytes, std::size_t, rmm::cuda_stream_view stream) noexcept {
  cudaFreeAsync(p, stream.value());
  live -= 1;
  live_bytes -= static_cast<int64_t>(bytes);
}

ledger_resource& current() {
  static ledger_resource r;
  return r;
}

int width_of(cudf::data_type t) {
  using cudf::type_id;
  switch (t.id()) {
    case type_id::INT8: case type_id::UINT8: case type_id::BOOL8: return 1;
    case type_id::INT16: case type_id::UINT16: return 2;
    case type_id::INT32: case type_id::UINT32: case type_id::FLOAT32: case type_id::TIMESTAMP_DAYS:
    case type_id::DURATION_DAYS: case type_id::DECIMAL32: return 4;
    default: return 8;
  }
}

}  // namespace standin

namespace rmm {
void cuda_stream_view::synchronize() const { cudaStreamSynchronize(s_); }
namespace mr {
device_async_resource_ref get_current_device_resource_ref() { return device_async_resource_ref(standin::current()); }
}  // namespace mr
}  // namespace rmm

namespace cudf {

size_type null_count(bitmask_type const* bitmask, size_type start, size_type stop, rmm::cuda_stream_view stream) {
  if (bitmask == nullptr || stop <= start) return 0;
  std::vector<bitmask_type> h(static_cast<size_t>((stop + 31) / 32));
  stream.synchronize();
  cudaMemcpy(h.data(), bitmask, h.size() * sizeof(bitmask_type), cudaMemcpyDeviceToHost);
  size_type n = 0;
  for (size_type i = start; i < stop; ++i) n += ((h[i / 32] >> (i % 32)) & 1u) ? 0 : 1;
  return n;
}

column::column(column_view view, rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr)
  : type_(view.type()), size_(view.size()),
    data_(static_cast<std::size_t>(view.size()) * standin::width_of(view.type()), stream, mr),
    mask_(view.nullable() ? static_cast<std::size_t>((view.size() + 31) / 32) * 4 : 0, stream, mr),
    null_count_(view.null_count()) {
  const int w = standin::width_of(view.type());
  if (data_.size())
    cudaMemcpyAsync(data_.data(), static_cast<char const*>(view.head()) + static_cast<int64_t>(view.offset()) * w,
                    data_.size(), cudaMemcpyDeviceToDevice, stream.value());
  if (mask_.size()) {
    if (view.offset() % 32 != 0) throw std::runtime_error("standin: deep copy of a bit-offset mask");
    cudaMemcpyAsync(mask_.data(), view.null_mask() + view.offset() / 32, mask_.size(), cudaMemcpyDeviceToDevice,
                    stream.value());
  }
}

}  // namespace cudf
