// Stand-in: the subset of rmm::cuda_stream_view the adapter uses.
#pragma once
#include "cuda_runtime_api.h"
namespace rmm {
class cuda_stream_view {
 public:
  constexpr cuda_stream_view() = default;
  constexpr cuda_stream_view(cudaStream_t s) : s_(s) {}
  [[nodiscard]] constexpr cudaStream_t value() const noexcept { return s_; }
  void synchronize() const;
 private:
  cudaStream_t s_{nullptr};
};
}  // namespace rmm
