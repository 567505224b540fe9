// Stand-in: the subset of rmm::cuda_stream_view the adapter uses.
#pragma once
struct CUstream_st;
#ifndef __CUDA_RUNTIME_H__
typedef struct CUstream_st* cudaStream_t;
#endif
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
