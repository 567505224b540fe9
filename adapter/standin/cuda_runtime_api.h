/* Stand-in: the CUDA runtime names the adapter (and the stand-in runtime that lets it run in a
 * test) use. The real header is the CUDA toolkit's; these declarations have the same C names and
 * argument meaning, so the adapter links against the real libcudart. */
#pragma once
#include <stddef.h>
struct CUstream_st;
typedef struct CUstream_st* cudaStream_t;
typedef int cudaError_t;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
                      cudaMemcpyDeviceToDevice = 3 };
#define cudaSuccess 0
#ifdef __cplusplus
extern "C" {
#endif
cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t count, enum cudaMemcpyKind kind, cudaStream_t stream);
cudaError_t cudaStreamSynchronize(cudaStream_t stream);
cudaError_t cudaMallocAsync(void** ptr, size_t size, cudaStream_t stream);
cudaError_t cudaFreeAsync(void* ptr, cudaStream_t stream);
cudaError_t cudaMemsetAsync(void* ptr, int value, size_t count, cudaStream_t stream);
#ifdef __cplusplus
}
#endif
