/* Stand-in: the two CUDA runtime names the adapter uses (the real header is the CUDA toolkit's). */
#pragma once
#include <stddef.h>
struct CUstream_st;
typedef struct CUstream_st* cudaStream_t;
typedef int cudaError_t;
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
#define cudaSuccess 0
#ifdef __cplusplus
extern "C" {
#endif
cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t count, enum cudaMemcpyKind kind, cudaStream_t stream);
cudaError_t cudaStreamSynchronize(cudaStream_t stream);
#ifdef __cplusplus
}
#endif
