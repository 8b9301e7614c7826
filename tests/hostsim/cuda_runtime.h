#pragma once
// Test infrastructure: a stand-in for the CUDA runtime header, so that
// fa_api.cu's host-side packing helpers compile for the host simulation.
// The simulation never calls the runtime; every stub fails.
#include <stddef.h>
typedef int cudaError_t;
typedef struct CUstream_st* cudaStream_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1 };
enum { cudaDevAttrMultiProcessorCount = 16 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };
enum { cudaStreamNonBlocking = 1 };
#define STUB(name) template <class... A> static inline cudaError_t name(A...) { return 1; }
STUB(cudaDeviceGetAttribute) STUB(cudaDeviceSynchronize) STUB(cudaFree) STUB(cudaFreeHost) STUB(cudaGetDevice)
STUB(cudaGetDeviceCount) STUB(cudaGetLastError) STUB(cudaMalloc) STUB(cudaMallocHost) STUB(cudaMemcpy)
STUB(cudaMemcpyAsync) STUB(cudaMemset) STUB(cudaMemsetAsync) STUB(cudaSetDevice) STUB(cudaStreamCreateWithFlags)
STUB(cudaStreamDestroy) STUB(cudaStreamSynchronize) STUB(cudaMemcpy2D) STUB(cudaHostGetDevicePointer)
static inline const char* cudaGetErrorString(cudaError_t) { return "host simulation"; }
