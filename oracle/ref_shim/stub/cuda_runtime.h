/* Host stand-in for <cuda_runtime.h>: device memory is host memory. */
#pragma once
#include "shim_cuda.h"

typedef int cudaError_t;
enum { cudaSuccess = 0 };
typedef void* cudaStream_t;
typedef void* cudaEvent_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost,
    cudaMemcpyHostToDevice,
    cudaMemcpyDeviceToHost,
    cudaMemcpyDeviceToDevice
};
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
inline cudaError_t cudaMalloc(void** p, size_t n)
{
    *p = calloc(1, n ? n : 1);
    return 0;
}
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t n)
{
    return cudaMalloc((void**)p, n);
}
inline cudaError_t cudaFree(void* p)
{
    free(p);
    return 0;
}
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind)
{
    memcpy(d, s, n);
    return 0;
}
inline cudaError_t cudaMemset(void* d, int v, size_t n)
{
    memset(d, v, n);
    return 0;
}
inline cudaError_t cudaDeviceSynchronize() { return 0; }
inline const char* cudaGetErrorString(cudaError_t) { return "host shim"; }
