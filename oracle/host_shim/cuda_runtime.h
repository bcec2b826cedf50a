// TEST INFRASTRUCTURE ONLY: host stand-in for the CUDA runtime header, so that the reference's
// kernel bodies compile with g++ -fopenmp as plain C++ (the CPU baseline).  Device memory is host
// memory, copies are memcpy, synchronisation is a no-op (launches are synchronous OpenMP loops,
// see gref_host_launch.h).  Only what the reference's FM and LOD headers use is provided.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline

struct float3 { float x, y, z; };
struct int3 { int x, y, z; };
struct uint3 { unsigned x, y, z; };
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }

enum cudaError_t { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                      cudaMemcpyDeviceToDevice, cudaMemcpyDefault };
enum cudaLimit { cudaLimitStackSize, cudaLimitPrintfFifoSize, cudaLimitMallocHeapSize };

template <class T>
inline cudaError_t cudaMalloc(T** p, size_t bytes) {
    *p = static_cast<T*>(std::malloc(bytes ? bytes : 1));
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t bytes, cudaMemcpyKind) {
    std::memcpy(d, s, bytes);
    return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaDeviceGetLimit(size_t* v, cudaLimit) {
    *v = 0;
    return cudaSuccess;
}
inline cudaError_t cudaMemGetInfo(size_t* f, size_t* t) {
    *f = *t = 0;
    return cudaSuccess;
}

#include "gref_host_launch.h"
