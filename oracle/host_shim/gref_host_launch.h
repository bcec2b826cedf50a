// TEST INFRASTRUCTURE ONLY: a kernel launch on the host.  The reference's launch
//   kernel<<<grid, block>>>(args);
// is rewritten (oracle/make_ref_host.py) to
//   gref_host_launch(grid, block, [&] { kernel(args); });
// which runs every (block, thread) of the grid as one iteration of an OpenMP loop, with
// blockIdx/threadIdx set for the iteration.  The reference's FM and LOD kernels use neither
// shared memory nor __syncthreads, so each thread's body can run on its own.  Atomics are host
// atomics on the same addresses.
#pragma once
#include <omp.h>

#include <cstdint>
#include <cstring>

inline thread_local uint3 threadIdx;
inline thread_local uint3 blockIdx;
inline dim3 blockDim;
inline dim3 gridDim;

template <class F>
inline void gref_host_launch(dim3 g, dim3 b, F&& body) {
    gridDim = g;
    blockDim = b;
    const long long nt = (long long)b.x * b.y * b.z;
    const long long total = (long long)g.x * g.y * g.z * nt;
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < total; ++t) {
        const long long blk = t / nt, th = t - blk * nt;
        blockIdx = uint3{(unsigned)(blk % g.x), (unsigned)((blk / g.x) % g.y), (unsigned)(blk / ((long long)g.x * g.y))};
        threadIdx = uint3{(unsigned)(th % b.x), (unsigned)((th / b.x) % b.y), (unsigned)(th / ((long long)b.x * b.y))};
        body();
    }
}

inline float atomicAdd(float* a, float v) {
    uint32_t old = __atomic_load_n(reinterpret_cast<uint32_t*>(a), __ATOMIC_RELAXED);
    for (;;) {
        float f;
        std::memcpy(&f, &old, 4);
        const float n = f + v;
        uint32_t nu;
        std::memcpy(&nu, &n, 4);
        if (__atomic_compare_exchange_n(reinterpret_cast<uint32_t*>(a), &old, nu, true, __ATOMIC_RELAXED,
                                        __ATOMIC_RELAXED))
            return f;
    }
}
inline int atomicAdd(int* a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
inline int atomicMin(int* a, int v) {
    int old = __atomic_load_n(a, __ATOMIC_RELAXED);
    while (v < old && !__atomic_compare_exchange_n(a, &old, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
    return old;
}
inline int atomicMax(int* a, int v) {
    int old = __atomic_load_n(a, __ATOMIC_RELAXED);
    while (v > old && !__atomic_compare_exchange_n(a, &old, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
    return old;
}
