// noalloc.cu — gell_sort_keys_noalloc: the stable Morton-key sort of FM_update for callers that
// cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they need this sort: code running while a
// CUDA stream is being captured into a graph (an allocation there breaks the capture), callers
// that must not touch the device allocator at all (a pooled or pre-reserved memory budget, real-
// time loops that forbid allocation after start-up), and plain C callers that only own the input
// and output buffers.  This entry point takes the caller's input and output buffers and keeps its
// own scratch (the ping-pong key/index buffer and the digit-count table) in one file-scope device
// array of fixed size, so it never allocates.
//
// The array is a static __device__ object: every GPU that loads the library holds it (about
// 8.3 MB) until the process exits.  In host code its name is only a host-side stand-in, so the
// device address is looked up once per device with cudaGetSymbolAddress, with that device
// current, on the first call made on that device (and again on the first call under another
// driver context of the device); that first call should therefore come before any stream
// capture.  A cudaDeviceReset can leave a cached address stale (a new primary context may reuse
// the old handle), so a process that resets a device must not call this entry point again.  All
// calls share the one array and it keeps the last call's contents: nothing in it needs to start
// at zero (every table entry is written before it is read), and two calls whose work overlaps on
// the GPU race on it.  The call neither allocates nor frees anything.
#include <cuda.h>

#include <mutex>

#include "gell_internal.cuh"

namespace gell {

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaItems = 16;
constexpr int kNaTile = kNaThreads * kNaItems;  // 4096 keys per block
constexpr int kNaMaxTiles = (GELL_NOALLOC_MAX_KEYS + kNaTile - 1) / kNaTile;
constexpr unsigned kFull = 0xffffffffu;

// scratch: keys[MAX] | idx[MAX] | digit-major count table [256][kNaMaxTiles]
constexpr size_t kNaWords = 2 * (size_t)GELL_NOALLOC_MAX_KEYS + 256 * (size_t)kNaMaxTiles;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNaWords];

// Key of pass p: the reference's signed key (-1 = outside the grid) plus one, as unsigned.
__device__ __forceinline__ uint32_t ukey(int32_t k) { return (uint32_t)k + 1u; }

__global__ void __launch_bounds__(kNaThreads) na_hist(const uint32_t* __restrict__ keys, const int32_t* __restrict__ skeys,
                                                      int n, int shift, int R, uint32_t* __restrict__ hist, int nb) {
    __shared__ uint32_t h[256];
    for (int d = threadIdx.x; d < R; d += kNaThreads) h[d] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kNaTile;
    const uint32_t mask = (uint32_t)R - 1u;
    for (int k = 0; k < kNaItems; ++k) {
        const long long i = base + k * kNaThreads + threadIdx.x;
        if (i < n) {
            const uint32_t key = skeys ? ukey(skeys[i]) : keys[i];
            atomicAdd(&h[(key >> shift) & mask], 1u);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kNaThreads) hist[(long long)d * nb + blockIdx.x] = h[d];
}

// Exclusive scan of m entries in place by one block of 1024 threads.
__global__ void __launch_bounds__(1024) na_scan(uint32_t* a, long long m) {
    __shared__ uint32_t ws[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const long long per = (m + 1023) / 1024;
    const long long lo = t * per, hi = lo + per < m ? lo + per : m;
    uint32_t s = 0;
    for (long long i = lo; i < hi; ++i) s += a[i];
    uint32_t v = s;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        uint32_t x = ws[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        ws[lane] = x;
    }
    __syncthreads();
    uint32_t run = v - s + (w > 0 ? ws[w - 1] : 0u);
    for (long long i = lo; i < hi; ++i) {
        const uint32_t x = a[i];
        a[i] = run;
        run += x;
    }
}

// Stable scatter of one digit pass.  Item k of lane l of warp w is tile element w*512 + k*32 + l,
// ranked in that order, so equal digits keep their input order.  The first pass reads the
// caller's signed keys and uses the element index as the payload; the last pass writes the
// caller's outputs (signed keys, int32 permutation).
__global__ void __launch_bounds__(kNaThreads) na_scatter(const uint32_t* __restrict__ kin, const int32_t* __restrict__ skin,
                                                         const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
                                                         int32_t* __restrict__ skout, uint32_t* __restrict__ vout, int n,
                                                         int shift, int R, const uint32_t* __restrict__ offs, int nb) {
    __shared__ uint32_t wcnt[kNaThreads / 32][256];
    __shared__ uint32_t gbase[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kNaThreads / 32) * 256; i += kNaThreads) (&wcnt[0][0])[i] = 0;
    for (int d = threadIdx.x; d < R; d += kNaThreads) gbase[d] = offs[(long long)d * nb + blockIdx.x];
    __syncthreads();
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    const uint32_t mask = (uint32_t)R - 1u;
    const long long base = (long long)blockIdx.x * kNaTile + w * (kNaTile / (kNaThreads / 32));
    uint32_t key[kNaItems], loc[kNaItems];
#pragma unroll
    for (int k = 0; k < kNaItems; ++k) {
        const long long i = base + k * 32 + lane;
        const bool valid = i < n;
        key[k] = valid ? (skin ? ukey(skin[i]) : kin[i]) : 0u;
        const uint32_t dig = (key[k] >> shift) & mask;
        const unsigned peers = __match_any_sync(kFull, valid ? dig : 0xffffffffu);
        const uint32_t before = wcnt[w][dig & 255];
        loc[k] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0) wcnt[w][dig] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kNaThreads) {
        uint32_t run = 0;
        for (int ww = 0; ww < kNaThreads / 32; ++ww) {
            const uint32_t c = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kNaItems; ++k) {
        const long long i = base + k * 32 + lane;
        if (i < n) {
            const uint32_t dig = (key[k] >> shift) & mask;
            const uint32_t pos = gbase[dig] + wcnt[w][dig] + loc[k];
            const uint32_t val = skin ? (uint32_t)i : vin[i];
            if (skout) skout[pos] = (int32_t)(key[k] - 1u);
            else kout[pos] = key[k];
            vout[pos] = val;
        }
    }
}

// Device address of the scratch array, looked up with the device current and cached per device
// together with the driver context it was looked up in: a call made under another context of the
// same device (a non-primary context, or a primary context created anew) looks the address up again.
struct NaScratch {
    void* ctx;
    uint32_t* ptr;
};
std::mutex g_na_mutex;
NaScratch g_na_cache[64] = {};

using CtxGetCurrent = CUresult (*)(CUcontext*);

cudaError_t current_context(void** out) {
    static CtxGetCurrent fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (q != cudaDriverEntryPointSuccess || !f) return cudaErrorNotSupported;
        fn = reinterpret_cast<CtxGetCurrent>(f);
    }
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    *out = c;
    return cudaSuccess;
}

cudaError_t scratch_for_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    void* ctx = nullptr;  // null before the runtime has made the device's primary context current
    e = current_context(&ctx);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    NaScratch& c = g_na_cache[dev];
    if (!c.ptr || !ctx || c.ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        if (!ctx) {
            e = current_context(&ctx);
            if (e != cudaSuccess) return e;
        }
        c.ptr = static_cast<uint32_t*>(p);
        c.ctx = ctx;
    }
    *out = c.ptr;
    return cudaSuccess;
}

// Whether [a, a + n) and [b, b + n) (int32 elements) share any byte.
bool overlap(const void* a, const void* b, int n) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)n * sizeof(int32_t);
    return x < y + len && y < x + len;
}

}  // namespace

}  // namespace gell

extern "C" gell_status gell_sort_keys_noalloc(const int32_t* keys, int32_t* sorted_keys, int32_t* perm, int n,
                                              int key_bits, void* stream) {
    using namespace gell;
    if (n < 0 || (n > 0 && (!keys || !sorted_keys || !perm))) return GELL_ERR_INVALID_ARG;
    if (key_bits < 1 || key_bits > 32) return GELL_ERR_INVALID_ARG;
    if (n > GELL_NOALLOC_MAX_KEYS) return GELL_ERR_CAPACITY;
    if (n == 0) return GELL_OK;
    // pass 0 reads keys while (for an odd pass count) it writes the outputs, and the passes use
    // sorted_keys and perm as two separate ping-pong buffers: the three must not share memory
    if (overlap(keys, sorted_keys, n) || overlap(keys, perm, n) || overlap(sorted_keys, perm, n))
        return GELL_ERR_INVALID_ARG;
    // an error left pending by the caller's earlier work is reported as it is, not consumed here
    if (cudaPeekAtLastError() != cudaSuccess) return GELL_ERR_CUDA;
    uint32_t* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();  // the failed look-up's own error
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? GELL_ERR_NO_DEVICE : GELL_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t* sk = scratch;                                  // scratch keys
    uint32_t* sv = scratch + GELL_NOALLOC_MAX_KEYS;          // scratch payload
    uint32_t* hist = scratch + 2 * (size_t)GELL_NOALLOC_MAX_KEYS;
    uint32_t* ok = reinterpret_cast<uint32_t*>(sorted_keys);  // output buffers double as ping-pong
    uint32_t* ov = reinterpret_cast<uint32_t*>(perm);
    const int nb = (n + kNaTile - 1) / kNaTile;
    const int passes = (key_bits + 7) / 8;
    const int d = (key_bits + passes - 1) / passes;
    const int R = 1 << d;
    // the passes alternate between scratch and the outputs, ending in the outputs
    bool to_out = (passes % 2) == 1;
    const uint32_t* kin = nullptr;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * d;
        const int32_t* skin = p == 0 ? keys : nullptr;
        uint32_t* kout = to_out ? ok : sk;
        uint32_t* vout = to_out ? ov : sv;
        int32_t* skout = (p == passes - 1) ? sorted_keys : nullptr;
        na_hist<<<nb, kNaThreads, 0, s>>>(kin, skin, n, shift, R, hist, nb);
        na_scan<<<1, 1024, 0, s>>>(hist, (long long)R * nb);
        na_scatter<<<nb, kNaThreads, 0, s>>>(kin, skin, vin, kout, skout, vout, n, shift, R, hist, nb);
        e = cudaGetLastError();
        if (e != cudaSuccess) return GELL_ERR_CUDA;
        kin = kout;
        vin = vout;
        to_out = !to_out;
    }
    return GELL_OK;
}
