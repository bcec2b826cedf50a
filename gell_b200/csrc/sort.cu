// sort.cu — stable LSD radix sort of (u32 key, u32 payload) and a device-wide exclusive scan.
//
// Replaces thrust::sort_by_key (include/FMkernel.cuh:190, a stable cub radix sort of int keys
// carrying 72-byte Cell values) and the scan inside thrust::remove_if (include/PDkernel.cuh:103).
// Keys are the Morton code + 1 (0 for a cell outside the grid, so it orders first like the
// reference's -1), and only the bits a key of this grid can set are sorted.  Payloads are cell
// indices; the cell records themselves move once, in the gather that follows (mech.cu).
//
// One pass per digit of d <= 8 bits: k_hist (per-tile digit counts), k_scan_hist (one CTA, exclusive
// scan of the digit-major count table), k_scatter (stable rank inside the tile with warp match,
// then scatter).  A tile is 8 warps x 16 items; item k of lane l of warp w is tile element
// w*512 + k*32 + l, so processing k in order and lanes in order visits the tile in input order,
// which is what makes the ranks, and the sort, stable.
#include "mech_body.cuh"

namespace gell {

namespace {
__global__ void __launch_bounds__(kSortThreads) k_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                   int R, uint32_t* __restrict__ hist, int nb) {
    hist_body(keys, n, shift, R, hist, nb, blockIdx.x);
}

// Exclusive scan of m entries in place by one CTA of 1024 threads; total to *total if not null.
__global__ void __launch_bounds__(1024) k_scan_single(uint32_t* a, long long m, int* total) {
    __shared__ uint32_t warp_sums[32];
    const int t = threadIdx.x;
    const long long per = (m + 1023) / 1024;
    const long long lo = t * per, hi = lo + per < m ? lo + per : m;
    uint32_t s = 0;
    for (long long i = lo; i < hi; ++i) s += a[i];
    // block exclusive scan of s
    uint32_t v = s;
    const int lane = t & 31, w = t >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    if (w == 0) {
        uint32_t ws = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(FULL, ws, o);
            if (lane >= o) ws += y;
        }
        warp_sums[lane] = ws;
    }
    __syncthreads();
    uint32_t run = v - s + (w > 0 ? warp_sums[w - 1] : 0u);
    for (long long i = lo; i < hi; ++i) {
        uint32_t x = a[i];
        a[i] = run;
        run += x;
    }
    if (total && t == 1023) *total = (int)(warp_sums[31]);
}

__global__ void __launch_bounds__(kSortThreads) k_digit_scan(uint32_t* __restrict__ hist, int nb,
                                                         uint32_t* __restrict__ totals) {
    digit_scan_body(hist, nb, totals, blockIdx.x);
}

__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                      uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int n,
                                                      int shift, int R, const uint32_t* __restrict__ offs, int nb,
                                                      const uint32_t* __restrict__ totals, int iota) {
    scatter_body(kin, vin, kout, vout, n, shift, R, offs, nb, totals, iota, blockIdx.x);
}

// Scan helpers: per-tile sums, then tile-local exclusive scan plus the tile's offset.
__global__ void __launch_bounds__(kSortThreads) k_tile_sum(const uint32_t* __restrict__ in, int n, uint32_t* __restrict__ sums) {
    __shared__ uint32_t ws[kSortThreads / 32];
    const long long base = (long long)blockIdx.x * kSortTile;
    uint32_t s = 0;
#pragma unroll 4
    for (int k = 0; k < kSortItems; ++k) {
        long long i = base + k * kSortThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kSortThreads / 32; ++w) t += ws[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kSortThreads) k_tile_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int n,
                                                        const uint32_t* __restrict__ offs) {
    // thread t owns elements base + t*16 .. +15 (contiguous), so a thread-serial scan inside
    // plus a block scan over threads gives the tile's exclusive scan in order
    __shared__ uint32_t ws[kSortThreads / 32];
    const long long base = (long long)blockIdx.x * kSortTile + (long long)threadIdx.x * kSortItems;
    uint32_t v[kSortItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t wpre = 0;
    for (int j = 0; j < w; ++j) wpre += ws[j];
    uint32_t run = offs[blockIdx.x] + wpre + x - s;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        long long i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

}  // namespace

// digit-major count table, then the 256 digit totals
size_t sort_hist_entries(int cap) { return (size_t)256 * ((cap + kSortTile - 1) / kSortTile) + 256 + 64; }

gell_status radix_sort(gell_ctx* c, int n, int bits, bool vals_are_iota) {
    SortScratch& S = c->sort;
    int in = 0;
    if (n <= 0) {
        S.which = 0;
        return GELL_OK;
    }
    const int nb = (n + kSortTile - 1) / kSortTile;
    int passes = (bits + 7) / 8;
    if (passes < 1) passes = 1;
    const int d = (bits + passes - 1) / passes;
    const int R = 1 << d;
    bool iota = vals_are_iota;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * d;
        GELL_KERNEL(c, "k_hist", k_hist<<<nb, kSortThreads, 0, c->stream>>>(S.keys[in], n, shift, R, S.hist, nb));
        uint32_t* totals = S.hist + (size_t)R * nb;
        GELL_KERNEL(c, "k_digit_scan", k_digit_scan<<<R, kSortThreads, 0, c->stream>>>(S.hist, nb, totals));
        GELL_KERNEL(c, "k_scatter", k_scatter<<<nb, kSortThreads, 0, c->stream>>>(S.keys[in], S.vals[in], S.keys[in ^ 1], S.vals[in ^ 1], n, shift,
                                                   R, S.hist, nb, totals, iota ? 1 : 0));
        iota = false;
        in ^= 1;
    }
    S.which = in;
    return GELL_OK;
}

gell_status scan_u32(gell_ctx* c, const uint32_t* in, uint32_t* out, int n, int* total_dev) {
    if (n <= 0) {
        GELL_CUDA(c, cudaMemsetAsync(total_dev, 0, 4, c->stream));
        return GELL_OK;
    }
    const int nb = (n + kSortTile - 1) / kSortTile;
    GELL_KERNEL(c, "k_tile_sum", k_tile_sum<<<nb, kSortThreads, 0, c->stream>>>(in, n, c->scan_tmp));
    GELL_KERNEL(c, "k_scan_single", k_scan_single<<<1, 1024, 0, c->stream>>>(c->scan_tmp, nb, total_dev));
    GELL_KERNEL(c, "k_tile_scan", k_tile_scan<<<nb, kSortThreads, 0, c->stream>>>(in, out, n, c->scan_tmp));
    return GELL_OK;
}

}  // namespace gell
