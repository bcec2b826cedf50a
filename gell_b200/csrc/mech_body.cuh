// mech_body.cuh — the per-block bodies of the mechanics kernels (mech.cu: keys, gather, force and
// move; sort.cu: the radix sort's histogram, digit scan and scatter; lod.cu: the uptake map), shared
// by the one-context kernels and the ensemble's batched kernels (mech_batch.cu), which run the same
// body for block `blk` of one member.  Each body is the kernel it came from with blockIdx.x
// replaced by `blk`, so a batched launch computes what the member's own launches compute.
#pragma once

#include "async_copy.cuh"
#include "gell_internal.cuh"

namespace gell {

// ------------------------------------------------------------------ FM_update (mech.cu)

// Also advances the cell-list epoch, which lives in device memory so that a captured step reads
// the current one when it is replayed.
__device__ __forceinline__ void keys_body(const CellsSoA& c, int n, const Geom& g, uint32_t* __restrict__ keys,
                                          int* __restrict__ epoch, int blk) {
    const int i = blk * blockDim.x + threadIdx.x;
    if (i == 0) *epoch += 1;
    if (i >= n) return;
    const float4 pr = c.posr[i];
    const int3 b = find_bin(pr.x, pr.y, pr.z, g.len);
    if (!inside(b.x, b.y, b.z, g.N)) {
        c.sign[i] = 0;
        keys[i] = 0u;
        return;
    }
    keys[i] = morton3(b.x, b.y, b.z) + 1u;
    c.mesh[i] = b.x + b.y * g.N + b.z * g.N * g.N;
}

__device__ __forceinline__ void gather_body(const CellsSoA& s, const CellsSoA& d, const uint32_t* __restrict__ keys,
                                            const uint32_t* __restrict__ perm, int n, int4* __restrict__ bins,
                                            const int* __restrict__ epoch_p, int blk) {
    const int i = blk * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int epoch = *epoch_p;
    const int j = (int)perm[i];
    d.sign[i] = s.sign[j];
    const int m = s.mesh[j];
    d.mesh[i] = m;
    d.posr[i] = s.posr[j];
    d.force[i] = s.force[j];
    d.oldf[i] = s.oldf[j];
    d.V[i] = s.V[j];
    d.Vf[i] = s.Vf[j];
    d.Vcs[i] = s.Vcs[j];
    d.Vns[i] = s.Vns[j];
    d.clock[i] = s.clock[j];
    d.phase[i] = s.phase[j];
    const uint32_t k = keys[i];
    if (k == 0u) return;  // outside the grid: in no bin
    // a run of equal keys is one bin; its head writes the start and epoch, its tail the end
    if (i == 0 || keys[i - 1] != k) {
        bins[m].x = i;
        bins[m].z = epoch;
    }
    if (i == n - 1 || keys[i + 1] != k) bins[m].y = i;
}

struct MechArgs {
    CellsSoA cur, alt;
    const int4* bins;
    const int* epoch;
    int n;
    Geom g;
    float max_dist, cccr, ccca;
    double ra_ratio;
    float half_dt;
};

// forcekernel + movementkernel.  Per candidate j, in the order xi, yi, zi (bins), then ascending
// sorted index, with the cutoff `thres` carried from the previous accepted candidate:
//   d = sqrt(float(double(fma(dz,dz, fma(dx,dx, dy*dy))) + 0.0001)); skip if d >= thres;
//   R = max(r_j + r_i, 0.01); thres = float(double(R) * Ra_ratio); skip if d >= thres;
//   coefr = Cccr*((1-d/R)^2/d) if d <= R; coefa = Ccca*((1-d/thres)^2/d);
//   f = fma(p_i - p_j, coefr - coefa, f)
// then pos += dt/2 * (3f - f_old) as fma(dt/2, fma(3, f, -f_old), pos).
__device__ __forceinline__ void force_move_body(const MechArgs& a, int blk) {
    const int i = blk * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const uint8_t sg = a.cur.sign[i];
    const float4 pr = a.cur.posr[i];
    const float4 of = a.cur.oldf[i];
    if (!sg) {
        a.alt.sign[i] = 0;
        a.alt.posr[i] = pr;
        a.alt.oldf[i] = of;
        a.alt.force[i] = a.cur.force[i];
        a.alt.mesh[i] = a.cur.mesh[i];
        return;
    }
    const int N = a.g.N;
    const long long NN = (long long)N * N;
    const int epoch = *a.epoch;
    const int3 b = find_bin(pr.x, pr.y, pr.z, a.g.len);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    float thres = a.max_dist;
    // d >= thres is certain when |dp|^2 alone exceeds thres^2 (1 + 2^-20), a relative margin far
    // above the roundings between |dp|^2 + 0.0001 and d: such candidates skip the double-precision
    // add and the square root.  The float threshold is that bound rounded up.
    float thr_hi = __double2float_ru((double)thres * (double)thres * (1.0 + 0x1p-20));
    // the 27 bins in the reference's order: xi outer, then yi, then zi
#pragma unroll 1
    for (int o = 0; o < 27; ++o) {
        const int xi = b.x - 1 + o / 9, yi = b.y - 1 + (o / 3) % 3, zi = b.z - 1 + o % 3;
        if (!inside(xi, yi, zi, N)) continue;
        const int4 e = a.bins[xi + (long long)yi * N + zi * NN];
        if (e.z != epoch) continue;
#pragma unroll 1
        for (int j = e.x; j <= e.y; ++j) {
            if (!a.cur.sign[j]) continue;
            const float4 q = a.cur.posr[j];
            const float dx = __fsub_rn(pr.x, q.x);
            const float dy = __fsub_rn(pr.y, q.y);
            const float dz = __fsub_rn(pr.z, q.z);
            const float ss = __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
            if (ss > thr_hi) continue;
            const float d = __fsqrt_rn(__double2float_rn(__dadd_rn((double)ss, 0.0001)));
            if (d >= thres) continue;
            const float rs = __fadd_rn(q.w, pr.w);
            const float R = rs > 0.01f ? rs : 0.01f;
            thres = __double2float_rn(__dmul_rn((double)R, a.ra_ratio));
            thr_hi = __double2float_ru((double)thres * (double)thres * (1.0 + 0x1p-20));
            if (d >= thres) continue;
            float cr = 0.f, ca = 0.f;
            if (d <= R) {
                const float t = __fsub_rn(1.f, __fdiv_rn(d, R));
                cr = __fmul_rn(a.cccr, __fdiv_rn(__fmul_rn(t, t), d));
            }
            if (d <= thres) {
                const float t = __fsub_rn(1.f, __fdiv_rn(d, thres));
                ca = __fmul_rn(a.ccca, __fdiv_rn(__fmul_rn(t, t), d));
            }
            const float cf = __fsub_rn(cr, ca);
            fx = __fmaf_rn(dx, cf, fx);
            fy = __fmaf_rn(dy, cf, fy);
            fz = __fmaf_rn(dz, cf, fz);
        }
    }
    const float h = a.half_dt;
    const float nx = __fmaf_rn(h, __fmaf_rn(3.f, fx, -of.x), pr.x);
    const float ny = __fmaf_rn(h, __fmaf_rn(3.f, fy, -of.y), pr.y);
    const float nz = __fmaf_rn(h, __fmaf_rn(3.f, fz, -of.z), pr.z);
    const int3 nb = find_bin(nx, ny, nz, a.g.len);
    if (!inside(nb.x, nb.y, nb.z, N)) {
        // leaves the grid: only the sign changes (the reference returns before writing)
        a.alt.sign[i] = 0;
        a.alt.posr[i] = pr;
        a.alt.oldf[i] = of;
        a.alt.force[i] = make_float4(fx, fy, fz, 0.f);
        a.alt.mesh[i] = a.cur.mesh[i];
        return;
    }
    a.alt.sign[i] = 1;
    a.alt.posr[i] = make_float4(nx, ny, nz, pr.w);
    a.alt.oldf[i] = make_float4(fx, fy, fz, 0.f);
    a.alt.force[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    a.alt.mesh[i] = nb.x + nb.y * N + nb.z * N * N;
}

// ------------------------------------------------------------------ radix sort (sort.cu)

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ void hist_body(const uint32_t* __restrict__ keys, int n, int shift, int R,
                                          uint32_t* __restrict__ hist, int nb, int blk) {
    __shared__ uint32_t h[256];
    for (int d = threadIdx.x; d < R; d += kSortThreads) h[d] = 0;
    __syncthreads();
    const long long base = (long long)blk * kSortTile;
    const uint32_t mask = (uint32_t)R - 1u;
#pragma unroll 4
    for (int k = 0; k < kSortItems; ++k) {
        long long i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kSortThreads) hist[(long long)d * nb + blk] = h[d];
}

// Exclusive scan of one digit's per-tile counts (row d of the digit-major table), in place, by
// CTA d (`blk`); the digit's total goes to totals[d].  The scatter adds the prefix of the totals.
__device__ __forceinline__ void digit_scan_body(uint32_t* __restrict__ hist, int nb, uint32_t* __restrict__ totals,
                                                int blk) {
    __shared__ uint32_t ws[kSortThreads / 32];
    uint32_t* row = hist + (long long)blk * nb;
    const int per = (nb + kSortThreads - 1) / kSortThreads;
    const int lo = threadIdx.x * per, hi = lo + per < nb ? lo + per : nb;
    uint32_t s = 0;
    for (int i = lo; i < hi; ++i) s += row[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t wpre = 0;
    for (int j = 0; j < w; ++j) wpre += ws[j];
    uint32_t run = wpre + x - s;
    for (int i = lo; i < hi; ++i) {
        const uint32_t v = row[i];
        row[i] = run;
        run += v;
    }
    if (threadIdx.x == kSortThreads - 1) totals[blk] = run;
}

__device__ __forceinline__ void scatter_body(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                             uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int n, int shift,
                                             int R, const uint32_t* __restrict__ offs, int nb,
                                             const uint32_t* __restrict__ totals, int iota, int blk) {
    __shared__ uint32_t wcnt[kSortThreads / 32][256];
    __shared__ uint32_t gbase[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kSortThreads / 32) * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    if (w == 0) {
        // exclusive prefix of the digit totals: lane l sums digits 8l .. 8l+7 (R <= 256)
        uint32_t t[8], s = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int d = 8 * lane + k;
            t[k] = d < R ? totals[d] : 0u;
            s += t[k];
        }
        uint32_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        uint32_t run = x - s;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int d = 8 * lane + k;
            if (d < R) gbase[d] = run;
            run += t[k];
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kSortThreads) gbase[d] += offs[(long long)d * nb + blk];
    __syncthreads();
    const uint32_t mask = (uint32_t)R - 1u;
    const long long base = (long long)blk * kSortTile + w * (kSortTile / (kSortThreads / 32));
    uint32_t key[kSortItems], loc[kSortItems];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const long long i = base + k * 32 + lane;
        const bool valid = i < n;
        key[k] = valid ? kin[i] : 0u;
        const uint32_t dig = (key[k] >> shift) & mask;
        const unsigned peers = __match_any_sync(FULL, valid ? dig : 0xffffffffu);
        const uint32_t before = wcnt[w][dig & 255];
        loc[k] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0) wcnt[w][dig] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kSortThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < kSortThreads / 32; ++ww) {
            uint32_t c = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const long long i = base + k * 32 + lane;
        if (i < n) {
            const uint32_t dig = (key[k] >> shift) & mask;
            const uint32_t pos = gbase[dig] + wcnt[w][dig] + loc[k];
            kout[pos] = key[k];
            vout[pos] = iota ? (uint32_t)i : vin[i];
        }
    }
}

// ------------------------------------------------------------------ uptake map (lod.cu)

// Clear the lines flagged by the previous map (oxy_consumption_reset, include/LODkernel.cuh:183-190,
// restricted to the lines that can be nonzero).
// One warp per listed line: the row (P floats, P a multiple of 4) is cleared with 16-byte stores.
template <class A>
__device__ __forceinline__ void rate_reset_body(const A& a, int blk, int nblk) {
    const int P4 = a.g.P >> 2;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blk * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)nblk * blockDim.x) >> 5;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = 0; s < a.nsub; ++s) {
        const int cnt = *a.count[s];
        for (long long li = gw; li < cnt; li += nw) {
            const int line = a.list[s][li];
            float4* row = reinterpret_cast<float4*>(a.rate[s] + (long long)line * a.g.P);
            for (int x4 = lane; x4 < P4; x4 += 32) row[x4] = z;
            if (lane == 0) a.flag[s][line] = 0;
        }
    }
}

// oxy_consumption_update (include/LODkernel.cuh:12-22) with Cell::O2_consume (include/Cells.cuh:74-89)
// at O2 = 1: rate[mesh_idx] += coef * (V/len/len/len) (times the dead factor for phase >= 3).
template <class A>
__device__ __forceinline__ void rate_accum_body(const CellsSoA& c, int n, const A& a, int blk) {
    const int i = blk * blockDim.x + threadIdx.x;
    if (i >= n || !c.sign[i]) return;
    const int ph = c.phase[i];
    if (ph < 0) return;
    const int N = a.g.N;
    const int m = c.mesh[i];
    if (m < 0 || (long long)m >= (long long)N * N * N) return;
    const int x = m % N, line = m / N;
    const float len = a.g.len;
    const float vf = __fdiv_rn(__fdiv_rn(__fdiv_rn(c.V[i], len), len), len);
    for (int s = 0; s < a.nsub; ++s) {
        float r = __fmul_rn(a.coef[s], vf);
        if (ph >= 3) r = __fmul_rn(r, a.dead);
        atomicAdd(a.rate[s] + (long long)line * a.g.P + x, r);
        uint32_t* f = a.flag[s] + line;
        if (*(volatile uint32_t*)f == 0 && atomicExch(f, 1u) == 0u) a.list[s][atomicAdd(a.count[s], 1)] = line;
    }
}

}  // namespace gell
