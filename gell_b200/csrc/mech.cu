// mech.cu — one mechanics step (MechanicsMesh_struct::FM_update, include/FMkernel.cuh:181-202).
//
//   k_keys        Morton key + 1 per cell, 0 (and sign = false) for a cell outside the grid;
//                 mesh_idx of the cells inside (updateCellMeshIdx, :22-36)
//   radix_sort    stable sort of (key, index) (thrust::sort_by_key, :190), sort.cu
//   k_gather      every cell field moved to its sorted slot in the other buffer, and the cell
//                 list: the first and last sorted index of every occupied bin, stamped with the
//                 step's epoch (replaces Mech_Mesh_se_Reset/Get, :38-53, which rewrite 2*N^3 ints)
//   k_force_move  forcekernel (:56-118) and movementkernel (:130-158) fused: one thread per cell
//                 walks the 27 bins in the reference's order and applies the move; it reads the
//                 sorted buffer and writes the other one, so no cell sees a moved neighbour
#include "gell_internal.cuh"

namespace gell {

namespace {

// Also advances the cell-list epoch, which lives in device memory so that a captured step reads
// the current one when it is replayed.
__global__ void k_keys(CellsSoA c, int n, Geom g, uint32_t* __restrict__ keys, int* __restrict__ epoch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

__global__ void k_gather(CellsSoA s, CellsSoA d, const uint32_t* __restrict__ keys,
                         const uint32_t* __restrict__ perm, int n, int4* __restrict__ bins,
                         const int* __restrict__ epoch_p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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
__global__ void __launch_bounds__(256) k_force_move(MechArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

// Reference-shaped s/e arrays (first and last LIVE sorted index per bin, Max_Cell_num+1 / -1 when
// empty) rebuilt from the cell list, for the parity tests.
__global__ void k_fill_se(int* s, int* e, long long nvox, int smax) {
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    s[v] = smax;
    e[v] = -1;
}
__global__ void k_se(const uint8_t* sign, const int32_t* mesh, const uint32_t* keys, int n, int* s, int* e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || keys[i] == 0u || !sign[i]) return;
    atomicMin(&s[mesh[i]], i);
    atomicMax(&e[mesh[i]], i);
}

}  // namespace

static int key_bits(int N) {
    // largest key: Morton code of (N-1, N-1, N-1) plus one
    uint32_t m = 0;
    for (int b = 0; b < 10; ++b) {
        uint32_t bit = ((uint32_t)(N - 1) >> b) & 1u;
        m |= bit << (3 * b) | bit << (3 * b + 1) | bit << (3 * b + 2);
    }
    uint32_t k = m + 1u;
    int bits = 0;
    while (k) { ++bits; k >>= 1; }
    return bits;
}

gell_status fm_update(gell_ctx* c) {
    const int n = c->n;
    if (n > 0) {
        GELL_KERNEL(c, "k_keys", k_keys<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->cur(), n, c->g, c->sort.keys[0],
                                                                                c->dev_epoch));
        gell_status st = radix_sort(c, n, key_bits(c->g.N), true);
        if (st != GELL_OK) return st;
        const int w = c->sort.which;
        GELL_KERNEL(c, "k_gather", k_gather<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->cur(), c->alt(), c->sort.keys[w], c->sort.vals[w], n,
                                                              c->bins, c->dev_epoch));
        c->swap_all();
        MechArgs a;
        a.cur = c->cur();
        a.alt = c->alt();
        a.bins = c->bins;
        a.epoch = c->dev_epoch;
        a.n = n;
        a.g = c->g;
        a.max_dist = c->P.cc_max_dist;
        a.cccr = c->P.cccr;
        a.ccca = c->P.ccca;
        a.ra_ratio = c->P.ra_ratio;
        a.half_dt = c->P.mechanics_dt / 2.f;
        GELL_KERNEL(c, "k_force_move", k_force_move<<<blocks_for(n, 256), 256, 0, c->stream>>>(a));
        c->sign.swap();
        c->mesh.swap();
        c->posr.swap();
        c->force.swap();
        c->oldf.swap();
    }
    c->sorted_valid = true;
    c->rate_valid = false;
    return GELL_OK;
}

gell_status dump_se(gell_ctx* c, int* host_out) {
    int* d = nullptr;
    const long long nv = c->nvox;
    GELL_CUDA(c, cudaMallocAsync((void**)&d, (size_t)nv * 8, c->stream));
    GELL_KERNEL(c, "k_fill_se", k_fill_se<<<blocks_for(nv, 256), 256, 0, c->stream>>>(d, d + nv, nv, c->cap + 1));
    // the sorted order is the order before the last move: signs of that order are in the
    // alternate sign buffer (k_force_move wrote the current one)
    if (c->n > 0) {
        GELL_KERNEL(c, "k_se", k_se<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(c->sign.alt(), c->mesh.alt(), c->sort.keys[c->sort.which],
                                                            c->n, d, d + nv));
    }
    GELL_CUDA(c, cudaMemcpyAsync(host_out, d, (size_t)nv * 8, cudaMemcpyDeviceToHost, c->stream));
    GELL_CUDA(c, cudaFreeAsync(d, c->stream));
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    return GELL_OK;
}

}  // namespace gell
