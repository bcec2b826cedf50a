// lod.cu — LOD reaction-diffusion of the substrates (include/LODkernel.cuh:12-136,183-300).
//
// One substep of the reference (Mesh_struct::LODsolver) is Setboundary, meshupdatekernel and the
// three Thomas sweeps LODkernel_x/y/z, each a launch of one thread per line.  Here a substep is
// four launches, all substrates in each:
//   k_source_lines  boundary layers + implicit uptake source on the x-lines that hold cells
//   k_sweep<0>      boundary layers of the other lines + x sweep (x-lines are contiguous)
//   k_sweep<1>      y sweep (element stride P)      k_sweep<2>  z sweep (element stride P*N)
//
// Streaming line tiles.  A warp owns a tile of 32 lines (one per lane) and walks its lane's line
// out of shared memory.  The line is cut into B = ceil(N/32) groups of 32 elements; each group of
// the tile is one 32x32 TMA tensor box (4 KB) moved by one instruction and completing on the
// group's mbarrier, so the forward elimination starts as soon as group 0 has landed.  The back
// substitution finishes the groups from the top down; each finished group is written back by one
// TMA tensor store, and the slot it occupied is refilled with a group of the warp's NEXT tile.
// Groups live in B slots of 4 KB: a tile of parity 0 keeps group g in slot g, a tile of parity 1
// in slot B-1-g, so the slots freed first by the back substitution (top groups) are the ones the
// next tile needs first (bottom groups).  Each warp therefore always has its next tile in flight.
//   y/z boxes are [32 elements][32 lines] (128-byte rows, one row per element)
//   x boxes are [32 lines][32 elements] with the 128-byte swizzle, so each lane reads four
//       consecutive elements of its line with one conflict-free 16-byte load
//
// Arithmetic per line, the reference kernels' with nvcc's multiply-add fusion:
//   Y0 = b; Y_i = fma(-E_i, Y_{i-1}, p_i) (i = 1..N-2); x_{N-1} = b;
//   x_i = fma(-s, x_{i+1}, Y_i) / F_i (i = N-2..1); x_0 = b;  s = E[1]*F[0]
// and the source p /= fma(-rate, dt, 1).  The division on the back-substitution chain is
// Markstein's (IBM J. Res. Dev. 34(1), 1990): with y = RN(1/F_i) precomputed on the host, two
// residual corrections q += (a - F q) y give the correctly rounded quotient, equal to IEEE
// division (checked against it by gell_selftest_division and by the bit-exact parity tests).
#include <cuda.h>

#include <cstring>
#include <vector>

#include "async_copy.cuh"
#include "gell_internal.cuh"
#include "mech_body.cuh"

namespace gell {

namespace {

constexpr int kMaxSub = 8;
constexpr int kSlotFloats = 32 * 32;

struct SubDev {
    float* p;          // field (pitched)
    const float* rate;
    const uint32_t* line_flag;
    const float* EFR;  // E[N], F[N], RN(1/F)[N]
    const float4* FRS; // per element (F, RN(1/F), s, s*RN(1/F)), boundary elements as identities
    float b;
    float side;
    // groups whose E, F are the line's converged constants, and those constants pre-negated:
    // -E, -s, -s*RN(1/F), -F and RN(1/F)
    uint32_t uni;
    float nE, nS, nSR, nF, R;
};

struct LodArgs {
    CUtensorMap tm[kMaxSub];  // one map per substrate for this kernel's axis
    SubDev sub[kMaxSub];
    int nsub;
    Geom g;
    float dt;
    int* err;
    int exact;  // every group on the exact chain (GELL_OPT_EXACT_CHAIN)
};


__host__ __device__ inline int align128(int b) { return (b + 127) / 128 * 128; }

// Correctly rounded a / f given y = RN(1/f) (Markstein): q0 = a*y is within 2 ulp, one residual
// step makes it faithful, the second rounds it correctly.  Valid away from overflow/underflow.
__device__ __forceinline__ float div_rn(float a, float f, float y) {
    float q = __fmul_rn(a, y);
    float r = __fmaf_rn(-q, f, a);
    q = __fmaf_rn(r, y, q);
    r = __fmaf_rn(-q, f, a);
    return __fmaf_rn(r, y, q);
}

// One tile: 32 lines of one substrate, addressed by TMA coordinates.
struct TileDesc {
    int s;       // substrate
    int c0, c2;  // x: line0 (c0);  y: x0 (c0), z (c2);  z: L0 (c0)
    bool interior_lane, flagged_lane;  // x only
    long long line;                    // x: this lane's line (y + z*N)
};

// Substrate and TMA coordinates of tile t.
template <int AXIS>
__device__ __forceinline__ TileDesc tile_coords(const LodArgs& a, long long t, long long per_sub) {
    TileDesc d;
    d.s = (int)(t / per_sub);
    const long long tt = t - d.s * per_sub;
    d.c2 = 0;
    d.interior_lane = d.flagged_lane = false;
    d.line = 0;
    if (AXIS == 0) {
        d.c0 = (int)(tt * 32);
    } else if (AXIS == 1) {
        const int ntx = (a.g.P + 31) / 32;
        d.c2 = (int)(tt / ntx);
        d.c0 = (int)(tt - (long long)d.c2 * ntx) * 32;
    } else {
        d.c0 = (int)(tt * 32);
    }
    return d;
}

// ... and, for x, what this lane's line is (interior, holds uptake).
template <int AXIS>
__device__ __forceinline__ TileDesc tile_desc(const LodArgs& a, long long t, long long per_sub) {
    TileDesc d = tile_coords<AXIS>(a, t, per_sub);
    if (AXIS == 0) {
        const int N = a.g.N;
        const long long nl = (long long)N * N;
        d.line = (long long)d.c0 + (threadIdx.x & 31);
        const bool valid = d.line < nl;
        const int y = valid ? (int)(d.line % N) : 0, z = valid ? (int)(d.line / N) : 0;
        d.interior_lane = valid && y >= 2 && y < N - 2 && z >= 2 && z < N - 2;
        d.flagged_lane = valid && a.sub[d.s].line_flag[d.line] != 0u;
    }
    return d;
}

// TMA box of group g of tile d: load into `slot` (completing on `bar`) or store from it.
template <int AXIS>
__device__ __forceinline__ void box_load(const LodArgs& a, const TileDesc& d, int g, float* slot, uint64_t* bar) {
    mbar_arrive_expect(bar, kSlotFloats * 4);
    if (AXIS == 0) tma_load_2d(slot, &a.tm[d.s], 32 * g, d.c0, bar);
    else if (AXIS == 1) tma_load_3d(slot, &a.tm[d.s], d.c0, 32 * g, d.c2, bar);
    else tma_load_2d(slot, &a.tm[d.s], d.c0, 32 * g, bar);
}
// The same load with an L2 eviction-priority policy.
template <int AXIS>
__device__ __forceinline__ void box_load_hint(const LodArgs& a, const TileDesc& d, int g, float* slot, uint64_t* bar,
                                              uint64_t pol) {
    mbar_arrive_expect(bar, kSlotFloats * 4);
    if (AXIS == 0) tma_load_2d_hint(slot, &a.tm[d.s], 32 * g, d.c0, bar, pol);
    else if (AXIS == 1) tma_load_3d_hint(slot, &a.tm[d.s], d.c0, 32 * g, d.c2, bar, pol);
    else tma_load_2d_hint(slot, &a.tm[d.s], d.c0, 32 * g, bar, pol);
}
template <int AXIS>
__device__ __forceinline__ void box_store(const LodArgs& a, const TileDesc& d, int g, const float* slot) {
    if (AXIS == 0) tma_store_2d(&a.tm[d.s], 32 * g, d.c0, slot);
    else if (AXIS == 1) tma_store_3d(&a.tm[d.s], d.c0, 32 * g, d.c2, slot);
    else tma_store_2d(&a.tm[d.s], d.c0, 32 * g, slot);
}

// Per-element tables.  Boundary elements (j = 0 and j >= N-1) are identities: E = 0 makes
// Y_j = p_j (= b, set by the pre-pass), and (F, 1/F, s) = (1, 1, 0) makes x_j = Y_j = b, which is
// what the reference's x_0 = x_{N-1} = b gives (it never uses Y at N-1).  Every group therefore
// runs the same code.
struct SweepCtx {
    const float* E;    // E[j] (16-byte aligned)
    const float4* FR;  // (F[j], RN(1/F[j]), s[j], 0) (16-byte aligned)
    float b, dt;
};

// Address of element e (0..31) of this lane's line in a slot.  x slots are [line][element] with
// the 128-byte swizzle (16-byte chunk c of row r stored at chunk c ^ (r & 7)); y/z slots are
// [element][line].
template <int AXIS>
__device__ __forceinline__ float* elem(float* slot, int e, int lane) {
    if (AXIS == 0) return slot + lane * 32 + (((e >> 2) ^ (lane & 7)) << 2) + (e & 3);
    return slot + e * 32 + lane;
}

// 8 consecutive elements e0..e0+7 (e0 a multiple of 8) of this lane's line.
template <int AXIS>
__device__ __forceinline__ void load8(float* slot, int e0, int lane, float v[8]) {
    if (AXIS == 0) {
        const float4 a = *reinterpret_cast<const float4*>(elem<0>(slot, e0, lane));
        const float4 b = *reinterpret_cast<const float4*>(elem<0>(slot, e0 + 4, lane));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = slot[(e0 + k) * 32 + lane];
    }
}
template <int AXIS>
__device__ __forceinline__ void store8(float* slot, int e0, int lane, const float v[8]) {
    if (AXIS == 0) {
        *reinterpret_cast<float4*>(elem<0>(slot, e0, lane)) = make_float4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<float4*>(elem<0>(slot, e0 + 4, lane)) = make_float4(v[4], v[5], v[6], v[7]);
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) slot[(e0 + k) * 32 + lane] = v[k];
    }
}

// x: Setboundary on the values the forward elimination loads.  Element j of this lane's line is
// replaced by b when j < lo or j > hi: lo = 2, hi = N-3 for interior lines without uptake (the two
// outer layers of the y/z faces); lo = 1, hi = N-2 for lines with uptake, which k_source_lines has
// already prepared (only the reference's Y_0 = b and x_{N-1} = b remain); lo = INT_MAX for the
// boundary lines themselves, all of whose elements are b.  `rs` (warp-uniform) says whether any
// lane resets an element of this group.
struct XReset {
    int lo, hi;
    float b;
};

__device__ __forceinline__ void reset8(float v[8], int j0, const XReset& r) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = (j0 + k < r.lo || j0 + k > r.hi) ? r.b : v[k];
}

// Forward elimination over group g: Y_j = fma(-E_j, Y_{j-1}, p_j) for the 32 elements of the group,
// 8 at a time with the next batch's values and E already requested.
template <int AXIS, bool STORE = true>
__device__ __forceinline__ void forward_group(const SweepCtx& c, float* slot, int g, int lane, float& Y, bool rs,
                                              const XReset& xr) {
    const int j0 = 32 * g;
    float v[8], w[8];
    float4 e0 = *reinterpret_cast<const float4*>(c.E + j0);
    float4 e1 = *reinterpret_cast<const float4*>(c.E + j0 + 4);
    load8<AXIS>(slot, 0, lane, v);
#pragma unroll
    for (int b8 = 0; b8 < 4; ++b8) {
        float4 n0 = e0, n1 = e1;
        if (b8 < 3) {
            load8<AXIS>(slot, 8 * b8 + 8, lane, w);
            n0 = *reinterpret_cast<const float4*>(c.E + j0 + 8 * b8 + 8);
            n1 = *reinterpret_cast<const float4*>(c.E + j0 + 8 * b8 + 12);
        }
        if (AXIS == 0 && rs) reset8(v, j0 + 8 * b8, xr);
        const float ev[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            Y = __fmaf_rn(-ev[k], Y, v[k]);
            v[k] = Y;
        }
        if (STORE) store8<AXIS>(slot, 8 * b8, lane, v);
        if (b8 < 3) {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = w[k];
            e0 = n0;
            e1 = n1;
        }
    }
}

// Back substitution step with the exact division: x = (y - s x) / F.
__device__ __forceinline__ float back_exact(float x, float y, float f, float rf, float sd) {
    return div_rn(__fmaf_rn(-sd, x, y), f, rf);
}

// Back substitution over a full group (elements 32g+31 .. 32g, all in [1, N-2]), results in o[].
// The chain carries a1, the once-corrected quotient started from fma(-s/F, x, y/F); the exact
// quotient a2 is computed beside it.  If any lane's a1 differs from its a2 anywhere in the group,
// the whole group is recomputed on the exact chain, so o[] always holds the exact values.
template <int AXIS>
__device__ __forceinline__ void backward_full(const SweepCtx& c, float* slot, int j0, int lane, float& x,
                                              float o[32], int exact) {
    const float x_in = x;
    uint32_t bad = 0;
    float v[8], w[8];
    const float4* fb = c.FR + j0;
    float4 f[8], h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) f[k] = __ldg(fb + 24 + k);
    load8<AXIS>(slot, 24, lane, v);
#pragma unroll
    for (int b8 = 3; b8 >= 0; --b8) {
        if (b8 > 0) {
            load8<AXIS>(slot, 8 * b8 - 8, lane, w);
#pragma unroll
            for (int k = 0; k < 8; ++k) h[k] = __ldg(fb + 8 * b8 - 8 + k);
        }
        float yr[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) yr[k] = __fmul_rn(v[k], f[k].y);
#pragma unroll
        for (int k = 7; k >= 0; --k) {
            const float t = __fmaf_rn(-f[k].z, x, v[k]);
            const float a0 = __fmaf_rn(-f[k].w, x, yr[k]);
            const float r0 = __fmaf_rn(-a0, f[k].x, t);
            const float a1 = __fmaf_rn(r0, f[k].y, a0);   // carried on the chain
            const float r1 = __fmaf_rn(-a1, f[k].x, t);
            const float a2 = __fmaf_rn(r1, f[k].y, a1);   // exact quotient of t by F
            bad |= __float_as_uint(a1) ^ __float_as_uint(a2);
            x = a1;
            o[8 * b8 + k] = a1;
        }
        if (b8 > 0) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                v[k] = w[k];
                f[k] = h[k];
            }
        }
    }
    if (__any_sync(FULL, bad != 0) || exact) {
        x = x_in;
#pragma unroll
        for (int e = 31; e >= 0; --e) {
            const float4 fr = __ldg(c.FR + j0 + e);
            x = back_exact(x, *elem<AXIS>(slot, e, lane), fr.x, fr.y, fr.z);
            o[e] = x;
        }
    }
}

// The same two steps for a group whose E and F are the line's converged constants (all lanes'
// lines share them): the factors live in registers, and independent multiply-adds are issued in
// pairs (FFMA2), without changing any operation or its rounding.
template <int AXIS, bool STORE = true>
__device__ __forceinline__ void forward_uniform(float* slot, int g, int lane, float& Y, float nE, bool rs,
                                                const XReset& xr) {
    float v[8], w[8];
    load8<AXIS>(slot, 0, lane, v);
#pragma unroll
    for (int b8 = 0; b8 < 4; ++b8) {
        if (b8 < 3) load8<AXIS>(slot, 8 * b8 + 8, lane, w);
        if (AXIS == 0 && rs) reset8(v, 32 * g + 8 * b8, xr);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            Y = __fmaf_rn(nE, Y, v[k]);
            v[k] = Y;
        }
        if (STORE) store8<AXIS>(slot, 8 * b8, lane, v);
        if (b8 < 3) {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = w[k];
        }
    }
}

template <int AXIS>
__device__ __forceinline__ void backward_uniform(const SubDev& sd, float* slot, int lane, float& x, float o[32],
                                                 int exact) {
    const float x_in = x;
    const float R = sd.R, nF = sd.nF;
    const float2 nS2 = make_float2(sd.nS, sd.nSR), R2 = make_float2(R, R), nF2 = make_float2(nF, nF);
    uint32_t bad = 0;
    float v[8], w[8];
    load8<AXIS>(slot, 24, lane, v);
#pragma unroll
    for (int b8 = 3; b8 >= 0; --b8) {
        if (b8 > 0) load8<AXIS>(slot, 8 * b8 - 8, lane, w);
        float yr[8];
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
            const float2 q = __fmul2_rn(make_float2(v[k], v[k + 1]), R2);
            yr[k] = q.x;
            yr[k + 1] = q.y;
        }
        float t[8], a1[8];
#pragma unroll
        for (int k = 7; k >= 0; --k) {
            // (t, a0) = (fma(-s, x, y), fma(-s/F, x, y/F))
            const float2 ta = __ffma2_rn(nS2, make_float2(x, x), make_float2(v[k], yr[k]));
            const float r0 = __fmaf_rn(ta.y, nF, ta.x);
            x = __fmaf_rn(r0, R, ta.y);  // a1, carried on the chain
            t[k] = ta.x;
            a1[k] = x;
            o[8 * b8 + k] = x;
        }
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
            const float2 a = make_float2(a1[k], a1[k + 1]);
            const float2 r1 = __ffma2_rn(a, nF2, make_float2(t[k], t[k + 1]));
            const float2 a2 = __ffma2_rn(r1, R2, a);  // exact quotients
            bad |= (__float_as_uint(a.x) ^ __float_as_uint(a2.x)) | (__float_as_uint(a.y) ^ __float_as_uint(a2.y));
        }
        if (b8 > 0) {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = w[k];
        }
    }
    if (__any_sync(FULL, bad != 0) || exact) {
        x = x_in;
#pragma unroll
        for (int e = 31; e >= 0; --e) {
            x = div_rn(__fmaf_rn(sd.nS, x, *elem<AXIS>(slot, e, lane)), -nF, R);
            o[e] = x;
        }
    }
}

// Back substitution over group g, from its top element down; the results replace the group's
// values in its slot, from where one TMA store writes them back.
template <int AXIS>
__device__ __forceinline__ void backward_group(const SweepCtx& c, const SubDev& sd, float* slot, int g, int lane,
                                               float& x, int exact) {
    float o[32];
    if ((sd.uni >> g) & 1u) backward_uniform<AXIS>(sd, slot, lane, x, o, exact);
    else backward_full<AXIS>(c, slot, 32 * g, lane, x, o, exact);
#pragma unroll
    for (int b8 = 0; b8 < 4; ++b8) store8<AXIS>(slot, 8 * b8, lane, o + 8 * b8);
}

// y/z: rows of the end groups that hold boundary elements (j = 0 and j >= N-1) get b.
template <int AXIS>
__device__ __forceinline__ void edge_rows(const SweepCtx& c, float* slot, int g, int N, int lane) {
    const int j0 = 32 * g;
    if (g == 0) slot[lane] = c.b;
    for (int e = max(N - 1 - j0, 0); e < 32; ++e) slot[e * 32 + lane] = c.b;
    __syncwarp();
}

// Warp roles.  Each compute warp owns B slots of 4 KB and walks its tiles: the forward
// elimination waits for each group's box on full[g]; the back substitution leaves each group's
// results in its slot and signals empty[g].  One producer thread issues every TMA copy: the first
// tile of each compute warp, then for every signalled group the store of its results and, once that
// store has read the slot, the load of the warp's next tile's group that takes the slot over.  Both
// barriers complete once per tile, so tile k of a warp waits on parity k & 1.
//
// Slots: a tile of parity 0 keeps group g in slot g, a tile of parity 1 in slot B-1-g.  The back
// substitution frees slots from the top group down, which is where the next tile's bottom groups
// (the ones its forward elimination needs first) go: group B-1-g of tile k+1 reuses the slot of
// group g of tile k.
__host__ __device__ __forceinline__ int slot_index(int g, int q, int B) { return q ? B - 1 - g : g; }

template <int AXIS, int Q>
__device__ __forceinline__ bool run_tile(const LodArgs& a, const TileDesc& d, float* buf, uint64_t* full,
                                         uint64_t* empty, const float* sEFR, int Na) {
    const int N = a.g.N;
    const int B = (N + 31) >> 5;
    const int lane = threadIdx.x & 31;
    const SubDev& sd = a.sub[d.s];
    SweepCtx c;
    c.E = sEFR + (size_t)d.s * Na;
    c.FR = sd.FRS;
    c.b = sd.b;
    c.dt = a.dt;
    uint32_t special = 0;
    XReset xr{0, 0, c.b};
    if (AXIS == 0) {
        const bool sp = !d.flagged_lane && !d.interior_lane;
        xr.lo = d.flagged_lane ? 1 : (d.interior_lane ? 2 : 0x7fffffff);
        xr.hi = d.flagged_lane ? N - 2 : N - 3;
        special = __ballot_sync(FULL, sp);  // boundary lines: every group needs the reset
    }

    float Y = c.b;
    for (int g = 0; g < B; ++g) {
        if (!mbar_wait(full + g, (uint32_t)Q, a.err, 1 + AXIS)) return false;
        float* slot = buf + (size_t)slot_index(g, Q, B) * kSlotFloats;
        const bool edge = g == 0 || 32 * g + 31 > N - 3;
        const bool rs = AXIS == 0 && (edge || special != 0);
        if (AXIS != 0 && edge) edge_rows<AXIS>(c, slot, g, N, lane);
        if ((sd.uni >> g) & 1u) forward_uniform<AXIS>(slot, g, lane, Y, sd.nE, rs, xr);
        else forward_group<AXIS>(c, slot, g, lane, Y, rs, xr);
    }
    float x = c.b;
    for (int g = B - 1; g >= 0; --g) {
        float* slot = buf + (size_t)slot_index(g, Q, B) * kSlotFloats;
        backward_group<AXIS>(c, sd, slot, g, lane, x, a.exact);
        // the slot now holds the results: make them visible to the TMA store, then hand it over
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + g);
    }
    return true;
}

// The producer of compute warp w (lane 0 of warp W + w) follows the same tiles: first tile's loads,
// then per signalled group the store of its results and the refill of the slot of the group before
// it (whose store has read the slot by then), as the compute warp frees them.
template <int AXIS>
__device__ void producer(const LodArgs& a, float* buf, uint64_t* full, uint64_t* empty, long long t, long long total,
                         long long step, long long per_sub) {
    const int B = (a.g.N + 31) >> 5;
    TileDesc d = tile_coords<AXIS>(a, t, per_sub);
    for (int g = 0; g < B; ++g) box_load<AXIS>(a, d, g, buf + (size_t)g * kSlotFloats, full + g);
    for (int k = 0;; ++k) {
        const int Q = k & 1;
        const long long tn = t + step;
        const bool has_next = tn < total;
        const TileDesc dn = has_next ? tile_coords<AXIS>(a, tn, per_sub) : d;
        for (int g = B - 1; g >= 0; --g) {
            if (!mbar_wait1(empty + g, (uint32_t)Q, a.err, 8 + AXIS)) {
                asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                return;
            }
            float* slot = buf + (size_t)slot_index(g, Q, B) * kSlotFloats;
            box_store<AXIS>(a, d, g, slot);
            bulk_commit();
            if (has_next && g + 1 <= B - 1) {
                // the store of group g+1 has read its slot: refill it with the next tile
                bulk_wait_read<1>();
                box_load<AXIS>(a, dn, B - 2 - g, buf + (size_t)slot_index(g + 1, Q, B) * kSlotFloats,
                               full + (B - 2 - g));
            }
        }
        if (!has_next) break;
        bulk_wait_read<0>();
        box_load<AXIS>(a, dn, B - 1, buf + (size_t)slot_index(0, Q, B) * kSlotFloats, full + (B - 1));
        t = tn;
        d = dn;
    }
    // no bulk store may outlive the CTA's shared memory
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// blockDim = 2W warps: W <= kMaxComputeWarps compute warps, then their W producer warps.
constexpr int kMaxComputeWarps = 4;
template <int AXIS>
__global__ void __launch_bounds__(64 * kMaxComputeWarps, 1) k_sweep(const __grid_constant__ LodArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const Geom g = a.g;
    const int N = g.N, P = g.P;
    const int Na = (N + 31) & ~31;  // per substrate: E[Na] in shared memory
    const int B = (N + 31) >> 5;
    const int W = blockDim.x >> 6, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // 1024-byte aligned slots first (the x boxes use the 128-byte swizzle), then tables, barriers
    const uint32_t base = smem_u32(sm);
    unsigned char* sm1 = sm + ((1024 - (base & 1023)) & 1023);
    float* slots = reinterpret_cast<float*>(sm1);
    float* sEFR = reinterpret_cast<float*>(sm1 + (size_t)W * B * kSlotFloats * 4);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm1 + (size_t)W * B * kSlotFloats * 4 + align128(a.nsub * Na * 4));
    uint64_t* empty = full + W * 32;
    for (int i = threadIdx.x; i < a.nsub * Na; i += blockDim.x) {
        const int s = i / Na, j = i - s * Na;
        // E of the elements the reference's recurrences update; 0 elsewhere (identity)
        sEFR[i] = (j >= 1 && j <= N - 2) ? a.sub[s].EFR[j] : 0.f;
    }
    for (int i = threadIdx.x; i < W * 32; i += blockDim.x) {
        mbar_init(full + i, 1u);
        mbar_init(empty + i, 1u);
    }
    fence_mbar_init();
    __syncthreads();

    long long per_sub;
    if (AXIS == 0) per_sub = ((long long)N * N + 31) / 32;
    else if (AXIS == 1) per_sub = (long long)((P + 31) / 32) * N;
    else per_sub = (g.PN + 31) / 32;
    const long long total = per_sub * a.nsub;
    const long long step = (long long)gridDim.x * W;

    if (warp >= W) {
        const int w = warp - W;
        const long long t = (long long)blockIdx.x * W + w;
        if (lane == 0 && t < total)
            producer<AXIS>(a, slots + (size_t)w * B * kSlotFloats, full + w * 32, empty + w * 32, t, total, step, per_sub);
        return;
    }
    float* buf = slots + (size_t)warp * B * kSlotFloats;
    uint64_t* fb = full + warp * 32;
    uint64_t* eb = empty + warp * 32;
    int k = 0;
    long long t = (long long)blockIdx.x * W + warp;
    if (t >= total) return;
    // the next tile's description (for x: each lane's uptake flag, a global load) is requested one
    // tile ahead, so its latency is not paid in front of the forward elimination
    TileDesc d = tile_desc<AXIS>(a, t, per_sub);
    for (; t < total; t += step, ++k) {
        const TileDesc dn = t + step < total ? tile_desc<AXIS>(a, t + step, per_sub) : d;
        const bool ok = (k & 1) ? run_tile<AXIS, 1>(a, d, buf, fb, eb, sEFR, Na)
                                : run_tile<AXIS, 0>(a, d, buf, fb, eb, sEFR, Na);
        if (!ok) break;
        d = dn;
    }
}

// ------------------------------------------------------------------ ring sweeps
//
// The kernel above keeps a whole 32-line tile in shared memory from its forward elimination to its
// back substitution, so shared memory bounds the lines in flight (4 compute warps per SM at
// N = 400, 2 at N = 600) and the dependent recurrences of those few warps leave the SM idle most
// of the time.  This variant needs only R group slots of 4 KB per warp, R < B, so 8 compute warps
// fit at both sizes:
//   * forward elimination streams the B groups of the tile through the ring; for the groups
//     [0, B-R) it keeps only the running value Y entering the group (a checkpoint, 4 B per lane
//     and group in shared memory) and frees the slot at once;
//   * the top R groups stay resident with their Y values, as in the kernel above;
//   * back substitution takes the groups from the top down; a group below B-R is loaded again
//     (the second read of the tile hits L2: the tile was read a few tens of microseconds before)
//     and its Y values are recomputed from the checkpoint with the same operations, so they are
//     bit-identical to the first pass; results go back to the field by TMA stores.
// Each compute warp issues its own copies (lane 0), always into a slot whose previous occupant it
// has finished with.  A TMA store's read of its slot can take thousands of cycles to complete, so a
// stored slot is refilled only L groups later (the warp waits for the store L groups back, never
// the last one): forward loads run R groups ahead of their use, back-substitution loads R-L.
// Group g of a tile of parity q lives in slot  g mod R  (q = 0) or  R-1 - (g mod R)  (q = 1),
// which makes the slots the back substitution frees last the ones the next tile's first groups
// take.
constexpr int kRingWarps = 8;
constexpr int kRingMaxSlots = 8;

__device__ __forceinline__ int ring_slot(int g, int q, int R) {
    const int m = g % R;
    return q ? R - 1 - m : m;
}

// Bounded clean-up after a failed wait: wait (briefly) for every load still in flight into this
// warp's slots and for its stores, so no copy outlives the CTA's shared memory.
__device__ __forceinline__ void ring_drain(uint64_t* full, uint32_t pend, uint32_t phase, int R, int* err, int lane) {
    for (int s = 0; s < R; ++s)
        if ((pend >> s) & 1u) mbar_wait(full + s, (phase >> s) & 1u, err, 20, 1 << 16);
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
}

template <int AXIS, bool HINT>
__device__ __forceinline__ bool ring_tile(const LodArgs& a, const TileDesc& d, const TileDesc& dn, bool has_next,
                                          int q, int R, int L, float* buf, uint64_t* full, float* ck,
                                          const float* sE, int Na, uint32_t& phase, uint32_t& pend) {
    const int N = a.g.N;
    const int B = (N + 31) >> 5;
    const int keep = B - R;  // groups [keep, B) stay resident between the two passes
    const int lane = threadIdx.x & 31;
    const SubDev& sd = a.sub[d.s];
    SweepCtx c;
    c.E = sE + (size_t)d.s * Na;
    c.FR = sd.FRS;
    c.b = sd.b;
    c.dt = a.dt;
    uint32_t special = 0;
    XReset xr{0, 0, c.b};
    if (AXIS == 0) {
        const bool sp = !d.flagged_lane && !d.interior_lane;
        xr.lo = d.flagged_lane ? 1 : (d.interior_lane ? 2 : 0x7fffffff);
        xr.hi = d.flagged_lane ? N - 2 : N - 3;
        special = __ballot_sync(FULL, sp);
    }
    auto wait_slot = [&](int s) -> bool {
        if (!mbar_wait(full + s, (phase >> s) & 1u, a.err, 1 + AXIS)) return false;
        phase ^= 1u << s;
        pend &= ~(1u << s);
        return true;
    };
    // with HINT, a group that will be read a second time is loaded with priority to stay in L2 and
    // every other load (a last read) with priority to leave it first
    auto load = [&](const TileDesc& t, int g, int s, bool again) {
        if (lane == 0) {
            if (HINT) box_load_hint<AXIS>(a, t, g, buf + (size_t)s * kSlotFloats, full + s,
                                          again ? l2_evict_last() : l2_evict_first());
            else box_load<AXIS>(a, t, g, buf + (size_t)s * kSlotFloats, full + s);
        }
        pend |= 1u << s;
    };
    // one group's forward elimination from the running value Y, storing Y into the slot or not
    auto forward = [&](float* slot, int g, float& Y, bool store) {
        const bool edge = g == 0 || 32 * g + 31 > N - 3;
        const bool rs = AXIS == 0 && (edge || special != 0);
        if (AXIS != 0 && edge) edge_rows<AXIS>(c, slot, g, N, lane);
        const bool uni = (sd.uni >> g) & 1u;
        if (store) {
            if (uni) forward_uniform<AXIS, true>(slot, g, lane, Y, sd.nE, rs, xr);
            else forward_group<AXIS, true>(c, slot, g, lane, Y, rs, xr);
        } else {
            if (uni) forward_uniform<AXIS, false>(slot, g, lane, Y, sd.nE, rs, xr);
            else forward_group<AXIS, false>(c, slot, g, lane, Y, rs, xr);
        }
    };

    float Y = c.b;
    for (int g = 0; g < B; ++g) {
        const int s = ring_slot(g, q, R);
        if (!wait_slot(s)) return false;
        float* slot = buf + (size_t)s * kSlotFloats;
        if (g < keep) {
            ck[g * 32 + lane] = Y;
            forward(slot, g, Y, false);
            fence_proxy_async();  // the edge rows may have written the slot
            __syncwarp();
            load(d, g + R, s, g + R < keep);  // same slot: (g + R) mod R == g mod R
        } else {
            forward(slot, g, Y, true);
        }
    }
    float x = c.b;
    for (int h = B - 1; h >= 0; --h) {
        const int s = ring_slot(h, q, R);
        float* slot = buf + (size_t)s * kSlotFloats;
        if (h < keep) {
            if (!wait_slot(s)) return false;
            float Yh = ck[h * 32 + lane];
            forward(slot, h, Yh, true);  // the same Y values as the first pass
        }
        backward_group<AXIS>(c, sd, slot, h, lane, x, a.exact);
        // results in the slot: visible to the TMA store, then stored
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            box_store<AXIS>(a, d, h, slot);
            bulk_commit();
        }
        // the slot of group h+L, stored L groups ago, is refilled once that store has read it: the L
        // stores issued since may still be reading theirs
        const int hl = h + L;
        if (hl <= B - 1) {
            if (hl >= R) {
                if (lane == 0) bulk_wait_read_n(L);
                load(d, hl - R, ring_slot(hl, q, R), false);  // back substitution's second read of group h+L-R
            } else if (has_next) {
                if (lane == 0) bulk_wait_read_n(L);
                load(dn, R - 1 - hl, ring_slot(hl, q, R), R - 1 - hl < keep);  // next tile, group R-1-(h+L)
            }
        }
        if (h == 0 && has_next) {
            // the slots of groups L-1 .. 0 take the next tile's groups R-L .. R-1
            if (lane == 0) bulk_wait_read_n(0);
            for (int j = (L < B ? L : B) - 1; j >= 0; --j)
                if (R - 1 - j >= 0) load(dn, R - 1 - j, ring_slot(j, q, R), R - 1 - j < keep);
        }
        __syncwarp();
    }
    return true;
}

template <int AXIS, bool HINT>
__global__ void __launch_bounds__(32 * kRingWarps, 1) k_sweep_ring(const __grid_constant__ LodArgs a, int R, int L) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const Geom g = a.g;
    const int N = g.N, P = g.P;
    const int Na = (N + 31) & ~31;
    const int B = (N + 31) >> 5;
    const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = smem_u32(sm);
    unsigned char* sm1 = sm + ((1024 - (base & 1023)) & 1023);
    float* slots = reinterpret_cast<float*>(sm1);
    size_t off = (size_t)W * R * kSlotFloats * 4;
    float* sE = reinterpret_cast<float*>(sm1 + off);
    off += align128(a.nsub * Na * 4);
    float* cks = reinterpret_cast<float*>(sm1 + off);
    off += align128(W * B * 32 * 4);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm1 + off);
    for (int i = threadIdx.x; i < a.nsub * Na; i += blockDim.x) {
        const int s = i / Na, j = i - s * Na;
        sE[i] = (j >= 1 && j <= N - 2) ? a.sub[s].EFR[j] : 0.f;
    }
    for (int i = threadIdx.x; i < W * R; i += blockDim.x) mbar_init(full + i, 1u);
    fence_mbar_init();
    __syncthreads();

    long long per_sub;
    if (AXIS == 0) per_sub = ((long long)N * N + 31) / 32;
    else if (AXIS == 1) per_sub = (long long)((P + 31) / 32) * N;
    else per_sub = (g.PN + 31) / 32;
    const long long total = per_sub * a.nsub;
    const long long step = (long long)gridDim.x * W;

    long long t = (long long)blockIdx.x * W + warp;
    if (t >= total) return;
    float* buf = slots + (size_t)warp * R * kSlotFloats;
    uint64_t* fb = full + warp * R;
    float* ck = cks + (size_t)warp * B * 32;
    uint32_t phase = 0, pend = 0;
    TileDesc d = tile_desc<AXIS>(a, t, per_sub);
    // the first tile's first R groups
    for (int gg = 0; gg < R; ++gg) {
        if (lane == 0) {
            float* sl = buf + (size_t)ring_slot(gg, 0, R) * kSlotFloats;
            if (HINT) box_load_hint<AXIS>(a, d, gg, sl, fb + ring_slot(gg, 0, R),
                                          gg < B - R ? l2_evict_last() : l2_evict_first());
            else box_load<AXIS>(a, d, gg, sl, fb + ring_slot(gg, 0, R));
        }
        pend |= 1u << ring_slot(gg, 0, R);
    }
    for (int k = 0;; ++k) {
        const long long tn = t + step;
        const bool has_next = tn < total;
        const TileDesc dn = has_next ? tile_desc<AXIS>(a, tn, per_sub) : d;
        if (!ring_tile<AXIS, HINT>(a, d, dn, has_next, k & 1, R, L, buf, fb, ck, sE, Na, phase, pend)) {
            ring_drain(fb, pend, phase, R, a.err, lane);
            return;
        }
        if (!has_next) break;
        t = tn;
        d = dn;
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------------------ batched sweeps (ensembles)
//
// One launch per axis sweeps the lines of MANY grids: every (member, substrate) pair of an
// ensemble is an item with its own geometry, tensor maps and Thomas tables, and the items' line
// tiles form one list that the persistent CTAs walk (warp w of CTA b takes tiles b*W + w + k*step).
// Each warp takes a contiguous range of the list holding an equal share of the work (a tile of B
// groups costs B + 1), so it stays on one item for many tiles.  The line-tile pipeline is the one
// above (a producer lane per compute warp, whole tiles in shared memory), with two changes for tiles
// of different lengths (B groups, up to kBatchMaxGroups):
//   * slots are assigned through a per-warp permutation: the next tile's group j takes the slot the
//     back substitution freed (B-1-j)-th, and groups beyond B take the slots this tile left unused;
//   * full and empty barriers belong to slots (a phase bit per slot), not to groups.
// E of the warp's current item is staged in a per-warp shared buffer when the item changes.
constexpr int kBatchMaxGroups = 8;  // lines up to 256 voxels
constexpr int kBatchWarps = 4;

struct alignas(64) BatchItem {
    CUtensorMap tm[3];
    SubDev sd;
    Geom g;
    long long tile0[3];  // first tile of this item in each axis' list
    long long cost0[3];  // work of the items before it (a tile costs B + 1)
    int B, exact;
};
struct SrcItem {
    float* p;
    const float* rate;
    const int* list;
    const int* count;
    float b, dt;
    int N, P;
};
struct BatchArgs {
    const BatchItem* items;
    int nitems;
    long long total[3];
    long long cost[3];  // total work per axis
    int* err;
};

// First tile whose work starts at or after `x`: the warps split the tiles into contiguous ranges
// of equal work (tiles of long lines cost more), so a warp stays on one item for many tiles.
template <int AXIS>
__device__ __forceinline__ long long tile_at_cost(const BatchArgs& a, long long x) {
    if (x >= a.cost[AXIS]) return a.total[AXIS];
    int i = 0;
    while (i + 1 < a.nitems && a.items[i + 1].cost0[AXIS] <= x) ++i;
    const BatchItem& it = a.items[i];
    const long long c = it.B + 1;
    long long j = it.tile0[AXIS] + (x - it.cost0[AXIS] + c - 1) / c;
    const long long end = i + 1 < a.nitems ? a.items[i + 1].tile0[AXIS] : a.total[AXIS];
    return j < end ? j : end;
}

__device__ __forceinline__ uint32_t perm_get(uint32_t perm, int g) { return (perm >> (4 * g)) & 15u; }
// Slots of the next tile (Bn groups) after a tile of B groups: first the slots this tile leaves
// unused (ascending; the producer fills them as soon as the tile starts, so a short tile's successor
// is loaded a whole tile ahead), then the slots this tile frees, in the order its back substitution
// frees them (top group first).
__device__ __forceinline__ uint32_t batch_perm_next(uint32_t perm, int B, int Bn, int Bmax) {
    uint32_t used = 0;
    for (int g = 0; g < B; ++g) used |= 1u << perm_get(perm, g);
    uint32_t out = 0;
    int j = 0;
    for (int sl = 0; sl < Bmax && j < Bn; ++sl)
        if (!((used >> sl) & 1u)) out |= (uint32_t)sl << (4 * j++);
    for (int g = B - 1; g >= 0 && j < Bn; --g) out |= perm_get(perm, g) << (4 * j++);
    return out;
}
__device__ __forceinline__ uint32_t perm_identity() {
    uint32_t p = 0;
    for (int j = 0; j < 8; ++j) p |= (uint32_t)j << (4 * j);
    return p;
}

struct BTile {
    int item;
    int c0, c2;
    bool interior_lane, flagged_lane;
};

// Item and TMA coordinates of tile t; `item` is a cursor that only moves forward (tiles of a warp
// increase), so the search is a short scan.
template <int AXIS>
__device__ __forceinline__ BTile btile(const BatchArgs& a, long long t, int& item) {
    while (item + 1 < a.nitems && t >= a.items[item + 1].tile0[AXIS]) ++item;
    const BatchItem& it = a.items[item];
    const int N = it.g.N, P = it.g.P;
    const long long tt = t - it.tile0[AXIS];
    BTile d;
    d.item = item;
    d.c2 = 0;
    d.interior_lane = d.flagged_lane = false;
    if (AXIS == 0) {
        d.c0 = (int)(tt * 32);
        const long long line = (long long)d.c0 + (threadIdx.x & 31);
        const bool valid = line < (long long)N * N;
        const int y = valid ? (int)(line % N) : 0, z = valid ? (int)(line / N) : 0;
        d.interior_lane = valid && y >= 2 && y < N - 2 && z >= 2 && z < N - 2;
        d.flagged_lane = valid && it.sd.line_flag[line] != 0u;
    } else if (AXIS == 1) {
        const int ntx = (P + 31) / 32;
        d.c2 = (int)(tt / ntx);
        d.c0 = (int)(tt - (long long)d.c2 * ntx) * 32;
    } else {
        d.c0 = (int)(tt * 32);
    }
    return d;
}

template <int AXIS>
__device__ __forceinline__ void bbox_load(const BatchItem& it, const BTile& d, int g, float* slot, uint64_t* bar) {
    mbar_arrive_expect(bar, kSlotFloats * 4);
    if (AXIS == 0) tma_load_2d(slot, &it.tm[0], 32 * g, d.c0, bar);
    else if (AXIS == 1) tma_load_3d(slot, &it.tm[1], d.c0, 32 * g, d.c2, bar);
    else tma_load_2d(slot, &it.tm[2], d.c0, 32 * g, bar);
}
template <int AXIS>
__device__ __forceinline__ void bbox_store(const BatchItem& it, const BTile& d, int g, const float* slot) {
    if (AXIS == 0) tma_store_2d(&it.tm[0], 32 * g, d.c0, slot);
    else if (AXIS == 1) tma_store_3d(&it.tm[1], d.c0, 32 * g, d.c2, slot);
    else tma_store_2d(&it.tm[2], d.c0, 32 * g, slot);
}

template <int AXIS>
__device__ __forceinline__ bool batch_tile(const BatchArgs& a, const BatchItem& it, const BTile& d, float* buf,
                                           uint64_t* full, uint64_t* empty, const float* sE, uint32_t perm,
                                           uint32_t& fph) {
    const int N = it.g.N;
    const int B = it.B;
    const int lane = threadIdx.x & 31;
    const SubDev& sd = it.sd;
    SweepCtx c;
    c.E = sE;
    c.FR = sd.FRS;
    c.b = sd.b;
    c.dt = 0.f;
    uint32_t special = 0;
    XReset xr{0, 0, c.b};
    if (AXIS == 0) {
        const bool sp = !d.flagged_lane && !d.interior_lane;
        xr.lo = d.flagged_lane ? 1 : (d.interior_lane ? 2 : 0x7fffffff);
        xr.hi = d.flagged_lane ? N - 2 : N - 3;
        special = __ballot_sync(FULL, sp);
    }
    float Y = c.b;
    for (int g = 0; g < B; ++g) {
        const int s = (int)perm_get(perm, g);
        if (!mbar_wait(full + s, (fph >> s) & 1u, a.err, 1 + AXIS)) return false;
        fph ^= 1u << s;
        float* slot = buf + (size_t)s * kSlotFloats;
        const bool edge = g == 0 || 32 * g + 31 > N - 3;
        const bool rs = AXIS == 0 && (edge || special != 0);
        if (AXIS != 0 && edge) edge_rows<AXIS>(c, slot, g, N, lane);
        if ((sd.uni >> g) & 1u) forward_uniform<AXIS>(slot, g, lane, Y, sd.nE, rs, xr);
        else forward_group<AXIS>(c, slot, g, lane, Y, rs, xr);
    }
    float x = c.b;
    for (int g = B - 1; g >= 0; --g) {
        const int s = (int)perm_get(perm, g);
        float* slot = buf + (size_t)s * kSlotFloats;
        backward_group<AXIS>(c, sd, slot, g, lane, x, it.exact);
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
    }
    return true;
}

template <int AXIS>
__device__ void batch_producer(const BatchArgs& a, float* buf, uint64_t* full, uint64_t* empty, long long t,
                               long long t_end, int Bmax) {
    int item = 0;
    BTile d = btile<AXIS>(a, t, item);
    uint32_t perm = perm_identity(), eph = 0;
    {
        const BatchItem& it = a.items[d.item];
        for (int g = 0; g < it.B; ++g) bbox_load<AXIS>(it, d, g, buf + (size_t)g * kSlotFloats, full + g);
    }
    for (;;) {
        const BatchItem& it = a.items[d.item];
        const int B = it.B;
        const long long tn = t + 1;
        const bool has_next = tn < t_end;
        int itemn = item;
        const BTile dn = has_next ? btile<AXIS>(a, tn, itemn) : d;
        const BatchItem& itn = a.items[dn.item];
        const int Bn = has_next ? itn.B : 0;
        const uint32_t permn = has_next ? batch_perm_next(perm, B, Bn, Bmax) : 0u;
        // the next tile's first groups into the slots this tile leaves unused (every store has read
        // its slot: the previous tile ended with a full wait)
        int nxt = 0;
        uint32_t used = 0;
        for (int g = 0; g < B; ++g) used |= 1u << perm_get(perm, g);
        for (int sl = 0; sl < Bmax && nxt < Bn; ++sl)
            if (!((used >> sl) & 1u)) {
                bbox_load<AXIS>(itn, dn, nxt, buf + (size_t)sl * kSlotFloats, full + sl);
                ++nxt;
            }
        for (int g = B - 1; g >= 0; --g) {
            const int s = (int)perm_get(perm, g);
            if (!mbar_wait1(empty + s, (eph >> s) & 1u, a.err, 8 + AXIS)) {
                asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                return;
            }
            eph ^= 1u << s;
            bbox_store<AXIS>(it, d, g, buf + (size_t)s * kSlotFloats);
            bulk_commit();
            if (g + 1 <= B - 1 && nxt < Bn) {
                // the store of group g+1 has read its slot: it takes the next tile's next group
                bulk_wait_read<1>();
                const int s1 = (int)perm_get(perm, g + 1);
                bbox_load<AXIS>(itn, dn, nxt, buf + (size_t)s1 * kSlotFloats, full + s1);
                ++nxt;
            }
        }
        if (!has_next) break;
        bulk_wait_read<0>();
        if (nxt < Bn) {
            const int s0 = (int)perm_get(perm, 0);
            bbox_load<AXIS>(itn, dn, nxt, buf + (size_t)s0 * kSlotFloats, full + s0);
            ++nxt;
        }
        perm = permn;
        t = tn;
        d = dn;
        item = itemn;
    }
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// blockDim = 2W warps: W compute warps, then their W producer warps.  Shared memory: W x Bmax slots,
// per-warp E buffers of Namax floats, then the slot barriers.
template <int AXIS>
__global__ void __launch_bounds__(64 * kBatchWarps, 1) k_sweep_batch(const __grid_constant__ BatchArgs a, int Bmax) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int W = blockDim.x >> 6, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Namax = 32 * Bmax;
    const uint32_t base = smem_u32(sm);
    unsigned char* sm1 = sm + ((1024 - (base & 1023)) & 1023);
    float* slots = reinterpret_cast<float*>(sm1);
    float* sEs = reinterpret_cast<float*>(sm1 + (size_t)W * Bmax * kSlotFloats * 4);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm1 + (size_t)W * Bmax * kSlotFloats * 4 + align128(W * Namax * 4));
    uint64_t* empty = full + W * kBatchMaxGroups;
    for (int i = threadIdx.x; i < W * kBatchMaxGroups; i += blockDim.x) {
        mbar_init(full + i, 1u);
        mbar_init(empty + i, 1u);
    }
    fence_mbar_init();
    __syncthreads();
    // this warp pair's contiguous range of tiles: an equal share of the axis' work
    const int wi = warp >= W ? warp - W : warp;
    const long long nwg = (long long)gridDim.x * W, wg = (long long)blockIdx.x * W + wi;
    const long long t_begin = tile_at_cost<AXIS>(a, a.cost[AXIS] * wg / nwg);
    const long long t_end = tile_at_cost<AXIS>(a, a.cost[AXIS] * (wg + 1) / nwg);
    if (warp >= W) {
        if (lane == 0 && t_begin < t_end)
            batch_producer<AXIS>(a, slots + (size_t)wi * Bmax * kSlotFloats, full + wi * kBatchMaxGroups,
                                 empty + wi * kBatchMaxGroups, t_begin, t_end, Bmax);
        return;
    }
    float* buf = slots + (size_t)warp * Bmax * kSlotFloats;
    float* sE = sEs + (size_t)warp * Namax;
    uint64_t* fb = full + warp * kBatchMaxGroups;
    uint64_t* eb = empty + warp * kBatchMaxGroups;
    uint32_t perm = perm_identity(), fph = 0;
    int item = 0, staged = -1;
    BTile dnext = t_begin < t_end ? btile<AXIS>(a, t_begin, item) : BTile{};
    for (long long t = t_begin; t < t_end; ++t) {
        // the next tile's description is requested one tile ahead (see k_sweep)
        const BTile d = dnext;
        if (t + 1 < t_end) dnext = btile<AXIS>(a, t + 1, item);
        const BatchItem& it = a.items[d.item];
        if (d.item != staged) {
            // E of the elements the reference's recurrences update; 0 elsewhere (identity)
            const int N = it.g.N;
            __syncwarp();
            for (int j = lane; j < 32 * it.B; j += 32) sE[j] = (j >= 1 && j <= N - 2) ? it.sd.EFR[j] : 0.f;
            __syncwarp();
            staged = d.item;
        }
        if (!batch_tile<AXIS>(a, it, d, buf, fb, eb, sE, perm, fph)) break;
        if (t + 1 < t_end) perm = batch_perm_next(perm, it.B, a.items[dnext.item].B, Bmax);
    }
}

// Setboundary + meshupdatekernel on the listed uptake lines of every item (k_source_lines over
// many grids).
// The listed lines of all items form one sequence (item by item, each item's list in order) that
// the warps share round-robin: line g of the sequence goes to warp g mod (warps in the grid), so
// every warp takes about the same number of lines whatever the items' counts.  The counts live on
// the device (PreLOD builds the lists), so each warp reads them 32 items at a time and scans them;
// a line's item is the last one whose first index is not after it.  A line (N <= 256 here) is one
// batch of 8 loads per lane.
__global__ void k_source_lines_batch(const SrcItem* items, int nitems) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    long long base = 0;  // lines of the items before this group of 32
    for (int i0 = 0; i0 < nitems; i0 += 32) {
        const int s = i0 + lane;
        const int cnt = s < nitems ? *items[s].count : 0;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - cnt;
        const int gtot = __shfl_sync(FULL, incl, 31);
        for (long long g = base + ((gw - base) % nw + nw) % nw; g < base + gtot; g += nw) {
            const int r = (int)(g - base);
            const unsigned m = __ballot_sync(FULL, s < nitems && excl <= r);
            const int src = 31 - __clz(m);
            const int li = r - __shfl_sync(FULL, excl, src);
            const SrcItem& it = items[i0 + src];
            const int N = it.N;
            const int line = it.list[li];
            const int y = line % N, z = line / N;
            const bool bl = y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
            float* pl = it.p + (long long)line * it.P;
            const float* rl = it.rate + (long long)line * it.P;
            float pv[8], rv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = 32 * k + lane;
                pv[k] = j < N ? pl[j] : 0.f;
                rv[k] = j < N ? rl[j] : 0.f;
            }
            // as k_source_lines: a zero rate divides by exactly 1, so interior elements without
            // uptake are left as they are
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = 32 * k + lane;
                const bool edge = bl || j < 2 || j > N - 3;
                if (j < N && (edge || rv[k] != 0.f)) pl[j] = __fdiv_rn(edge ? it.b : pv[k], __fmaf_rn(-rv[k], it.dt, 1.f));
            }
        }
        base += gtot;
    }
}

// The bounded wait's give-up path: nothing ever arrives on this barrier, so the wait must stop after
// `polls` polls and record code 12 in the context's error word, as a sweep does when a box never
// lands.  Run by gell_selftest_timeout; the context stays usable afterwards.
__global__ void k_wait_check(int polls, int* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1u);
    fence_mbar_init();
    __syncthreads();
    mbar_wait(&bar, 0u, err, 12, polls);
}

// Markstein division against IEEE division on random operands in the sweeps' range.
__global__ void k_div_check(long long n, unsigned long long seed, unsigned long long* bad) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 r = philox4x32_10(make_uint4((uint32_t)i, (uint32_t)(i >> 32), 7u, 0u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    // dividend: any sign, magnitudes 2^-20 .. 2^20; divisor: 1 .. 64 (F_i of the sweeps)
    const float a = __uint_as_float((r.x & 0x80000000u) | ((107u + (r.y % 41u)) << 23) | (r.z & 0x7fffffu));
    const float f = __uint_as_float((127u + (r.w % 6u)) << 23 | (r.x & 0x7fffffu));
    const float y = __frcp_rn(f);
    if (__float_as_uint(div_rn(a, f, y)) != __float_as_uint(__fdiv_rn(a, f))) atomicAdd(bad, 1ull);
}

// Setboundary + meshupdatekernel on the x-lines that hold uptake (the lines PreLOD listed), in
// place, one line per warp: p = (boundary ? b : p) / fma(-rate, dt, 1).  Runs before the x sweep,
// which then leaves these lines as they are (apart from elements 0 and N-1).
struct SrcArgs {
    float* p[kMaxSub];
    const float* rate[kMaxSub];
    const int* list[kMaxSub];
    const int* count[kMaxSub];
    float b[kMaxSub];
    int nsub;
    Geom g;
    float dt;
};

__global__ void k_source_lines(SrcArgs a) {
    const int N = a.g.N, P = a.g.P;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (int s = 0; s < a.nsub; ++s) {
        const int cnt = *a.count[s];
        for (long long li = gw; li < cnt; li += nw) {
            const int line = a.list[s][li];
            const int y = line % N, z = line / N;
            const bool bl = y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
            float* pl = a.p[s] + (long long)line * P;
            const float* rl = a.rate[s] + (long long)line * P;
            for (int j0 = 0; j0 < N; j0 += 32 * 8) {
                float pv[8], rv[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int j = j0 + 32 * k + lane;
                    pv[k] = j < N ? pl[j] : 0.f;
                    rv[k] = j < N ? rl[j] : 0.f;
                }
                // where the rate is 0 the divisor is exactly 1 and an interior element keeps its
                // value: only boundary elements and elements with uptake are divided and written
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int j = j0 + 32 * k + lane;
                    const bool edge = bl || j < 2 || j > N - 3;
                    if (j < N && (edge || rv[k] != 0.f)) {
                        const float v = edge ? a.b[s] : pv[k];
                        pl[j] = __fdiv_rn(v, __fmaf_rn(-rv[k], a.dt, 1.f));
                    }
                }
            }
        }
    }
}

// ------------------------------------------------------------------ uptake map (PreLOD)

struct PreArgs {
    float* rate[kMaxSub];
    uint32_t* flag[kMaxSub];
    int* list[kMaxSub];
    int* count[kMaxSub];
    float coef[kMaxSub];
    int nsub;
    Geom g;
    float dead;
};

__global__ void k_rate_reset(PreArgs a) { rate_reset_body(a, blockIdx.x, gridDim.x); }

__global__ void k_rate_accum(CellsSoA c, int n, PreArgs a) { rate_accum_body(c, n, a, blockIdx.x); }

int g_num_sms = 0;
int num_sms() {
    if (!g_num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

// The uptake-source kernels: as many CTAs of 256 threads as are resident at once (one wave), each
// warp walking its share of the listed lines; a second, partial wave would start its lines only as
// the first wave's CTAs end.  `cache` keeps the count per kernel.
int one_wave_ctas(const void* kern, int* cache) {
    if (!*cache) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, 0) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            occ = 4;
        }
        *cache = num_sms() * occ;
    }
    return *cache;
}
int g_source_ctas = 0, g_source_batch_ctas = 0;
int source_ctas() { return one_wave_ctas((const void*)k_source_lines, &g_source_ctas); }
int source_batch_ctas() { return one_wave_ctas((const void*)k_source_lines_batch, &g_source_batch_ctas); }

}  // namespace

gell_status prelod(gell_ctx* c, int sub) {
    if (c->subs.empty()) return GELL_OK;
    PreArgs a{};
    int s0 = sub < 0 ? 0 : sub, s1 = sub < 0 ? (int)c->subs.size() : sub + 1;
    for (int s = s0; s < s1; ++s) {
        Substrate& S = c->subs[s];
        a.rate[a.nsub] = S.rate;
        a.flag[a.nsub] = S.line_flag;
        a.list[a.nsub] = S.line_list;
        a.count[a.nsub] = S.line_count;
        a.coef[a.nsub] = S.s.uptake;
        a.nsub++;
    }
    a.g = c->g;
    a.dead = c->P.dead_uptake_factor;
    GELL_KERNEL(c, "k_rate_reset", k_rate_reset<<<num_sms() * 4, 256, 0, c->stream>>>(a));
    for (int s = 0; s < a.nsub; ++s) GELL_CUDA(c, cudaMemsetAsync(a.count[s], 0, 4, c->stream));
    if (c->n > 0) {
        GELL_KERNEL(c, "k_rate_accum", k_rate_accum<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(c->cur(), c->n, a));
    }
    c->rate_valid = true;
    return GELL_OK;
}

// The ring sweeps (k_sweep_ring): W warps per CTA, each with R group slots, R as large as shared
// memory allows (at most kRingMaxSlots, at least 2 unless a line is one group).
static gell_status lod_solver_ring(gell_ctx* c, const LodArgs& ax, const LodArgs& ay, const LodArgs& az, int s0,
                                   int s1, int substeps, cudaStream_t strm) {
    const int ns = ax.nsub;
    const int N = c->g.N;
    const int B = (N + 31) / 32;
    const int Na = (N + 31) & ~31;
    const int smem_cap = 227 * 1024;
    const int rmax = c->sweep_ring >= 2 ? c->sweep_ring : kRingMaxSlots;
    int W = c->sweep_warps > 0 ? 2 * c->sweep_warps : kRingWarps;
    if (W > kRingWarps) W = kRingWarps;
    int R = 0;
    for (; W >= 1; W /= 2) {
        const int fixed = 1024 + align128(ns * Na * 4) + align128(W * B * 32 * 4) + W * kRingMaxSlots * 8;
        R = (smem_cap - fixed) / (W * kSlotFloats * 4);
        if (R > rmax) R = rmax;
        if (R > B) R = B;
        if (R >= 2 || (B == 1 && R == 1)) break;
    }
    if (W < 1) return fail(c, GELL_ERR_UNSUPPORTED, "grid edge too large for the ring sweeps");
    const int smem = 1024 + W * R * kSlotFloats * 4 + align128(ns * Na * 4) + align128(W * B * 32 * 4) + W * R * 8;
    // stores in flight per warp before a stored slot is refilled (1..R-1; a one-slot ring refills at once)
    int L = c->sweep_ring_lag > 0 ? c->sweep_ring_lag : 1;
    if (L > R - 1) L = R - 1;
    const bool hint = c->sweep_l2hint;
    const void* kx = hint ? (const void*)k_sweep_ring<0, true> : (const void*)k_sweep_ring<0, false>;
    const void* ky = hint ? (const void*)k_sweep_ring<1, true> : (const void*)k_sweep_ring<1, false>;
    const void* kz = hint ? (const void*)k_sweep_ring<2, true> : (const void*)k_sweep_ring<2, false>;
    if (!c->ring_configured) {
        for (const void* k : {(const void*)k_sweep_ring<0, true>, (const void*)k_sweep_ring<1, true>,
                              (const void*)k_sweep_ring<2, true>, (const void*)k_sweep_ring<0, false>,
                              (const void*)k_sweep_ring<1, false>, (const void*)k_sweep_ring<2, false>})
            GELL_CUDA(c, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        c->ring_configured = true;
    }
    const long long xt = ((long long)N * N + 31) / 32 * ns;
    const long long yt = (long long)((c->g.P + 31) / 32) * N * ns;
    const long long zt = (c->g.PN + 31) / 32 * ns;
    auto grid = [&](long long tiles, const void* kern) {
        int occ = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, W * 32, smem) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            occ = 1;
        }
        long long want = (tiles + W - 1) / W;
        long long cap = (long long)num_sms() * occ;
        return (int)(want < cap ? want : cap);
    };
    const int gx = grid(xt, kx), gy = grid(yt, ky), gz = grid(zt, kz);
    SrcArgs sa{};
    for (int s = s0; s < s1; ++s) {
        const Substrate& S = c->subs[s];
        sa.p[sa.nsub] = S.p;
        sa.rate[sa.nsub] = S.rate;
        sa.list[sa.nsub] = S.line_list;
        sa.count[sa.nsub] = S.line_count;
        sa.b[sa.nsub] = S.s.boundary;
        sa.nsub++;
    }
    sa.g = c->g;
    sa.dt = c->P.diffusion_dt;
    for (int k = 0; k < substeps; ++k) {
        GELL_KERNEL(c, "k_source_lines", k_source_lines<<<source_ctas(), 256, 0, strm>>>(sa));
        if (hint) {
            GELL_KERNEL(c, "k_sweep_x", k_sweep_ring<0, true><<<gx, W * 32, smem, strm>>>(ax, R, L));
            GELL_KERNEL(c, "k_sweep_y", k_sweep_ring<1, true><<<gy, W * 32, smem, strm>>>(ay, R, L));
            GELL_KERNEL(c, "k_sweep_z", k_sweep_ring<2, true><<<gz, W * 32, smem, strm>>>(az, R, L));
        } else {
            GELL_KERNEL(c, "k_sweep_x", k_sweep_ring<0, false><<<gx, W * 32, smem, strm>>>(ax, R, L));
            GELL_KERNEL(c, "k_sweep_y", k_sweep_ring<1, false><<<gy, W * 32, smem, strm>>>(ay, R, L));
            GELL_KERNEL(c, "k_sweep_z", k_sweep_ring<2, false><<<gz, W * 32, smem, strm>>>(az, R, L));
        }
    }
    return GELL_OK;
}

// Whether the line-tile kernels keep fewer than four line tiles per SM at this grid edge (a tile is
// the whole line in shared memory), in which case the ring sweeps are used by default.
static bool ring_by_default(const gell_ctx* c, int ns) {
    const int N = c->g.N;
    const int B = (N + 31) / 32;
    const int Na = (N + 31) & ~31;
    const int fixed = 1024 + align128(ns * Na * 4) + 2 * 8 * 32 * 8;
    return (227 * 1024 - fixed) / (B * kSlotFloats * 4) < 4;
}

// LOD substeps of substrates [s0, s1) on stream `strm`.
static gell_status lod_solver_range(gell_ctx* c, int s0, int s1, int substeps, cudaStream_t strm) {
    LodArgs ax{}, ay{}, az{};
    int ns = 0;
    for (int s = s0; s < s1; ++s, ++ns) {
        const Substrate& S = c->subs[s];
        const int N = c->g.N;
        const float R = S.conv_R;
        const SubDev sd{S.p,         S.rate,  S.line_flag,       S.EF,         S.FRS, S.s.boundary,
                        S.side,      S.uniform_groups,           -S.E[N - 2],  -S.side,
                        -(S.side * R), -S.F[N - 2],              R};
        ax.sub[ns] = ay.sub[ns] = az.sub[ns] = sd;
        ax.tm[ns] = S.tmap[0];
        ay.tm[ns] = S.tmap[1];
        az.tm[ns] = S.tmap[2];
    }
    for (LodArgs* a : {&ax, &ay, &az}) {
        a->nsub = ns;
        a->g = c->g;
        a->dt = c->P.diffusion_dt;
        a->err = c->dev_err;
        a->exact = c->exact_chain ? 1 : 0;
    }
    const int N = c->g.N;
    const int B = (N + 31) / 32;
    const int Na = (N + 31) & ~31;
    const int smem_cap = 227 * 1024;
    if (c->sweep_ring > 0 || (c->sweep_ring < 0 && ring_by_default(c, ns)))
        return lod_solver_ring(c, ax, ay, az, s0, s1, substeps, strm);
    const int fixed = 1024 + align128(ns * Na * 4) + 2 * 8 * 32 * 8;
    int w = (smem_cap - fixed) / (B * kSlotFloats * 4);
    w = w > kMaxComputeWarps ? kMaxComputeWarps : w;
    if (c->sweep_warps > 0 && w > c->sweep_warps) w = c->sweep_warps;
    if (w < 1) return fail(c, GELL_ERR_UNSUPPORTED, "grid edge too large for the shared-memory line tiles");
    const int smem = 1024 + w * B * kSlotFloats * 4 + align128(ns * Na * 4) + 2 * w * 32 * 8;
    // the shared-memory opt-in is a per-device function attribute: set once per context (each
    // context lives on one device)
    if (!c->sweeps_configured) {
        GELL_CUDA(c, cudaFuncSetAttribute(k_sweep<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        GELL_CUDA(c, cudaFuncSetAttribute(k_sweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        GELL_CUDA(c, cudaFuncSetAttribute(k_sweep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        c->sweeps_configured = true;
    }
    const long long xt = ((long long)N * N + 31) / 32 * ns;
    const long long yt = (long long)((c->g.P + 31) / 32) * N * ns;
    const long long zt = (c->g.PN + 31) / 32 * ns;
    // as many CTAs as the tiles need, up to what can be resident at once (one per SM for large grids;
    // several for small ones, whose CTAs need less shared memory)
    auto grid = [&](long long tiles, const void* kern) {
        int occ = 1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, w * 64, smem) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            occ = 1;
        }
        long long want = (tiles + w - 1) / w;
        long long cap = (long long)num_sms() * occ;
        return (int)(want < cap ? want : cap);
    };
    const int gx = grid(xt, (const void*)k_sweep<0>), gy = grid(yt, (const void*)k_sweep<1>),
              gz = grid(zt, (const void*)k_sweep<2>);
    SrcArgs sa{};
    for (int s = s0; s < s1; ++s) {
        const Substrate& S = c->subs[s];
        sa.p[sa.nsub] = S.p;
        sa.rate[sa.nsub] = S.rate;
        sa.list[sa.nsub] = S.line_list;
        sa.count[sa.nsub] = S.line_count;
        sa.b[sa.nsub] = S.s.boundary;
        sa.nsub++;
    }
    sa.g = c->g;
    sa.dt = c->P.diffusion_dt;
    for (int k = 0; k < substeps; ++k) {
        GELL_KERNEL(c, "k_source_lines", k_source_lines<<<source_ctas(), 256, 0, strm>>>(sa));
        GELL_KERNEL(c, "k_sweep_x", k_sweep<0><<<gx, w * 64, smem, strm>>>(ax));
        GELL_KERNEL(c, "k_sweep_y", k_sweep<1><<<gy, w * 64, smem, strm>>>(ay));
        GELL_KERNEL(c, "k_sweep_z", k_sweep<2><<<gz, w * 64, smem, strm>>>(az));
    }
    return GELL_OK;
}

// ------------------------------------------------------------------ batched sweeps: host side

struct LodBatch {
    BatchItem* d_items = nullptr;
    SrcItem* d_src = nullptr;
    int nitems = 0;
    long long total[3] = {0, 0, 0}, cost[3] = {0, 0, 0};
    int Bmax = 0;
    gell_ctx* c0 = nullptr;  // launches counted and timeouts reported on the first member
};

gell_status lod_batch_build(const std::vector<gell_ctx*>& ms, LodBatch** out) {
    *out = nullptr;
    std::vector<BatchItem> items;
    std::vector<SrcItem> src;
    long long tot[3] = {0, 0, 0}, cost[3] = {0, 0, 0};
    int Bmax = 0;
    for (gell_ctx* c : ms) {
        const int N = c->g.N, P = c->g.P;
        const int B = (N + 31) / 32;
        if (B > kBatchMaxGroups) return GELL_ERR_UNSUPPORTED;
        for (Substrate& S : c->subs) {
            BatchItem it;
            std::memset(&it, 0, sizeof(it));
            for (int k = 0; k < 3; ++k) it.tm[k] = S.tmap[k];
            const float R = S.conv_R;
            it.sd = SubDev{S.p,    S.rate,           S.line_flag, S.EF,        S.FRS,      S.s.boundary, S.side,
                           S.uniform_groups, -S.E[N - 2], -S.side, -(S.side * R), -S.F[N - 2], R};
            it.g = c->g;
            it.B = B;
            it.exact = c->exact_chain ? 1 : 0;
            const long long tiles[3] = {((long long)N * N + 31) / 32, (long long)((P + 31) / 32) * N,
                                        (c->g.PN + 31) / 32};
            for (int k = 0; k < 3; ++k) {
                it.tile0[k] = tot[k];
                it.cost0[k] = cost[k];
                tot[k] += tiles[k];
                cost[k] += tiles[k] * (B + 1);
            }
            items.push_back(it);
            src.push_back(SrcItem{S.p, S.rate, S.line_list, S.line_count, S.s.boundary, c->P.diffusion_dt, N, P});
            if (B > Bmax) Bmax = B;
        }
    }
    if (items.empty()) return GELL_ERR_INVALID_ARG;
    LodBatch* b = new LodBatch;
    b->nitems = (int)items.size();
    for (int k = 0; k < 3; ++k) {
        b->total[k] = tot[k];
        b->cost[k] = cost[k];
    }
    b->Bmax = Bmax;
    b->c0 = ms[0];
    bool ok = cudaMalloc((void**)&b->d_items, sizeof(BatchItem) * items.size()) == cudaSuccess &&
              cudaMalloc((void**)&b->d_src, sizeof(SrcItem) * src.size()) == cudaSuccess &&
              cudaMemcpy(b->d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(b->d_src, src.data(), sizeof(SrcItem) * src.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (ok && dev >= 0 && dev < 64 && !configured[dev]) {
        for (const void* k : {(const void*)k_sweep_batch<0>, (const void*)k_sweep_batch<1>, (const void*)k_sweep_batch<2>})
            ok = ok && cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) == cudaSuccess;
        configured[dev] = ok;
    }
    if (!ok) {
        cudaGetLastError();
        lod_batch_free(b);
        return GELL_ERR_CUDA;
    }
    *out = b;
    return GELL_OK;
}

void lod_batch_free(LodBatch* b) {
    if (!b) return;
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_src) cudaFree(b->d_src);
    delete b;
}

gell_status lod_batch_run(LodBatch* b, cudaStream_t st, int substeps) {
    gell_ctx* c = b->c0;
    const int W = kBatchWarps;
    const int Namax = 32 * b->Bmax;
    const int smem = 1024 + W * b->Bmax * kSlotFloats * 4 + align128(W * Namax * 4) + 2 * W * kBatchMaxGroups * 8;
    BatchArgs a{};
    a.items = b->d_items;
    a.nitems = b->nitems;
    for (int k = 0; k < 3; ++k) {
        a.total[k] = b->total[k];
        a.cost[k] = b->cost[k];
    }
    a.err = c->dev_err;
    auto grid = [&](long long tiles) {
        const long long want = (tiles + W - 1) / W;
        return (int)(want < num_sms() ? want : num_sms());
    };
    for (int k = 0; k < substeps; ++k) {
        GELL_KERNEL(c, "k_source_lines", k_source_lines_batch<<<source_batch_ctas(), 256, 0, st>>>(b->d_src, b->nitems));
        GELL_KERNEL(c, "k_sweep_x", k_sweep_batch<0><<<grid(a.total[0]), W * 64, smem, st>>>(a, b->Bmax));
        GELL_KERNEL(c, "k_sweep_y", k_sweep_batch<1><<<grid(a.total[1]), W * 64, smem, st>>>(a, b->Bmax));
        GELL_KERNEL(c, "k_sweep_z", k_sweep_batch<2><<<grid(a.total[2]), W * 64, smem, st>>>(a, b->Bmax));
    }
    return GELL_OK;
}

// A stream per substrate (GELL_OPT_LOD_STREAMS): the substrates' substeps are independent chains,
// so on separate streams one sweep's ramp-up and drain (an SM whose last tile is done while others
// still work) overlap another substrate's sweep instead of idling the GPU between launches.
static bool substrate_streams(gell_ctx* c, int s0, int s1) {
    if (!c->lod_streams || s1 - s0 < 2 || c->prof_on) return false;
    for (int s = s0 + 1; s < s1; ++s) {
        if (c->sub_stream[s]) continue;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
        if (cudaStreamCreateWithFlags(&c->sub_stream[s], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->sub_join[s], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
    }
    if (!c->sub_fork && cudaEventCreateWithFlags(&c->sub_fork, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

gell_status lod_solver(gell_ctx* c, int sub, int substeps) {
    if (c->subs.empty() || substeps == 0) return GELL_OK;
    const int s0 = sub < 0 ? 0 : sub, s1 = sub < 0 ? (int)c->subs.size() : sub + 1;
    if (!substrate_streams(c, s0, s1)) return lod_solver_range(c, s0, s1, substeps, c->stream);
    GELL_CUDA(c, cudaEventRecord(c->sub_fork, c->stream));
    for (int s = s0 + 1; s < s1; ++s) GELL_CUDA(c, cudaStreamWaitEvent(c->sub_stream[s], c->sub_fork, 0));
    for (int s = s0; s < s1; ++s) {
        gell_status st = lod_solver_range(c, s, s + 1, substeps, s == s0 ? c->stream : c->sub_stream[s]);
        if (st != GELL_OK) return st;
    }
    for (int s = s0 + 1; s < s1; ++s) {
        GELL_CUDA(c, cudaEventRecord(c->sub_join[s], c->sub_stream[s]));
        GELL_CUDA(c, cudaStreamWaitEvent(c->stream, c->sub_join[s], 0));
    }
    return GELL_OK;
}

gell_status selftest_timeout(gell_ctx* c, int polls) {
    GELL_KERNEL(c, "k_wait_check", k_wait_check<<<1, 32, 0, c->stream>>>(polls, c->dev_err));
    return GELL_OK;
}

gell_status selftest_division(gell_ctx* c, long long n, unsigned long long seed, long long* mismatches) {
    unsigned long long* d = nullptr;
    GELL_CUDA(c, cudaMallocAsync((void**)&d, 8, c->stream));
    GELL_CUDA(c, cudaMemsetAsync(d, 0, 8, c->stream));
    GELL_KERNEL(c, "k_div_check", k_div_check<<<(int)((n + 255) / 256), 256, 0, c->stream>>>(n, seed, d));
    unsigned long long h = 0;
    GELL_CUDA(c, cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, c->stream));
    GELL_CUDA(c, cudaFreeAsync(d, c->stream));
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    *mismatches = (long long)h;
    return GELL_OK;
}

}  // namespace gell
