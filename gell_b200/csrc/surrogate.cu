// surrogate.cu — learned oxygen surrogate: a 3-D convolutional operator that replaces K LOD substeps
// of one substrate, judged after every use by one plain LOD substep and replaced by the plain solve
// when the judge rejects it.  No reference counterpart: the reference only has the plain solver
// (include/LODkernel.cuh:280-300), which is the fallback here and the source of the training pairs.
//
// Operator.  Input channels [p / b, rate * rate_scale, shell mask] (b = the substrate's boundary
// value, shell = the four boundary layers that Setboundary rewrites), a 3x3x3 convolution to 32
// channels with ReLU, four residual blocks h += conv(relu(conv(h))) (the inner one with ReLU), and a
// 3x3x3 convolution to one channel d; the output field is p + b * d inside and b on the shell.  All
// convolutions are zero-padded ("same"), weights and activations are bf16, sums are fp32.
//
// Activation layout in HBM ("8-channel planes").  A tensor of C channels over the N^3 voxels is
// C/8 planes; plane q holds channels 8q..8q+7 of voxel v = x + N*(y + N*z) as 16 contiguous bytes at
// byte 16*v.  An x-run of voxels of one plane is then exactly the canonical no-swizzle K-major
// operand layout of the tensor cores (8 rows of 16 bytes per core matrix, consecutive voxels 16
// bytes apart), so the operand of tap dx is the run staged for dx = 0 moved by 16*dx bytes.
//
// k_conv3 (implicit GEMM on tcgen05).  A tile is 128 consecutive voxels of one x-line (M = 128) by
// all output channels (N = NOUT); K runs over the 27 taps x the input channels, 16 channels per
// MMA.  Per tile one TMA box per (dy, dz) brings the 130-voxel run x0-1 .. x0+128 of all input
// planes (zero fill outside the grid gives the padding), 9 boxes in all; the weights of the whole
// layer stay in shared memory.  Warp 0 issues the TMA loads (two tile stages), one thread of warp 1
// issues the MMAs into one of two TMEM accumulators and commits them to mbarriers, warps 2-5 read
// the finished accumulator (tcgen05.ld), apply bias, ReLU / residual / field update and store.
// Every wait is bounded (codes 21-27 in the context's error word).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "async_copy.cuh"
#include "gell_internal.cuh"

namespace gell {

struct SurrogateState;

namespace {

constexpr int kTileM = 128;                  // voxels per tile
constexpr int kRunVox = kTileM + 2;          // staged voxels per (dy, dz) run, with the x halo
constexpr int kRunPlaneB = kRunVox * 16;     // bytes of one plane of one staged run (2080)
constexpr int kLayers = 10;                  // conv_in, 4 x (conv_a, conv_b), conv_out
constexpr int kHidden = 32;
constexpr int kInCh = 3;

// Epilogues: forward (kRelu, kResidual, kField) and the data gradients of the backward pass
// (kLinear: the gradient of a linear layer's input; kMask: times [aux > 0], the ReLU's gradient
// with aux = the ReLU's stored output; kResMask: residual add, then times [aux > 0]).
enum ConvMode { kRelu = 0, kResidual = 1, kField = 2, kLinear = 3, kMask = 4, kResMask = 5 };

struct ConvArgs {
    CUtensorMap in;                 // 5-D map {8, N, N, N, planes}, box {8, 130, 1, 1, planes}
    const uint8_t* w;               // packed weights, the shared-memory image
    const float* bias;              // NOUT
    uint4* out;                     // planes (kRelu, kResidual)
    const uint4* res;               // residual planes (kResidual, kResMask; may equal out)
    const uint4* aux;               // mask planes (kMask, kResMask): a channel passes where aux > 0
    float* field_out;               // pitched field (kField)
    const float* field_in;          // pitched field (kField)
    int N, P;
    long long PN;
    long long nvox;                 // N^3: plane length in voxels
    int tiles_x;
    long long tiles;
    float scale, bval;              // kField: out = in + scale * d inside, bval on the shell
    int* err;
};

// ---------------------------------------------------------------- tcgen05 / TMEM (inline PTX)

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t addr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols) : "memory");
}
// Shared-memory matrix descriptor, no swizzle: start, leading-dimension byte offset (between the
// two 8-element K chunks of an MMA), stride byte offset (between 8-row core-matrix groups), all in
// 16-byte units; bit 46 = descriptor version of sm_100.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
// The mbarrier completes one phase when every MMA issued so far by this thread has finished.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x 32 columns (x32) or 16 columns (x16) of fp32: thread t gets lane (base lane + t).
__device__ __forceinline__ void tmem_ld32(uint32_t a, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(a));
}
__device__ __forceinline__ void tmem_ld16(uint32_t a, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(a));
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpack_bf16(uint32_t u) {
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(h);
}

// Shared memory of one k_conv3 instance: two tile stages of 9 runs (each run padded to 128 bytes),
// the layer's weights, ten mbarriers and the TMEM address.
template <int CIN8, int NOUT>
struct ConvSmem {
    static constexpr int kRunB = (CIN8 * kRunPlaneB + 127) / 128 * 128;
    static constexpr int kStageB = 9 * kRunB;
    static constexpr int kHalves = CIN8 / 2;               // MMAs (16 input channels) per tap
    static constexpr int kWBlk = NOUT * 32;                // one (tap, half) weight block
    static constexpr int kWB = 27 * kHalves * kWBlk;
    static constexpr int kBars = 2 * kStageB + kWB;
    static constexpr int kBytes = kBars + 10 * 8 + 16;
};

__device__ __forceinline__ void tile_of(const ConvArgs& a, long long t, int& x0, int& y, int& z) {
    const long long line = t / a.tiles_x;
    x0 = (int)(t - line * a.tiles_x) * kTileM;
    y = (int)(line % a.N);
    z = (int)(line / a.N);
}

// Epilogue of one accumulator row (voxel x of line (y, z)): bias, then ReLU, residual add or the
// field update, and the store.
template <int NOUT, int MODE>
__device__ __forceinline__ void store_tile(const ConvArgs& a, const uint32_t (&v)[NOUT], const float (&bias)[NOUT],
                                           int x, int y, int z) {
    if (x >= a.N) return;
    if constexpr (MODE == kField) {
        const long long pi = (long long)x + (long long)a.P * y + a.PN * z;
        const int N = a.N;
        const bool shell = x < 2 || x > N - 3 || y < 2 || y > N - 3 || z < 2 || z > N - 3;
        const float d = __uint_as_float(v[0]) + bias[0];
        a.field_out[pi] = shell ? a.bval : __fmaf_rn(a.scale, d, a.field_in[pi]);
    } else {
        const long long vox = (long long)x + (long long)a.N * (y + (long long)a.N * z);
        float f[NOUT];
#pragma unroll
        for (int n = 0; n < NOUT; ++n) f[n] = __uint_as_float(v[n]) + bias[n];
#pragma unroll
        for (int pl = 0; pl < NOUT / 8; ++pl) {
            if constexpr (MODE == kResidual || MODE == kResMask) {
                const uint4 r = a.res[pl * a.nvox + vox];
                const uint32_t rr[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 u = unpack_bf16(rr[j]);
                    f[8 * pl + 2 * j] += u.x;
                    f[8 * pl + 2 * j + 1] += u.y;
                }
            }
            if constexpr (MODE == kMask || MODE == kResMask) {
                const uint4 m = a.aux[pl * a.nvox + vox];
                const uint32_t mm[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 u = unpack_bf16(mm[j]);
                    if (!(u.x > 0.f)) f[8 * pl + 2 * j] = 0.f;
                    if (!(u.y > 0.f)) f[8 * pl + 2 * j + 1] = 0.f;
                }
            }
            if constexpr (MODE == kRelu) {
#pragma unroll
                for (int j = 0; j < 8; ++j) f[8 * pl + j] = fmaxf(f[8 * pl + j], 0.f);
            }
            a.out[pl * a.nvox + vox] =
                make_uint4(pack_bf16(f[8 * pl], f[8 * pl + 1]), pack_bf16(f[8 * pl + 2], f[8 * pl + 3]),
                           pack_bf16(f[8 * pl + 4], f[8 * pl + 5]), pack_bf16(f[8 * pl + 6], f[8 * pl + 7]));
        }
    }
}

template <int CIN8, int NOUT, int MODE>
__global__ void __launch_bounds__(192, 1) k_conv3(const __grid_constant__ ConvArgs a) {
    using L = ConvSmem<CIN8, NOUT>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* wsm = smem + 2 * L::kStageB;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::kBars);
    uint64_t* full = bars;       // [2] stage loaded
    uint64_t* empty = bars + 2;  // [2] stage consumed by the MMAs
    uint64_t* accf = bars + 4;   // [2] accumulator complete
    uint64_t* acce = bars + 6;   // [2] accumulator read by the epilogue (4 warps)
    uint64_t* wbar = bars + 8;   // weights loaded
    uint64_t* done = bars + 9;   // every MMA of this CTA finished
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 10);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 4);
        }
        mbar_init(wbar, 1);
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(tslot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const long long T = a.tiles;

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect(wbar, (uint32_t)L::kWB);
            for (int off = 0; off < L::kWB; off += 16384) {
                const int nb = L::kWB - off < 16384 ? L::kWB - off : 16384;
                bulk_load(wsm + off, a.w + off, (uint32_t)nb, wbar);
            }
            int k = 0;
            for (long long t = blockIdx.x; t < T; t += gridDim.x, ++k) {
                const int s = k & 1;
                if (k >= 2 && !mbar_wait1(&empty[s], ((k >> 1) - 1) & 1, a.err, 21)) break;
                int x0, y, z;
                tile_of(a, t, x0, y, z);
                uint8_t* st = smem + s * L::kStageB;
                mbar_arrive_expect(&full[s], (uint32_t)(9 * CIN8 * kRunPlaneB));
                for (int r = 0; r < 9; ++r)
                    tma_load_5d(st + r * L::kRunB, &a.in, 0, x0 - 1, y + r % 3 - 1, z + r / 3 - 1, 0, &full[s]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(NOUT);
            bool ok = mbar_wait1(wbar, 0, a.err, 22);
            const uint64_t b0 = sdesc(smem_u32(wsm), NOUT * 16, 128);
            int k = 0;
            for (long long t = blockIdx.x; ok && t < T; t += gridDim.x, ++k) {
                const int s = k & 1;
                if (!mbar_wait1(&full[s], (k >> 1) & 1, a.err, 23)) break;
                if (k >= 2 && !mbar_wait1(&acce[s], ((k >> 1) - 1) & 1, a.err, 24)) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(s * 32);
                const uint64_t a0 = sdesc(smem_u32(smem + s * L::kStageB), kRunPlaneB, 128);
                // descriptors differ only in the start address (low 14 bits, 16-byte units, no carry
                // out: shared memory is below 256 KB), so each MMA adds a compile-time offset
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
#pragma unroll
                    for (int h = 0; h < L::kHalves; ++h) {
                        const uint32_t ao = ((tap / 3) * L::kRunB + (tap % 3) * 16 + 2 * h * kRunPlaneB) >> 4;
                        const uint32_t bo = ((tap * L::kHalves + h) * L::kWBlk) >> 4;
                        mma_bf16(d, a0 + ao, b0 + bo, idesc, (tap | h) != 0 ? 1u : 0u);
                    }
                }
                mma_commit(&empty[s]);
                mma_commit(&accf[s]);
            }
            mma_commit(done);
            mbar_wait1(done, 0, a.err, 25);
        }
    } else {
        const int q = warp & 3;  // TMEM lanes 32q..32q+31 are this warp's
        float bias[NOUT];
#pragma unroll
        for (int n = 0; n < NOUT; ++n) bias[n] = a.bias[n];
        int k = 0;
        for (long long t = blockIdx.x; t < T; t += gridDim.x, ++k) {
            const int s = k & 1;
            if (!mbar_wait(&accf[s], (k >> 1) & 1, a.err, 26)) break;
            tc_fence_after();
            uint32_t v[NOUT];
            const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(s * 32);
            if constexpr (NOUT == 32) tmem_ld32(ta, v);
            else tmem_ld16(ta, v);
            tmem_wait_ld();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[s]);
            int x0, y, z;
            tile_of(a, t, x0, y, z);
            store_tile<NOUT, MODE>(a, v, bias, x0 + 32 * q + lane, y, z);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 64);
    }
}

// ---------------------------------------------------------------- k_conv3_ring
// The same convolution with the input rows reused along y.  Work comes in units of up to kUnitY
// consecutive lines y0..y1-1 at one (x tile, z); a unit needs the row groups y0-1 .. y1 (a group =
// the three runs z-1, z, z+1 at one y, all planes), each loaded once into a ring of kRing group
// slots and used by the (up to) three tiles y-1, y, y+1 whose taps reach it.  A group's slot is
// released (tcgen05.commit on its empty barrier) by the last tile that reads it: the oldest group
// of every tile but the unit's last, and all three groups of the last.  L2 -> shared traffic is
// one group (3 runs) per tile instead of three.
constexpr int kUnitY = 32;
constexpr int kRing = 6;

template <int CIN8, int NOUT>
struct RingSmem {
    static constexpr int kRunB = (CIN8 * kRunPlaneB + 127) / 128 * 128;
    static constexpr int kGroupB = 3 * kRunB;
    static constexpr int kHalves = CIN8 / 2;
    static constexpr int kWBlk = NOUT * 32;
    static constexpr int kWB = 27 * kHalves * kWBlk;
    static constexpr int kBars = kRing * kGroupB + kWB;
    static constexpr int kBytes = kBars + (2 * kRing + 6) * 8 + 16;
};

__device__ __forceinline__ void unit_of(const ConvArgs& a, long long u, int& x0, int& y0, int& y1, int& z) {
    const int nyc = (a.N + kUnitY - 1) / kUnitY;
    const long long r = u / a.tiles_x;
    x0 = (int)(u - r * a.tiles_x) * kTileM;
    y0 = (int)(r % nyc) * kUnitY;
    y1 = y0 + kUnitY < a.N ? y0 + kUnitY : a.N;
    z = (int)(r / nyc);
}

template <int CIN8, int NOUT, int MODE>
__global__ void __launch_bounds__(192, 1) k_conv3_ring(const __grid_constant__ ConvArgs a) {
    using L = RingSmem<CIN8, NOUT>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* wsm = smem + kRing * L::kGroupB;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::kBars);
    uint64_t* full = bars;               // [kRing] group loaded
    uint64_t* empty = bars + kRing;      // [kRing] group released by the MMAs
    uint64_t* accf = bars + 2 * kRing;   // [2]
    uint64_t* acce = accf + 2;           // [2] (4 epilogue warps)
    uint64_t* wbar = acce + 2;
    uint64_t* done = wbar + 1;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 4);
        }
        mbar_init(wbar, 1);
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(tslot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int nyc = (a.N + kUnitY - 1) / kUnitY;
    const long long U = (long long)a.tiles_x * nyc * a.N;

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect(wbar, (uint32_t)L::kWB);
            for (int off = 0; off < L::kWB; off += 16384) {
                const int nb = L::kWB - off < 16384 ? L::kWB - off : 16384;
                bulk_load(wsm + off, a.w + off, (uint32_t)nb, wbar);
            }
            bool ok = true;
            int g = 0;
            for (long long u = blockIdx.x; ok && u < U; u += gridDim.x) {
                int x0, y0, y1, z;
                unit_of(a, u, x0, y0, y1, z);
                for (int yy = y0 - 1; yy <= y1; ++yy, ++g) {
                    const int sl = g % kRing;
                    if (g >= kRing && !mbar_wait1(&empty[sl], ((g / kRing) - 1) & 1, a.err, 21)) {
                        ok = false;
                        break;
                    }
                    uint8_t* gb = smem + sl * L::kGroupB;
                    mbar_arrive_expect(&full[sl], (uint32_t)(3 * CIN8 * kRunPlaneB));
                    for (int dz = 0; dz < 3; ++dz)
                        tma_load_5d(gb + dz * L::kRunB, &a.in, 0, x0 - 1, yy, z + dz - 1, 0, &full[sl]);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(NOUT);
            bool ok = mbar_wait1(wbar, 0, a.err, 22);
            const uint64_t b0 = sdesc(smem_u32(wsm), NOUT * 16, 128);
            const uint32_t rbase = smem_u32(smem);
            int g = 0, k = 0;
            for (long long u = blockIdx.x; ok && u < U; u += gridDim.x) {
                int x0, y0, y1, z;
                unit_of(a, u, x0, y0, y1, z);
                const int ny = y1 - y0;
                for (int i = 0; i < ny; ++i, ++k) {
                    const int ac = k & 1;
                    for (int j = 0; j < 3 && ok; ++j) {
                        const int gg = g + i + j;
                        ok = mbar_wait1(&full[gg % kRing], (gg / kRing) & 1, a.err, 23);
                    }
                    if (ok && k >= 2) ok = mbar_wait1(&acce[ac], ((k >> 1) - 1) & 1, a.err, 24);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(ac * 32);
                    uint64_t ga[3];  // descriptors of the three row groups (start addresses differ)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        ga[j] = sdesc(rbase + (uint32_t)(((g + i + j) % kRing) * L::kGroupB), kRunPlaneB, 128);
#pragma unroll
                    for (int tap = 0; tap < 27; ++tap) {
#pragma unroll
                        for (int h = 0; h < L::kHalves; ++h) {
                            const uint32_t ao = ((tap / 9) * L::kRunB + (tap % 3) * 16 + 2 * h * kRunPlaneB) >> 4;
                            const uint32_t bo = ((tap * L::kHalves + h) * L::kWBlk) >> 4;
                            mma_bf16(d, ga[(tap / 3) % 3] + ao, b0 + bo, idesc, (tap | h) != 0 ? 1u : 0u);
                        }
                    }
                    mma_commit(&accf[ac]);
                    if (i < ny - 1) {
                        mma_commit(&empty[(g + i) % kRing]);
                    } else {
                        for (int j = 0; j < 3; ++j) mma_commit(&empty[(g + i + j) % kRing]);
                    }
                }
                g += ny + 2;
            }
            mma_commit(done);
            mbar_wait1(done, 0, a.err, 25);
        }
    } else {
        const int q = warp & 3;
        float bias[NOUT];
#pragma unroll
        for (int n = 0; n < NOUT; ++n) bias[n] = a.bias[n];
        int k = 0;
        bool ok = true;
        for (long long u = blockIdx.x; ok && u < U; u += gridDim.x) {
            int x0, y0, y1, z;
            unit_of(a, u, x0, y0, y1, z);
            for (int y = y0; y < y1; ++y, ++k) {
                const int ac = k & 1;
                if (!mbar_wait(&accf[ac], (k >> 1) & 1, a.err, 26)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint32_t v[NOUT];
                const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(ac * 32);
                if constexpr (NOUT == 32) tmem_ld32(ta, v);
                else tmem_ld16(ta, v);
                tmem_wait_ld();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce[ac]);
                store_tile<NOUT, MODE>(a, v, bias, x0 + 32 * q + lane, y, z);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 64);
    }
}

// ---------------------------------------------------------------- weight gradients
// k_wgrad (32 -> 32 layers, tcgen05): dW[co][ci][tap] = sum over voxels v of X[ci, v + tap] * G[co, v]
// (X = the layer's input, G = the gradient of its output, zero outside the grid).  The voxels are
// the K dimension, so both operands are read MN-major from the 8-channel planes as staged (8
// channels of one voxel = 16 contiguous bytes, consecutive voxels 16 bytes apart: the canonical
// no-swizzle MN-major layout, channel groups SBO apart, voxel groups of 8 LBO = 128 bytes apart).
// Per tile (128 voxels of one x-line): the 9 runs of X (130 voxels, 4 planes) and the 128-voxel
// run of G (4 planes); A = four consecutive runs r0..r0+3 as M = 128 rows (run, ci) (the runs of a
// stage are 4 * 2080 bytes apart, so rows keep one stride), moved by dx voxels for tap dx; B = G.
// 3 row groups x 3 dx x 8 blocks of 16 voxels = 72 MMAs per tile into 9 TMEM accumulators (288
// columns) that persist over all tiles of the CTA; rows 9-11 of the last group read past the stage
// into other staged data and are discarded.  At the end each CTA writes its partial sums.
constexpr int kWgRunB = 4 * kRunPlaneB;            // 8320
constexpr int kWgXB = 9 * kWgRunB;                  // 74,880
constexpr int kWgGB = 4 * kTileM * 16;              // 8,192
constexpr int kWgStageB = kWgXB + kWgGB;            // 83,072
constexpr int kWgTail = 3 * kWgRunB;                // room for the discarded rows of the last stage
constexpr int kWgBars = 2 * kWgStageB + kWgTail;
constexpr int kWgBytes = kWgBars + 5 * 8 + 16;

__host__ __device__ constexpr uint32_t idesc_bf16_mn(int n) {
    return idesc_bf16(n) | (1u << 15) | (1u << 16);
}

struct WgradArgs {
    CUtensorMap x;  // {8, N, N, N, 4}, box {8, 130, 1, 1, 4}
    CUtensorMap g;  // {8, N, N, N, 4}, box {8, 128, 1, 1, 4}
    float* partial; // [gridDim.x][32 co][32 ci][27]
    int N, tiles_x;
    long long tiles;
    int* err;
};

__global__ void __launch_bounds__(192, 1) k_wgrad(const __grid_constant__ WgradArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kWgBars);
    uint64_t* full = bars;
    uint64_t* empty = bars + 2;
    uint64_t* done = bars + 4;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(tslot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const long long T = a.tiles;
    ConvArgs geo{};
    geo.N = a.N;
    geo.tiles_x = a.tiles_x;
    if (warp == 0) {
        if (lane == 0) {
            int k = 0;
            for (long long t = blockIdx.x; t < T; t += gridDim.x, ++k) {
                const int s = k & 1;
                if (k >= 2 && !mbar_wait1(&empty[s], ((k >> 1) - 1) & 1, a.err, 31)) break;
                int x0, y, z;
                tile_of(geo, t, x0, y, z);
                uint8_t* st = smem + s * kWgStageB;
                mbar_arrive_expect(&full[s], (uint32_t)(kWgXB + kWgGB));
                for (int r = 0; r < 9; ++r)
                    tma_load_5d(st + r * kWgRunB, &a.x, 0, x0 - 1, y + r % 3 - 1, z + r / 3 - 1, 0, &full[s]);
                tma_load_5d(st + kWgXB, &a.g, 0, x0, y, z, 0, &full[s]);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16_mn(32);
            int k = 0;
            for (long long t = blockIdx.x; t < T; t += gridDim.x, ++k) {
                const int s = k & 1;
                if (!mbar_wait1(&full[s], (k >> 1) & 1, a.err, 32)) break;
                tc_fence_after();
                const uint32_t sb = smem_u32(smem + s * kWgStageB);
                const uint64_t a0 = sdesc(sb, 128, kRunPlaneB);         // LBO = voxel groups, SBO = channel groups
                const uint64_t b0 = sdesc(sb + kWgXB, 128, kTileM * 16);
#pragma unroll
                for (int rg = 0; rg < 3; ++rg)
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx)
#pragma unroll
                        for (int kb = 0; kb < 8; ++kb) {
                            const uint32_t ao = (4 * rg * kWgRunB + (dx + 16 * kb) * 16) >> 4;
                            const uint32_t bo = (16 * kb * 16) >> 4;
                            mma_bf16(tmem + (uint32_t)(32 * (3 * rg + dx)), a0 + ao, b0 + bo, idesc,
                                     (k > 0 || kb > 0) ? 1u : 0u);
                        }
                mma_commit(&empty[s]);
            }
            mma_commit(done);
        }
    } else {
        // read the 9 accumulators once every MMA of the CTA has finished
        const int q = warp & 3;
        if (mbar_wait(done, 0, a.err, 33, 1 << 26)) {
            tc_fence_after();
            float* out = a.partial + (size_t)blockIdx.x * (32 * 32 * 27);
            const bool any = blockIdx.x < T;
            for (int j = 0; j < 9; ++j) {
                const int rg = j / 3, dx = j % 3;
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * j), v);
                tmem_wait_ld();
                const int r = 4 * rg + q;  // lane 32q + ci is row (run r, ci)
                if (r < 9) {
                    const int tap = 3 * r + dx;
#pragma unroll
                    for (int co = 0; co < 32; ++co)
                        out[((size_t)co * 32 + lane) * 27 + tap] = any ? __uint_as_float(v[co]) : 0.f;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

// Weight gradients of the thin layers on the CUDA cores (the first layer: 3 input channels; the
// last: one output channel).  A block takes one x-line at a time: the line's gradient run and, plane
// by plane, the 9 input runs (130 voxels) go to shared memory as fp32; thread t owns the real
// weights w = t, t + blockDim, ... in the layer's [co][ci][tap] order and accumulates over the
// line's voxels and over every line the block visits; each block writes its partial sums.
constexpr int kThinMaxW = 16;

// Staged runs are kept channel-major, xs[e][r][x] with a row pitch of 3 mod 32 words, so that the
// 27 taps a warp reads at one x fall in 27 different banks.
__host__ __device__ inline int thin_pitch(int N) { return (N + 2 - 3 + 31) / 32 * 32 + 3; }

__global__ void k_wgrad_thin(const uint4* X, int cin, const uint4* G, int cout, int N, long long nvox,
                             float* partial) {
    extern __shared__ float sm[];
    const int RUN = N + 2, RP = thin_pitch(N);
    float* xs = sm;                // [8][9][RP]
    float* gs = sm + 8 * 9 * RP;   // [N][cout]
    const int total = cout * cin * 27;
    float acc[kThinMaxW];
#pragma unroll
    for (int j = 0; j < kThinMaxW; ++j) acc[j] = 0.f;
    const long long lines = (long long)N * N;
    const int xplanes = (cin + 7) / 8;
    for (long long l = blockIdx.x; l < lines; l += gridDim.x) {
        const int y = (int)(l % N), z = (int)(l / N);
        __syncthreads();
        for (int i = threadIdx.x; i < N * cout; i += blockDim.x) {
            const int x = i / cout, co = i % cout;
            const long long vox = x + (long long)N * (y + (long long)N * z);
            const uint4 u = G[(co / 8) * nvox + vox];
            const uint32_t w4[4] = {u.x, u.y, u.z, u.w};
            const float2 f = unpack_bf16(w4[(co % 8) / 2]);
            gs[i] = (co & 1) ? f.y : f.x;
        }
        for (int pl = 0; pl < xplanes; ++pl) {
            __syncthreads();
            for (int i = threadIdx.x; i < 9 * RUN; i += blockDim.x) {
                const int r = i / RUN, xi = i % RUN;
                const int xx = xi - 1, yy = y + r % 3 - 1, zz = z + r / 3 - 1;
                uint4 u = make_uint4(0u, 0u, 0u, 0u);
                if (xx >= 0 && xx < N && yy >= 0 && yy < N && zz >= 0 && zz < N)
                    u = X[pl * nvox + xx + (long long)N * (yy + (long long)N * zz)];
                const uint32_t w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 f = unpack_bf16(w4[j]);
                    xs[((2 * j) * 9 + r) * RP + xi] = f.x;
                    xs[((2 * j + 1) * 9 + r) * RP + xi] = f.y;
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < kThinMaxW; ++j) {
                const int w = threadIdx.x + j * blockDim.x;
                if (w < total) {
                    const int co = w / (cin * 27), ci = (w / 27) % cin, tap = w % 27;
                    if (ci / 8 == pl) {
                        const int r = tap / 3, dx = tap % 3;
                        const float* xr = xs + ((ci % 8) * 9 + r) * RP + dx;
                        float sacc = 0.f;
                        for (int x = 0; x < N; ++x) sacc = __fmaf_rn(xr[x], gs[x * cout + co], sacc);
                        acc[j] += sacc;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kThinMaxW; ++j) {
        const int w = threadIdx.x + j * blockDim.x;
        if (w < total) partial[(size_t)blockIdx.x * total + w] = acc[j];
    }
}

// Sum of per-block partials: out[i] = sum_b partial[b * stride + i] (fixed order: the result does
// not depend on scheduling).
__global__ void k_sum_partials(const float* partial, int blocks, int n, int stride, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < blocks; ++b) s += partial[(size_t)b * stride + i];
        out[i] = s;
    }
}

// Per-channel sums over the voxels of a planes tensor (bias gradients): block partials [block][C].
__global__ void k_channel_sums(const uint4* G, int planes, long long nvox, float* partial) {
    __shared__ float red[8][32];
    const int C = planes * 8;
    for (int pl = 0; pl < planes; ++pl) {
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
            const uint4 u = G[pl * nvox + v];
            const uint32_t w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 f = unpack_bf16(w4[j]);
                s[2 * j] += f.x;
                s[2 * j + 1] += f.y;
            }
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            float t = s[e];
            for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
            if ((threadIdx.x & 31) == 0) red[e][threadIdx.x >> 5] = t;
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            float t = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
            partial[(size_t)blockIdx.x * C + pl * 8 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

// Input planes of the operator: plane 0 = (p / b, rate * rate_scale, shell, 0, ...); plane 1 stays
// zero (the first convolution reads 16 input channels).
__global__ void k_pack_input(const float* p, const float* rate, Geom g, float inv_b, float rate_scale, uint4* out) {
    const long long nvox = (long long)g.N * g.N * g.N;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % g.N);
        const long long yz = v / g.N;
        const int y = (int)(yz % g.N), z = (int)(yz / g.N);
        const long long pi = x + (long long)g.P * y + g.PN * z;
        const int N = g.N;
        const bool shell = x < 2 || x > N - 3 || y < 2 || y > N - 3 || z < 2 || z > N - 3;
        out[v] = make_uint4(pack_bf16(__fmul_rn(p[pi], inv_b), __fmul_rn(rate[pi], rate_scale)),
                            pack_bf16(shell ? 1.f : 0.f, 0.f), 0u, 0u);
    }
}

// Input planes of the delta form: channel 0 = (p1 - p0) / m (the change of one plain substep,
// normalised by its largest magnitude inside the shell), channel 1 = rate * rate_scale, channel 2
// = the shell mask.
__global__ void k_pack_input_delta(const float* p1, const float* p0, const float* rate, Geom g, float inv_m,
                                   float rate_scale, uint4* out) {
    const long long nvox = (long long)g.N * g.N * g.N;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % g.N);
        const long long yz = v / g.N;
        const int y = (int)(yz % g.N), z = (int)(yz / g.N);
        const long long pi = x + (long long)g.P * y + g.PN * z;
        const int N = g.N;
        const bool shell = x < 2 || x > N - 3 || y < 2 || y > N - 3 || z < 2 || z > N - 3;
        const float d = shell ? 0.f : __fmul_rn(__fsub_rn(p1[pi], p0[pi]), inv_m);
        out[v] = make_uint4(pack_bf16(d, __fmul_rn(rate[pi], rate_scale)), pack_bf16(shell ? 1.f : 0.f, 0.f), 0u, 0u);
    }
}

// max |a - b| over the voxels inside the shell (the values the next substep carries forward), as
// the bits of a non-negative float (ordered like the floats).
__global__ void k_absdiff_max(const float* a, const float* b, Geom g, unsigned* out) {
    const int N = g.N, M = N - 4;
    const long long n = (long long)M * M * M;
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % M) + 2;
        const long long yz = i / M;
        const int y = (int)(yz % M) + 2, z = (int)(yz / M) + 2;
        const long long pi = x + (long long)g.P * y + g.PN * z;
        m = fmaxf(m, fabsf(a[pi] - b[pi]));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// ---------------------------------------------------------------- training: packing, loss, Adam

// Weight images from the fp32 master weights W[cout][cin][27] of one layer (device-side packing, so
// a training step never leaves the GPU): the forward image (input channel 16h + 8kc + e, output
// channel n, as pack_layer) or, with `transpose`, the image of the convolution that maps the
// gradient of the layer's output to the gradient of its input: input channels = the layer's
// outputs, output channels = the layer's inputs, taps mirrored (tap -> 26 - tap).
__global__ void k_pack_w(const float* W, int cin, int cout, int cin8, int nout, int transpose, __nv_bfloat16* img) {
    const int halves = cin8 / 2;
    const int n_img = 27 * halves * 2 * nout * 8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_img; i += gridDim.x * blockDim.x) {
        const int e = i % 8, n = (i / 8) % nout, kc = (i / (8 * nout)) % 2, h = (i / (16 * nout)) % halves;
        const int tap = i / (16 * nout * halves);
        const int k = 16 * h + 8 * kc + e;  // input channel of the packed convolution
        float v = 0.f;
        if (!transpose) {
            if (n < cout && k < cin) v = W[((size_t)n * cin + k) * 27 + tap];
        } else {
            if (k < cout && n < cin) v = W[((size_t)k * cin + n) * 27 + (26 - tap)];
        }
        img[i] = __float2bfloat16_rn(v);
    }
}
__global__ void k_pack_bias(const float* b, int cout, int nout, float* out) {
    const int i = threadIdx.x;
    if (i < nout) out[i] = i < cout ? b[i] : 0.f;
}

// Gradient of the loss L = mean over the voxels inside the shell of ((q - y) / b)^2 with respect to
// the last convolution's output d (q = p + b d inside): 2 (q - y) / (b n), in channel 0 of plane 0
// of the gradient planes; zero on the shell.  Block partial sums of ((q - y) / b)^2 go to `loss`.
__global__ void k_loss_grad(const float* q, const float* y, Geom g, float b, float inv_n, uint4* gd, float* loss) {
    __shared__ float red[32];
    const int N = g.N;
    const long long nvox = (long long)N * N * N;
    float acc = 0.f;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % N);
        const long long yz = v / N;
        const int yy = (int)(yz % N), zz = (int)(yz / N);
        const bool shell = x < 2 || x > N - 3 || yy < 2 || yy > N - 3 || zz < 2 || zz > N - 3;
        float gr = 0.f;
        if (!shell) {
            const long long pi = x + (long long)g.P * yy + g.PN * zz;
            const float e = (q[pi] - y[pi]) / b;
            acc = __fmaf_rn(e, e, acc);
            gr = 2.f * e * inv_n;
        }
        gd[v] = make_uint4(pack_bf16(gr, 0.f), 0u, 0u, 0u);
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        loss[blockIdx.x] = t;
    }
}

// Sum of squares of the gradient (for clipping by its global norm): one block.
__global__ void k_sumsq(const float* g, long long n, float* out) {
    __shared__ float red[32];
    float acc = 0.f;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) acc = __fmaf_rn(g[i], g[i], acc);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *out = t;
    }
}

// Adam (Kingma & Ba, ICLR 2015) with bias correction, on the gradient scaled to global norm
// <= clip: m = b1 m + (1 - b1) g; v = b2 v + (1 - b2) g^2; w -= lr (m / bc1) / (sqrt(v / bc2) + eps).
__global__ void k_adam(float* w, const float* g, float* m, float* v, long long n, const float* sumsq, float clip,
                       float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const float norm = sqrtf(*sumsq);
    const float sc = norm > clip ? clip / norm : 1.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] * sc;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// Layer table: input planes, output channels (padded), mode.
struct LayerShape {
    int cin, cout, cin8, nout;
};
constexpr LayerShape kShape[kLayers] = {
    {kInCh, kHidden, 2, 32},   {kHidden, kHidden, 4, 32}, {kHidden, kHidden, 4, 32}, {kHidden, kHidden, 4, 32},
    {kHidden, kHidden, 4, 32}, {kHidden, kHidden, 4, 32}, {kHidden, kHidden, 4, 32}, {kHidden, kHidden, 4, 32},
    {kHidden, kHidden, 4, 32}, {kHidden, 1, 4, 16}};

}  // namespace

// ---------------------------------------------------------------- host state

// Training state of one substrate's operator (gell_surrogate_train_*): fp32 master weights in the
// layout of gell_surrogate_load, their gradient and Adam moments, the images of the data-gradient
// convolutions, every activation of the forward pass and the gradient planes.
struct TrainState {
    long long count = 0;
    long long off_w[kLayers] = {}, off_b[kLayers] = {};
    float *master = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    float* partial = nullptr;    // block partial sums
    long long partial_n = 0;
    float* zero_bias = nullptr;  // 32 zeros
    float* scal = nullptr;       // [0] gradient sum of squares, [1] loss, [2..] loss partials
    float* hloss = nullptr;      // pinned
    uint8_t* wt[kLayers] = {};   // data-gradient images (layers 1..9)
    uint4* hb[5] = {};
    uint4* tb[4] = {};
    uint4 *gh = nullptr, *gu = nullptr, *gd = nullptr;
    float* tgt = nullptr;        // the plain solver's field after the substeps (pitched)
    CUtensorMap mh[5], mt[4], mgd, mgh, mgu, mgh_g, mgu_g;
    int step = 0;
};

struct SurrogateState {
    int substeps = 0;
    float rate_scale = 0.f, threshold = 0.f;
    // input channel 0: 0 = the field p / b; 1 = the change of one plain substep, (L(p) - p) / m with
    // m = its largest magnitude inside the shell, and the output scaled by m instead of b
    int input_kind = 0;
    float* p0 = nullptr;        // field before the step (pitched), delta input
    uint8_t* w[kLayers] = {};   // packed weight images
    float* bias[kLayers] = {};  // padded to the layer's NOUT
    uint4* in = nullptr;        // 2 planes
    uint4* h = nullptr;         // 4 planes
    uint4* t = nullptr;         // 4 planes
    float* ph = nullptr;        // surrogate output field (pitched)
    float* backup = nullptr;    // field before the step (pitched)
    unsigned* dmax = nullptr;   // judge scratch
    unsigned* hmax = nullptr;   // pinned host copy
    CUtensorMap map_in, map_h, map_t;
    struct TrainState* train = nullptr;
};

void surrogate_free(gell_ctx* c) {
    for (auto*& s : c->sur) {
        if (!s) continue;
        for (int l = 0; l < kLayers; ++l) {
            if (s->w[l]) cudaFree(s->w[l]);
            if (s->bias[l]) cudaFree(s->bias[l]);
        }
        for (void* p : {(void*)s->in, (void*)s->h, (void*)s->t, (void*)s->ph, (void*)s->backup, (void*)s->dmax,
                        (void*)s->p0})
            if (p) cudaFree(p);
        if (s->hmax) cudaFreeHost(s->hmax);
        if (TrainState* t = s->train) {
            for (void* p : {(void*)t->master, (void*)t->grad, (void*)t->m, (void*)t->v, (void*)t->partial,
                            (void*)t->zero_bias, (void*)t->scal, (void*)t->gh, (void*)t->gu, (void*)t->gd, (void*)t->tgt})
                if (p) cudaFree(p);
            for (auto* p : t->wt) if (p) cudaFree(p);
            for (auto* p : t->hb) if (p) cudaFree(p);
            for (auto* p : t->tb) if (p) cudaFree(p);
            if (t->hloss) cudaFreeHost(t->hloss);
            delete t;
        }
        delete s;
        s = nullptr;
    }
}

static gell_status plane_map(gell_ctx* c, CUtensorMap* m, void* base, int planes, int box_x = kRunVox) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(c, GELL_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t N = (cuuint64_t)c->g.N;
    const cuuint64_t dims[5] = {8, N, N, N, (cuuint64_t)planes};
    const cuuint64_t strides[4] = {16, 16 * N, 16 * N * N, 16 * N * N * N};
    const cuuint32_t box[5] = {8, (cuuint32_t)box_x, 1, 1, (cuuint32_t)planes};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, GELL_ERR_CUDA, "cuTensorMapEncodeTiled (planes) failed (" + std::to_string((int)r) + ")");
    return GELL_OK;
}

// Pack one layer's fp32 weights W[cout][cin][3][3][3] (PyTorch conv3d order, kz kz ky kx = dz dy dx
// + 1) into the shared-memory image: block (tap, half) holds [kc][n][8] with input channel
// 16*half + 8*kc + e and output channel n; padding channels are zero.
static void pack_layer(const float* W, const LayerShape& s, std::vector<uint16_t>& img) {
    const int halves = s.cin8 / 2;
    img.assign((size_t)27 * halves * 2 * s.nout * 8, 0);
    auto bf = [](float f) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)0x7fc0u;
        u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest even
        return (uint16_t)(u >> 16);
    };
    for (int tap = 0; tap < 27; ++tap)
        for (int h = 0; h < halves; ++h)
            for (int kc = 0; kc < 2; ++kc)
                for (int n = 0; n < s.nout; ++n)
                    for (int e = 0; e < 8; ++e) {
                        const int ci = 16 * h + 8 * kc + e;
                        float v = 0.f;
                        if (n < s.cout && ci < s.cin) v = W[((size_t)n * s.cin + ci) * 27 + tap];
                        img[((((size_t)tap * halves + h) * 2 + kc) * s.nout + n) * 8 + e] = bf(v);
                    }
}

template <int CIN8, int NOUT, int MODE>
static gell_status launch_conv(gell_ctx* c, const char* name, const CUtensorMap& in, const uint8_t* w, const float* bias,
                               uint4* out, const uint4* res, const uint4* aux, float* fout, const float* fin, float scale,
                               float bval) {
    using L = ConvSmem<CIN8, NOUT>;
    using R = RingSmem<CIN8, NOUT>;
    // the shared-memory opt-in is a per-device attribute; setting it is cheap, so every launch does
    if (c->conv_ring)
        GELL_CUDA(c, cudaFuncSetAttribute(k_conv3_ring<CIN8, NOUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          R::kBytes));
    else
        GELL_CUDA(c, cudaFuncSetAttribute(k_conv3<CIN8, NOUT, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          L::kBytes));
    ConvArgs a{};
    a.in = in;
    a.w = w;
    a.bias = bias;
    a.out = out;
    a.res = res;
    a.aux = aux;
    a.field_out = fout;
    a.field_in = fin;
    a.N = c->g.N;
    a.P = c->g.P;
    a.PN = c->g.PN;
    a.nvox = c->nvox;
    a.tiles_x = (c->g.N + kTileM - 1) / kTileM;
    a.tiles = (long long)a.tiles_x * c->g.N * c->g.N;
    a.scale = scale;
    a.bval = bval;
    a.err = c->dev_err;
    int sms = 0;
    GELL_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    if (c->conv_ring) {
        const long long units = (long long)a.tiles_x * ((c->g.N + kUnitY - 1) / kUnitY) * c->g.N;
        const int grid = (int)(units < sms ? units : sms);
        GELL_KERNEL(c, name, (k_conv3_ring<CIN8, NOUT, MODE><<<grid, 192, R::kBytes, c->stream>>>(a)));
    } else {
        const int grid = (int)(a.tiles < sms ? a.tiles : sms);
        GELL_KERNEL(c, name, (k_conv3<CIN8, NOUT, MODE><<<grid, 192, L::kBytes, c->stream>>>(a)));
    }
    return GELL_OK;
}

// The input packing and the first `layers` convolutions of one inference of substrate `sub`:
//   layer 0        h  = relu(conv_in(input))
//   layer 2k+1     t  = relu(conv_a(h))          (k = 0..3)
//   layer 2k+2     h += conv_b(t)
//   layer 9        S->ph = p + b * conv_out(h) inside the shell, b on it
// The delta form's input planes: one plain substep from the field p0 (kept in S->p0), the largest
// change m inside the shell (read back to the host), the planes packed from (L(p0) - p0) / m, and
// the field put back to p0.  *m_out = m.
static gell_status delta_input(gell_ctx* c, int sub, SurrogateState* S, float* m_out) {
    Substrate& Su = c->subs[sub];
    const size_t fb = (size_t)c->nvox_p * 4;
    GELL_CUDA(c, cudaMemcpyAsync(S->p0, Su.p, fb, cudaMemcpyDeviceToDevice, c->stream));
    gell_status st = lod_solver(c, sub, 1);
    if (st != GELL_OK) return st;
    GELL_CUDA(c, cudaMemsetAsync(S->dmax, 0, 4, c->stream));
    GELL_KERNEL(c, "k_absdiff_max", (k_absdiff_max<<<148 * 8, 256, 0, c->stream>>>(Su.p, S->p0, c->g, S->dmax)));
    GELL_CUDA(c, cudaMemcpyAsync(S->hmax, S->dmax, 4, cudaMemcpyDeviceToHost, c->stream));
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    float m;
    std::memcpy(&m, S->hmax, 4);
    const int pb = blocks_for(c->nvox, 256);
    GELL_KERNEL(c, "k_pack_input",
                (k_pack_input_delta<<<pb < 148 * 16 ? pb : 148 * 16, 256, 0, c->stream>>>(
                    Su.p, S->p0, Su.rate, c->g, m > 0.f ? 1.f / m : 0.f, S->rate_scale, S->in)));
    GELL_CUDA(c, cudaMemcpyAsync(Su.p, S->p0, fb, cudaMemcpyDeviceToDevice, c->stream));
    *m_out = m;
    return GELL_OK;
}

static gell_status run_layers(gell_ctx* c, int sub, SurrogateState* S, int layers) {
    Substrate& Su = c->subs[sub];
    const float b = Su.s.boundary;
    const int pb = blocks_for(c->nvox, 256);
    float scale = b;  // the output's scale: b, or m in the delta form
    if (S->input_kind == 1) {
        if (gell_status sd = delta_input(c, sub, S, &scale)) return sd;
    } else {
        GELL_KERNEL(c, "k_pack_input",
                    (k_pack_input<<<pb < 148 * 16 ? pb : 148 * 16, 256, 0, c->stream>>>(Su.p, Su.rate, c->g, 1.f / b,
                                                                                     S->rate_scale, S->in)));
    }
    gell_status st = GELL_OK;
    for (int l = 0; l < layers && st == GELL_OK; ++l) {
        const uint8_t* w = S->w[l];
        const float* bi = S->bias[l];
        if (l == 0)
            st = launch_conv<2, 32, kRelu>(c, "k_conv3_in", S->map_in, w, bi, S->h, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f);
        else if (l == kLayers - 1)
            st = launch_conv<4, 16, kField>(c, "k_conv3_out", S->map_h, w, bi, nullptr, nullptr, nullptr, S->ph, Su.p, scale, b);
        else if (l & 1)
            st = launch_conv<4, 32, kRelu>(c, "k_conv3_hidden", S->map_h, w, bi, S->t, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f);
        else
            st = launch_conv<4, 32, kResidual>(c, "k_conv3_hidden", S->map_t, w, bi, S->h, S->h, nullptr, nullptr, nullptr, 0.f, 0.f);
    }
    return st;
}
static gell_status infer(gell_ctx* c, int sub, SurrogateState* S) { return run_layers(c, sub, S, kLayers); }

// Shapes of the data-gradient convolution of layer l: input planes (the layer's outputs, padded to
// 16 channels) and outputs (the layer's inputs).
static int dgrad_cin8(int l) { return kShape[l].cout <= 16 ? 2 : 4; }
static int dgrad_nout(int l) { return kShape[l].cin <= 16 ? 16 : 32; }

static gell_status repack(gell_ctx* c, SurrogateState* S) {
    TrainState* T = S->train;
    for (int l = 0; l < kLayers; ++l) {
        const LayerShape& sh = kShape[l];
        GELL_KERNEL(c, "k_pack_w", (k_pack_w<<<64, 256, 0, c->stream>>>(T->master + T->off_w[l], sh.cin, sh.cout, sh.cin8,
                                                                         sh.nout, 0, (__nv_bfloat16*)S->w[l])));
        GELL_KERNEL(c, "k_pack_bias", (k_pack_bias<<<1, 32, 0, c->stream>>>(T->master + T->off_b[l], sh.cout, sh.nout, S->bias[l])));
        if (l >= 1)
            GELL_KERNEL(c, "k_pack_w", (k_pack_w<<<64, 256, 0, c->stream>>>(T->master + T->off_w[l], sh.cin, sh.cout,
                                                                             dgrad_cin8(l), dgrad_nout(l), 1,
                                                                             (__nv_bfloat16*)T->wt[l])));
    }
    return GELL_OK;
}

static int thin_blocks() { return 148 * 4; }

// Weight gradient of layer l into T->grad (the layer's block): tcgen05 for the 32 -> 32 layers,
// CUDA cores for the thin first and last layers; bias gradient = per-channel sums of G.
static gell_status wgrad_layer(gell_ctx* c, SurrogateState* S, int l, const CUtensorMap* xmap, const uint4* X,
                               const CUtensorMap* gmap, const uint4* G, int gplanes) {
    TrainState* T = S->train;
    const LayerShape& sh = kShape[l];
    const int N = c->g.N;
    const int nw = sh.cout * sh.cin * 27;
    if (sh.cin == kHidden && sh.cout == kHidden) {
        WgradArgs a{};
        a.x = *xmap;
        a.g = *gmap;
        a.partial = T->partial;
        a.N = N;
        a.tiles_x = (N + kTileM - 1) / kTileM;
        a.tiles = (long long)a.tiles_x * N * N;
        a.err = c->dev_err;
        int sms = 0;
        GELL_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        const int grid = (int)(a.tiles < sms ? a.tiles : sms);
        GELL_CUDA(c, cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgBytes));
        GELL_KERNEL(c, "k_wgrad", (k_wgrad<<<grid, 192, kWgBytes, c->stream>>>(a)));
        GELL_KERNEL(c, "k_sum_partials", (k_sum_partials<<<(nw + 255) / 256, 256, 0, c->stream>>>(T->partial, grid, nw, nw,
                                                                                                  T->grad + T->off_w[l])));
    } else {
        const int smem = (8 * 9 * thin_pitch(N) + N * sh.cout) * 4;
        GELL_CUDA(c, cudaFuncSetAttribute(k_wgrad_thin, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        GELL_KERNEL(c, "k_wgrad_thin", (k_wgrad_thin<<<thin_blocks(), 256, smem, c->stream>>>(X, sh.cin, G, sh.cout, N,
                                                                                                c->nvox, T->partial)));
        GELL_KERNEL(c, "k_sum_partials", (k_sum_partials<<<(nw + 255) / 256, 256, 0, c->stream>>>(
                                              T->partial, thin_blocks(), nw, nw, T->grad + T->off_w[l])));
    }
    const int C = gplanes * 8;
    GELL_KERNEL(c, "k_channel_sums", (k_channel_sums<<<thin_blocks(), 256, 0, c->stream>>>(G, gplanes, c->nvox, T->partial)));
    GELL_KERNEL(c, "k_sum_partials", (k_sum_partials<<<1, 32, 0, c->stream>>>(T->partial, thin_blocks(), sh.cout, C,
                                                                              T->grad + T->off_b[l])));
    return GELL_OK;
}

// One training pair: the plain solver advances the field by the operator's substeps (the target),
// the operator runs from the field before them with every activation kept, the loss gradient goes
// back through the ten layers (data gradients on tcgen05, weight gradients as above), Adam updates
// the master weights, the images are repacked, and the field is left at the target.
static gell_status train_pair(gell_ctx* c, int sub, SurrogateState* S, float lr, float* loss_out) {
    TrainState* T = S->train;
    Substrate& Su = c->subs[sub];
    const float b = Su.s.boundary;
    const size_t fb = (size_t)c->nvox_p * 4;
    GELL_CUDA(c, cudaMemcpyAsync(S->backup, Su.p, fb, cudaMemcpyDeviceToDevice, c->stream));
    // delta form: the input planes from one plain substep first (the field is put back), the output
    // and the loss in units of m, the substep's largest change (a fixed point, m = 0, has q = p = y)
    float scale = b, loss_unit = b;
    gell_status st = GELL_OK;
    if (S->input_kind == 1) {
        if ((st = delta_input(c, sub, S, &scale)) != GELL_OK) return st;
        loss_unit = scale > 0.f ? scale : b;
    }
    st = lod_solver(c, sub, S->substeps);
    if (st != GELL_OK) return st;
    GELL_CUDA(c, cudaMemcpyAsync(T->tgt, Su.p, fb, cudaMemcpyDeviceToDevice, c->stream));
    GELL_CUDA(c, cudaMemcpyAsync(Su.p, S->backup, fb, cudaMemcpyDeviceToDevice, c->stream));

    // forward, every activation kept
    const int pb = blocks_for(c->nvox, 256);
    if (S->input_kind == 0)
        GELL_KERNEL(c, "k_pack_input", (k_pack_input<<<pb < 148 * 16 ? pb : 148 * 16, 256, 0, c->stream>>>(
                                            Su.p, Su.rate, c->g, 1.f / b, S->rate_scale, S->in)));
    st = launch_conv<2, 32, kRelu>(c, "k_conv3_in", S->map_in, S->w[0], S->bias[0], T->hb[0], nullptr, nullptr, nullptr,
                                   nullptr, 0.f, 0.f);
    for (int k = 0; k < 4 && st == GELL_OK; ++k) {
        st = launch_conv<4, 32, kRelu>(c, "k_conv3_hidden", T->mh[k], S->w[2 * k + 1], S->bias[2 * k + 1], T->tb[k],
                                       nullptr, nullptr, nullptr, nullptr, 0.f, 0.f);
        if (st == GELL_OK)
            st = launch_conv<4, 32, kResidual>(c, "k_conv3_hidden", T->mt[k], S->w[2 * k + 2], S->bias[2 * k + 2],
                                               T->hb[k + 1], T->hb[k], nullptr, nullptr, nullptr, 0.f, 0.f);
    }
    if (st == GELL_OK)
        st = launch_conv<4, 16, kField>(c, "k_conv3_out", T->mh[4], S->w[9], S->bias[9], nullptr, nullptr, nullptr, S->ph,
                                        Su.p, scale, b);
    if (st != GELL_OK) return st;

    // loss and its gradient
    const long long inner = (long long)(c->g.N - 4) * (c->g.N - 4) * (c->g.N - 4);
    const int lb = 148 * 8;
    GELL_KERNEL(c, "k_loss_grad", (k_loss_grad<<<lb, 256, 0, c->stream>>>(S->ph, T->tgt, c->g, loss_unit, 1.f / (float)inner, T->gd,
                                                                          T->scal + 2)));
    GELL_KERNEL(c, "k_sum_partials", (k_sum_partials<<<1, 32, 0, c->stream>>>(T->scal + 2, lb, 1, 1, T->scal + 1)));

    // backward
    if ((st = wgrad_layer(c, S, 9, nullptr, T->hb[4], nullptr, T->gd, 1)) != GELL_OK) return st;
    st = launch_conv<2, 32, kLinear>(c, "k_conv3_dgrad", T->mgd, T->wt[9], T->zero_bias, T->gh, nullptr, nullptr, nullptr,
                                     nullptr, 0.f, 0.f);
    for (int k = 3; k >= 0 && st == GELL_OK; --k) {
        if ((st = wgrad_layer(c, S, 2 * k + 2, &T->mt[k], T->tb[k], &T->mgh_g, T->gh, 4)) != GELL_OK) return st;
        st = launch_conv<4, 32, kMask>(c, "k_conv3_dgrad", T->mgh, T->wt[2 * k + 2], T->zero_bias, T->gu, nullptr,
                                       T->tb[k], nullptr, nullptr, 0.f, 0.f);
        if (st != GELL_OK) return st;
        if ((st = wgrad_layer(c, S, 2 * k + 1, &T->mh[k], T->hb[k], &T->mgu_g, T->gu, 4)) != GELL_OK) return st;
        if (k > 0)
            st = launch_conv<4, 32, kResidual>(c, "k_conv3_dgrad", T->mgu, T->wt[2 * k + 1], T->zero_bias, T->gh, T->gh,
                                               nullptr, nullptr, nullptr, 0.f, 0.f);
        else
            st = launch_conv<4, 32, kResMask>(c, "k_conv3_dgrad", T->mgu, T->wt[1], T->zero_bias, T->gh, T->gh, T->hb[0],
                                              nullptr, nullptr, 0.f, 0.f);
    }
    if (st != GELL_OK) return st;
    if ((st = wgrad_layer(c, S, 0, nullptr, S->in, nullptr, T->gh, 4)) != GELL_OK) return st;

    // Adam on the clipped gradient, new images
    GELL_KERNEL(c, "k_sumsq", (k_sumsq<<<1, 1024, 0, c->stream>>>(T->grad, T->count, T->scal)));
    T->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)T->step), bc2 = 1.f - powf(b2, (float)T->step);
    GELL_KERNEL(c, "k_adam", (k_adam<<<64, 256, 0, c->stream>>>(T->master, T->grad, T->m, T->v, T->count, T->scal, 1.f, lr,
                                                                b1, b2, 1e-8f, bc1, bc2)));
    if ((st = repack(c, S)) != GELL_OK) return st;
    GELL_CUDA(c, cudaMemcpyAsync(Su.p, T->tgt, fb, cudaMemcpyDeviceToDevice, c->stream));
    if (loss_out) {
        GELL_CUDA(c, cudaMemcpyAsync(T->hloss, T->scal + 1, 4, cudaMemcpyDeviceToHost, c->stream));
        GELL_CUDA(c, cudaStreamSynchronize(c->stream));
        *loss_out = *T->hloss / (float)inner;
    }
    return GELL_OK;
}

}  // namespace gell

using namespace gell;

static long long weight_count() {
    long long n = 0;
    for (const auto& s : kShape) n += (long long)s.cout * s.cin * 27 + s.cout;
    return n;
}

extern "C" {

long long gell_surrogate_weight_count(void) { return weight_count(); }

gell_status gell_surrogate_load(gell_ctx* c, int sub, const float* weights, long long count, int substeps,
                                float rate_scale, float threshold) {
    GELL_RANGE("gell_surrogate_load");
    if (!c || !weights || sub < 0 || sub >= (int)c->subs.size() || substeps < 1) return GELL_ERR_INVALID_ARG;
    if (count != weight_count()) return fail(c, GELL_ERR_INVALID_ARG, "surrogate weight count does not match the operator");
    if (!(c->subs[sub].s.boundary != 0.f)) return fail(c, GELL_ERR_UNSUPPORTED, "the surrogate scales by the boundary value, which is 0");
    if (c->g.N < 8 || c->g.N > 1023) return fail(c, GELL_ERR_UNSUPPORTED, "grid edge outside the surrogate's range");
    SurrogateState* S = c->sur[sub];  // reloading keeps the buffers and replaces the weights
    const bool fresh = S == nullptr;
    if (fresh) S = new SurrogateState();
    S->substeps = substeps;
    S->rate_scale = rate_scale;
    S->threshold = threshold;
    S->input_kind = c->sur_input;
    const float* W = weights;
    for (int l = 0; l < kLayers; ++l) {
        const LayerShape& s = kShape[l];
        std::vector<uint16_t> img;
        pack_layer(W, s, img);
        W += (size_t)s.cout * s.cin * 27;
        std::vector<float> bias(s.nout, 0.f);
        for (int n = 0; n < s.cout; ++n) bias[n] = W[n];
        W += s.cout;
        if (!S->w[l]) {
            c->sur[sub] = S;  // owned by the context from here on (freed with it)
            if (cudaMalloc(&S->w[l], img.size() * 2) != cudaSuccess || cudaMalloc(&S->bias[l], bias.size() * 4) != cudaSuccess)
                return fail(c, GELL_ERR_ALLOC, "surrogate weights");
        }
        // copies on the context's stream (a non-blocking stream: a plain cudaMemcpy would not be
        // ordered before the kernels that read these buffers), finished before the vectors go away
        GELL_CUDA(c, cudaMemcpyAsync(S->w[l], img.data(), img.size() * 2, cudaMemcpyHostToDevice, c->stream));
        GELL_CUDA(c, cudaMemcpyAsync(S->bias[l], bias.data(), bias.size() * 4, cudaMemcpyHostToDevice, c->stream));
        GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    c->sur[sub] = S;
    if (fresh) {
        const size_t plane = (size_t)c->nvox * 16, field = (size_t)c->nvox_p * 4;
        if (cudaMalloc(&S->in, 2 * plane) != cudaSuccess || cudaMalloc(&S->h, 4 * plane) != cudaSuccess ||
            cudaMalloc(&S->t, 4 * plane) != cudaSuccess || cudaMalloc(&S->ph, field) != cudaSuccess ||
            cudaMalloc(&S->backup, field) != cudaSuccess || cudaMalloc(&S->dmax, 4) != cudaSuccess ||
            cudaMallocHost(&S->hmax, 4) != cudaSuccess)
            return fail(c, GELL_ERR_ALLOC, "surrogate activations (10 planes of 16 bytes per voxel)");
        GELL_CUDA(c, cudaMemsetAsync(S->in, 0, 2 * plane, c->stream));
        gell_status st = GELL_OK;
        if (cudaMalloc(&S->p0, field) != cudaSuccess) return fail(c, GELL_ERR_ALLOC, "surrogate field copy");
        st = plane_map(c, &S->map_in, S->in, 2);
        if (st == GELL_OK) st = plane_map(c, &S->map_h, S->h, 4);
        if (st == GELL_OK) st = plane_map(c, &S->map_t, S->t, 4);
        if (st != GELL_OK) return st;
    }
    return GELL_OK;
}

gell_status gell_surrogate_infer(gell_ctx* c, int sub) {
    GELL_RANGE("gell_surrogate_infer");
    if (!c || sub < 0 || sub >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    SurrogateState* S = c->sur[sub];
    if (!S) return fail(c, GELL_ERR_INVALID_ARG, "no surrogate loaded for this substrate");
    gell_status st = infer(c, sub, S);
    if (st != GELL_OK) return st;
    GELL_CUDA(c, cudaMemcpyAsync(c->subs[sub].p, S->ph, (size_t)c->nvox_p * 4, cudaMemcpyDeviceToDevice, c->stream));
    return GELL_OK;
}

gell_status gell_lod_surrogate(gell_ctx* c, int sub, int* accepted, float* residual) {
    GELL_RANGE("gell_lod_surrogate");
    if (!c || sub < 0 || sub >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    SurrogateState* S = c->sur[sub];
    if (!S) return fail(c, GELL_ERR_INVALID_ARG, "no surrogate loaded for this substrate");
    Substrate& Su = c->subs[sub];
    const size_t fb = (size_t)c->nvox_p * 4;
    GELL_CUDA(c, cudaMemcpyAsync(S->backup, Su.p, fb, cudaMemcpyDeviceToDevice, c->stream));
    gell_status st = infer(c, sub, S);
    if (st != GELL_OK) return st;
    // judge: one plain substep from the surrogate's field; a field on the solver's trajectory moves
    // little in one substep
    GELL_CUDA(c, cudaMemcpyAsync(Su.p, S->ph, fb, cudaMemcpyDeviceToDevice, c->stream));
    st = lod_solver(c, sub, 1);
    if (st != GELL_OK) return st;
    GELL_CUDA(c, cudaMemsetAsync(S->dmax, 0, 4, c->stream));
    GELL_KERNEL(c, "k_absdiff_max", (k_absdiff_max<<<148 * 8, 256, 0, c->stream>>>(Su.p, S->ph, c->g, S->dmax)));
    GELL_CUDA(c, cudaMemcpyAsync(S->hmax, S->dmax, 4, cudaMemcpyDeviceToHost, c->stream));
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    float r;
    std::memcpy(&r, S->hmax, 4);
    r /= Su.s.boundary;
    if (residual) *residual = r;
    const bool ok = r <= S->threshold;
    if (accepted) *accepted = ok ? 1 : 0;
    if (ok) {
        GELL_CUDA(c, cudaMemcpyAsync(Su.p, S->ph, fb, cudaMemcpyDeviceToDevice, c->stream));
        return GELL_OK;
    }
    GELL_CUDA(c, cudaMemcpyAsync(Su.p, S->backup, fb, cudaMemcpyDeviceToDevice, c->stream));
    return lod_solver(c, sub, S->substeps);
}

gell_status gell_surrogate_train_init(gell_ctx* c, int sub, const float* weights, long long count, int substeps,
                                      float rate_scale) {
    GELL_RANGE("gell_surrogate_train_init");
    gell_status st = gell_surrogate_load(c, sub, weights, count, substeps, rate_scale, 0.f);
    if (st != GELL_OK) return st;
    SurrogateState* S = c->sur[sub];
    if (!S->train) {
        TrainState* T = new TrainState();
        S->train = T;
        T->count = count;
        long long off = 0;
        for (int l = 0; l < kLayers; ++l) {
            T->off_w[l] = off;
            off += (long long)kShape[l].cout * kShape[l].cin * 27;
            T->off_b[l] = off;
            off += kShape[l].cout;
        }
        const size_t plane = (size_t)c->nvox * 16, field = (size_t)c->nvox_p * 4;
        T->partial_n = 148LL * 32 * 32 * 27;
        bool ok = cudaMalloc(&T->master, count * 4) == cudaSuccess && cudaMalloc(&T->grad, count * 4) == cudaSuccess &&
                  cudaMalloc(&T->m, count * 4) == cudaSuccess && cudaMalloc(&T->v, count * 4) == cudaSuccess &&
                  cudaMalloc(&T->partial, T->partial_n * 4) == cudaSuccess &&
                  cudaMalloc(&T->zero_bias, 32 * 4) == cudaSuccess &&
                  cudaMalloc(&T->scal, (2 + 148 * 8) * 4) == cudaSuccess && cudaMallocHost(&T->hloss, 4) == cudaSuccess &&
                  cudaMalloc(&T->gh, 4 * plane) == cudaSuccess && cudaMalloc(&T->gu, 4 * plane) == cudaSuccess &&
                  cudaMalloc(&T->gd, 2 * plane) == cudaSuccess && cudaMalloc(&T->tgt, field) == cudaSuccess;
        for (int k = 0; ok && k < 5; ++k) ok = cudaMalloc(&T->hb[k], 4 * plane) == cudaSuccess;
        for (int k = 0; ok && k < 4; ++k) ok = cudaMalloc(&T->tb[k], 4 * plane) == cudaSuccess;
        for (int l = 1; ok && l < kLayers; ++l)
            ok = cudaMalloc(&T->wt[l], (size_t)27 * (dgrad_cin8(l) / 2) * 2 * dgrad_nout(l) * 8 * 2) == cudaSuccess;
        if (!ok) return fail(c, GELL_ERR_ALLOC, "surrogate training buffers (46 planes of 16 bytes per voxel)");
        GELL_CUDA(c, cudaMemsetAsync(T->zero_bias, 0, 32 * 4, c->stream));
        GELL_CUDA(c, cudaMemsetAsync(T->gd, 0, 2 * plane, c->stream));
        for (int k = 0; k < 5 && st == GELL_OK; ++k) st = plane_map(c, &T->mh[k], T->hb[k], 4);
        for (int k = 0; k < 4 && st == GELL_OK; ++k) st = plane_map(c, &T->mt[k], T->tb[k], 4);
        if (st == GELL_OK) st = plane_map(c, &T->mgd, T->gd, 2);
        if (st == GELL_OK) st = plane_map(c, &T->mgh, T->gh, 4);
        if (st == GELL_OK) st = plane_map(c, &T->mgu, T->gu, 4);
        if (st == GELL_OK) st = plane_map(c, &T->mgh_g, T->gh, 4, kTileM);
        if (st == GELL_OK) st = plane_map(c, &T->mgu_g, T->gu, 4, kTileM);
        if (st != GELL_OK) return st;
    }
    TrainState* T = S->train;
    T->step = 0;
    GELL_CUDA(c, cudaMemcpyAsync(T->master, weights, count * 4, cudaMemcpyHostToDevice, c->stream));
    GELL_CUDA(c, cudaMemsetAsync(T->m, 0, count * 4, c->stream));
    GELL_CUDA(c, cudaMemsetAsync(T->v, 0, count * 4, c->stream));
    if ((st = repack(c, S)) != GELL_OK) return st;
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));  // `weights` may go away after the return
    return GELL_OK;
}

gell_status gell_surrogate_train_pair(gell_ctx* c, int sub, float lr, float* loss) {
    GELL_RANGE("gell_surrogate_train_pair");
    if (!c || sub < 0 || sub >= (int)c->subs.size() || !c->sur[sub] || !c->sur[sub]->train) return GELL_ERR_INVALID_ARG;
    return train_pair(c, sub, c->sur[sub], lr, loss);
}

gell_status gell_surrogate_train_read(gell_ctx* c, int sub, int which, float* host, long long count) {
    if (!c || !host || sub < 0 || sub >= (int)c->subs.size() || !c->sur[sub] || !c->sur[sub]->train)
        return GELL_ERR_INVALID_ARG;
    TrainState* T = c->sur[sub]->train;
    if (which == 2) {
        if (count != c->nvox_p) return GELL_ERR_INVALID_ARG;
        GELL_CUDA(c, cudaMemcpyAsync(host, T->tgt, (size_t)count * 4, cudaMemcpyDeviceToHost, c->stream));
    } else {
        if (count != T->count || (which != 0 && which != 1)) return GELL_ERR_INVALID_ARG;
        GELL_CUDA(c, cudaMemcpyAsync(host, which == 0 ? T->master : T->grad, (size_t)count * 4, cudaMemcpyDeviceToHost,
                                     c->stream));
    }
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    return GELL_OK;
}

gell_status gell_surrogate_run_layers(gell_ctx* c, int sub, int layers) {
    if (!c || sub < 0 || sub >= (int)c->subs.size() || layers < 0 || layers > kLayers) return GELL_ERR_INVALID_ARG;
    SurrogateState* S = c->sur[sub];
    if (!S) return fail(c, GELL_ERR_INVALID_ARG, "no surrogate loaded for this substrate");
    return run_layers(c, sub, S, layers);
}

gell_status gell_surrogate_read(gell_ctx* c, int sub, int which, void* host, long long bytes) {
    if (!c || !host || sub < 0 || sub >= (int)c->subs.size() || !c->sur[sub]) return GELL_ERR_INVALID_ARG;
    SurrogateState* S = c->sur[sub];
    const long long plane = c->nvox * 16;
    const void* src = which == 0 ? (const void*)S->in : which == 1 ? (const void*)S->h : which == 2 ? (const void*)S->t
                    : which == 3 ? (const void*)S->ph : nullptr;
    const long long need = which == 0 ? 2 * plane : which == 3 ? c->nvox_p * 4 : 4 * plane;
    if (!src || bytes != need) return GELL_ERR_INVALID_ARG;
    GELL_CUDA(c, cudaMemcpyAsync(host, src, (size_t)bytes, cudaMemcpyDeviceToHost, c->stream));
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    return GELL_OK;
}

}  // extern "C"
