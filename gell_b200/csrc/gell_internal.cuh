// gell_internal.cuh — context, storage layout and device helpers shared by the gell_b200 kernels.
//
// HBM layout
//   cells    structure of arrays, two buffers per field (a gather writes the other buffer):
//            sign u8, mesh_idx i32, posr float4 (x, y, z, r), force float4, oldforce float4,
//            V, Vf, Vcs, Vns, cell_clock f32, phase i32.  77 bytes per cell per buffer.
//   keys     u32 Morton key + 1 (0 = outside the grid), with u32 payload, two ping-pong buffers
//   bins     int4 per voxel {first sorted index, last sorted index, epoch, 0}; an entry is valid
//            only when its epoch equals the current mechanics step, so nothing is ever cleared
//   fields   per substrate: concentration and uptake rate, x fastest, row pitch P = N rounded up
//            to a multiple of 4 floats (16-byte rows for bulk copies), plane pitch P*N
//   lines    per substrate, one flag word per x-line (y, z) whose uptake is nonzero, and a list of
//            them: the uptake map is zero elsewhere and only listed lines are read or cleared
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/gell.h"

namespace gell {

// ------------------------------------------------------------------ double buffers
template <class T>
struct DBuf {
    T* b[2] = {nullptr, nullptr};
    int c = 0;
    T* cur() const { return b[c]; }
    T* alt() const { return b[c ^ 1]; }
    void swap() { c ^= 1; }
};

struct CellsSoA {
    uint8_t* sign;
    int32_t* mesh;
    float4* posr;
    float4* force;
    float4* oldf;
    float* V;
    float* Vf;
    float* Vcs;
    float* Vns;
    float* clock;
    int32_t* phase;
};

struct Substrate {
    gell_substrate s;
    float* p = nullptr;     // field, pitched
    float* rate = nullptr;  // uptake map, pitched; nonzero only on flagged lines
    float* EF = nullptr;    // device: E[N], F[N], RN(1/F)[N]
    float4* FRS = nullptr;  // device: (F, RN(1/F), s, s*RN(1/F)) per element of 32*ceil(N/32), boundary
                            // elements (0 and >= N-1) as identities (1, 1, 0, 0)
    uint32_t* line_flag = nullptr;  // N*N: x-line (y + z*N) holds uptake
    int* line_list = nullptr;       // flagged lines
    int* line_count = nullptr;      // device: number of flagged lines
    std::vector<float> E, F;
    float side = 0.f;       // E[1]*F[0], the sweeps' off-diagonal (thomas_side)
    // Groups of 32 elements (bit g = elements 32g..32g+31) that lie inside 1..N-2 and whose E and
    // F equal E[N-2], F[N-2] bit for bit: the LU factors of the constant-coefficient line converge
    // within a few dozen elements, so all groups but the first and the last usually qualify.
    uint32_t uniform_groups = 0;
    float conv_R = 0.f;     // RN(1/F[N-2]), the reciprocal of the converged F
    CUtensorMap tmap[3];    // TMA maps of the field for the x, y and z sweeps (32x32 boxes)
};

// Kernel-side view of the geometry.
struct Geom {
    int N;        // voxels per axis
    int P;        // row pitch (floats)
    long long PN; // plane pitch (floats) = P*N
    float len;    // voxel length
};

struct SurrogateState;  // learned substrate surrogate (surrogate.cu)

struct SortScratch {
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* vals[2] = {nullptr, nullptr};
    uint32_t* hist = nullptr;  // digit-major [R][blocks]
    int which = 0;             // buffer holding the sorted output of the last sort
    int bits = 0;              // key bits to sort
};

}  // namespace gell

struct gell_ctx {
    gell_params P{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    gell::Geom g{};
    long long nvox = 0;     // N^3
    long long nvox_p = 0;   // P*N*N
    int cap = 0;
    int n = 0;              // current cell count (host mirror)

    gell::DBuf<uint8_t> sign;
    gell::DBuf<int32_t> mesh;
    gell::DBuf<float4> posr, force, oldf;
    gell::DBuf<float> V, Vf, Vcs, Vns, clock;
    gell::DBuf<int32_t> phase;

    gell::SortScratch sort;
    int4* bins = nullptr;
    int* dev_epoch = nullptr;  // cell-list epoch (device: replayed graphs read the current one)
    bool sorted_valid = false;  // keys/perm describe the current order

    std::vector<gell::Substrate> subs;
    gell::SurrogateState* sur[8] = {};  // per substrate, created by gell_surrogate_load
    bool conv_ring = true;              // GELL_OPT_CONV_RING: the surrogate's convolutions reuse rows along y
    int sur_input = 0;                  // GELL_OPT_SURROGATE_INPUT for surrogates loaded from now on
    bool rate_valid = false;
    bool exact_chain = false;  // GELL_OPT_EXACT_CHAIN
    int sweep_warps = 0;       // GELL_OPT_SWEEP_WARPS (0: as many as shared memory allows)
    int sweep_ring = -1;       // GELL_OPT_SWEEP_RING: -1 auto, 0 line tiles, 1 ring, >= 2 ring of at most that many slots
    bool sweep_l2hint = false;  // GELL_OPT_SWEEP_L2HINT: the ring sweeps' L2 eviction priorities
    int sweep_ring_lag = 0;     // GELL_OPT_SWEEP_RING_LAG: stores in flight per ring warp (0: default)
    int lod_streams = 1;        // GELL_OPT_LOD_STREAMS: a stream per substrate for the LOD substeps
    cudaStream_t sub_stream[8] = {};
    cudaEvent_t sub_join[8] = {};
    cudaEvent_t sub_fork = nullptr;
    bool sweeps_configured = false;  // the sweeps' shared-memory attribute is set on this device
    bool ring_configured = false;    // the same for the ring sweeps

    // gell_run_mechanics: captured graphs of two mechanics steps and what each was captured for
    // (two entries: an odd number of steps flips the double buffers to the other assignment)
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        int n = -1, substeps = -1, nsub = -1;
        uint32_t parity = 0;
        long long launches = 0;  // kernels in one replay
        long long used = 0;
    };
    StepGraph graphs[2];
    long long graph_clock = 0;
    bool stepped = false;  // a mechanics step has run outside a capture (kernel set-up done)

    // PD
    curandState* xorwow = nullptr;
    uint32_t bio_step = 0;
    uint32_t* flags = nullptr;     // cap + 1
    uint32_t* scan_tmp = nullptr;  // block sums
    int* dev_count = nullptr;      // device scalars for counts
    int* dev_err = nullptr;        // device error word (bounded waits)

    gell_cell* staging = nullptr;  // cap AoS records

    // queued host transfers of the cells (gell_cells_import_async / _export_async): a stream of
    // their own, ordered after the last work that used the cells (cells_ev, recorded on `stream`),
    // and waited for (xfer_ev) by the next work that uses them
    cudaStream_t xfer = nullptr;
    cudaEvent_t cells_ev = nullptr, xfer_ev = nullptr;
    bool xfer_pending = false;

    // launch accounting and optional per-kernel event timing
    long long launches = 0;
    bool prof_on = false;
    struct ProfEntry {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<ProfEntry> prof;       // recorded since the last read
    std::vector<cudaEvent_t> ev_pool;  // free events

    std::string err;

    gell::CellsSoA cur() const {
        return {sign.cur(), mesh.cur(), posr.cur(), force.cur(), oldf.cur(), V.cur(),
                Vf.cur(), Vcs.cur(), Vns.cur(), clock.cur(), phase.cur()};
    }
    gell::CellsSoA alt() const {
        return {sign.alt(), mesh.alt(), posr.alt(), force.alt(), oldf.alt(), V.alt(),
                Vf.alt(), Vcs.alt(), Vns.alt(), clock.alt(), phase.alt()};
    }
    void swap_all() {
        sign.swap(); mesh.swap(); posr.swap(); force.swap(); oldf.swap();
        V.swap(); Vf.swap(); Vcs.swap(); Vns.swap(); clock.swap(); phase.swap();
    }
};

namespace gell {

// ------------------------------------------------------------------ error handling
gell_status fail(gell_ctx* c, gell_status s, const std::string& msg);
gell_status cuda_fail(gell_ctx* c, cudaError_t e, const char* where);
#define GELL_CUDA(ctx, call)                                         \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return gell::cuda_fail(ctx, e_, #call); \
    } while (0)
#define GELL_LAUNCH(ctx, what)                                         \
    do {                                                               \
        cudaError_t e_ = cudaGetLastError();                           \
        if (e_ != cudaSuccess) return gell::cuda_fail(ctx, e_, what);  \
    } while (0)

// An NVTX range around an entry point, for timeline tools (header-only NVTX 3: free when no tool
// is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
#define GELL_RANGE(name) gell::NvtxRange gell_range_(name)

// Every kernel launch goes through GELL_KERNEL: it is counted, timed when profiling is on, and
// its launch error is turned into a status.
int prof_begin(gell_ctx* c, const char* name);
void prof_end(gell_ctx* c, int slot);
#define GELL_KERNEL(ctx, name, ...)                     \
    do {                                                \
        int slot_ = gell::prof_begin(ctx, name);        \
        __VA_ARGS__;                                    \
        gell::prof_end(ctx, slot_);                     \
        (ctx)->launches++;                              \
        GELL_LAUNCH(ctx, name);                         \
    } while (0)

// ------------------------------------------------------------------ device helpers

// Bin of a position: (int)(p / len) per axis, a truncating conversion, so positions in
// (-len, 0) fall in bin 0 (include/BasicFunctions.cuh:60-66).
__device__ __forceinline__ int3 find_bin(float x, float y, float z, float len) {
    return make_int3((int)__fdiv_rn(x, len), (int)__fdiv_rn(y, len), (int)__fdiv_rn(z, len));
}
__device__ __forceinline__ bool inside(int i, int j, int k, int N) {
    return !(i < 0 || i >= N || j < 0 || j >= N || k < 0 || k >= N);
}
// Spread the low 10 bits of v to every third bit (bit b -> bit 3b).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// 30-bit Morton code of a bin: x at bits 3b, y at 3b+1, z at 3b+2 (include/BasicFunctions.cuh:111-137).
__device__ __forceinline__ uint32_t morton3(int i, int j, int k) {
    return spread3((uint32_t)i) | (spread3((uint32_t)j) << 1) | (spread3((uint32_t)k) << 2);
}

// Philox4x32-10 (Salmon et al., SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
// Uniform on (0, 1]: top 24 bits plus one, times 2^-24.
__device__ __forceinline__ float u01(uint32_t x) {
    return __fmul_rn((float)((x >> 8) + 1u), 1.0f / 16777216.0f);
}

// ------------------------------------------------------------------ launch helpers
inline int blocks_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b);
}

// ------------------------------------------------------------------ entry points between files
gell_status lod_solver(gell_ctx* c, int sub, int substeps);
// LOD substeps of many contexts at once (ensembles): one launch per sweep axis over every member's
// line tiles.  build allocates the device work list (outside any stream capture); run queues
// `substeps` substeps of every member on `st`.
struct LodBatch;
gell_status lod_batch_build(const std::vector<gell_ctx*>& members, LodBatch** out);
gell_status lod_batch_run(LodBatch* b, cudaStream_t st, int substeps);
void lod_batch_free(LodBatch* b);
gell_status prelod(gell_ctx* c, int sub);
// FM_update and PreLOD of every member of an ensemble, one launch per kernel for all members, on
// `st` (mech.cu); mech_batch_ok says whether the members fit its limits (64 members, 4 substrates)
bool mech_batch_ok(const std::vector<gell_ctx*>& members);
gell_status mech_batch_step(const std::vector<gell_ctx*>& members, cudaStream_t st);
gell_status fm_update(gell_ctx* c);
gell_status selftest_timeout(gell_ctx* c, int polls);
// one mechanics step (fm_update, prelod of all substrates, `substeps` LOD substeps) on c->stream
gell_status one_mechanics_step(gell_ctx* c, int substeps);
// which buffer of each double-buffered cell field is current (a captured step is only valid for
// the assignment it was captured with)
uint32_t buffer_parity(const gell_ctx* c);
// work that uses the cells waits for queued transfers first, and marks where the next one starts
gell_status cells_begin(gell_ctx* c);
gell_status cells_end(gell_ctx* c, gell_status st);
gell_status birth(gell_ctx* c, int* n_out);
gell_status death(gell_ctx* c, int* n_out);
gell_status init_xorwow(gell_ctx* c);
// exclusive scan of flags[0..n) into out[0..n) and the total into *total_dev
gell_status scan_u32(gell_ctx* c, const uint32_t* in, uint32_t* out, int n, int* total_dev);
// stable LSD radix sort of (keys, vals) over the low `bits` bits; result in c->sort.which
gell_status radix_sort(gell_ctx* c, int n, int bits, bool vals_are_iota);
gell_status dump_se(gell_ctx* c, int* host_out);
void surrogate_free(gell_ctx* c);
gell_status selftest_division(gell_ctx* c, long long n, unsigned long long seed, long long* mismatches);
size_t sort_hist_entries(int cap);

}  // namespace gell
