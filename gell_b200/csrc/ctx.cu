// ctx.cu — C ABI of gell_b200 (include/gell.h): context lifetime, cell and field import/export,
// and debug dumps.  The compute entry points live in lod.cu, mech.cu and pd.cu.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cudaTypedefs.h>
#include <new>

#include "gell_internal.cuh"

using namespace gell;

static_assert(sizeof(gell_cell) == 72, "gell_cell must match the reference's 72-byte struct Cell");
static_assert(offsetof(gell_cell, mesh_idx) == 4 && offsetof(gell_cell, pos) == 8 &&
                  offsetof(gell_cell, force) == 20 && offsetof(gell_cell, oldforce) == 32 &&
                  offsetof(gell_cell, r) == 44 && offsetof(gell_cell, V) == 48 &&
                  offsetof(gell_cell, phase) == 64 && offsetof(gell_cell, cell_clock) == 68,
              "gell_cell field offsets");

namespace gell {

gell_status fail(gell_ctx* c, gell_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

gell_status cuda_fail(gell_ctx* c, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (c) c->err = m;
    if (e == cudaErrorMemoryAllocation) return GELL_ERR_ALLOC;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GELL_ERR_NO_DEVICE;
    return GELL_ERR_CUDA;
}

// ------------------------------------------------------------------ AoS <-> SoA kernels

__global__ void k_import(const gell_cell* __restrict__ in, CellsSoA o, int n, Geom g) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gell_cell c = in[i];
    o.sign[i] = c.sign ? 1 : 0;
    o.mesh[i] = c.mesh_idx;
    o.posr[i] = make_float4(c.pos[0], c.pos[1], c.pos[2], c.r);
    o.force[i] = make_float4(c.force[0], c.force[1], c.force[2], 0.f);
    o.oldf[i] = make_float4(c.oldforce[0], c.oldforce[1], c.oldforce[2], 0.f);
    o.V[i] = c.V;
    o.Vf[i] = c.Vf;
    o.Vcs[i] = c.Vcs;
    o.Vns[i] = c.Vns;
    o.phase[i] = c.phase;
    o.clock[i] = c.cell_clock;
}

__global__ void k_export(CellsSoA s, gell_cell* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gell_cell c;
    memset(&c, 0, sizeof c);
    c.sign = s.sign[i];
    c.mesh_idx = s.mesh[i];
    float4 pr = s.posr[i], f = s.force[i], of = s.oldf[i];
    c.pos[0] = pr.x; c.pos[1] = pr.y; c.pos[2] = pr.z; c.r = pr.w;
    c.force[0] = f.x; c.force[1] = f.y; c.force[2] = f.z;
    c.oldforce[0] = of.x; c.oldforce[1] = of.y; c.oldforce[2] = of.z;
    c.V = s.V[i]; c.Vf = s.Vf[i]; c.Vcs = s.Vcs[i]; c.Vns = s.Vns[i];
    c.phase = s.phase[i];
    c.cell_clock = s.clock[i];
    out[i] = c;
}

// dense N^3 <-> pitched field
__global__ void k_field_in(const float* __restrict__ d, float* __restrict__ p, Geom g) {
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nvox = (long long)g.N * g.N * g.N;
    if (v >= nvox) return;
    int x = (int)(v % g.N);
    long long line = v / g.N;
    p[line * g.P + x] = d[v];
}
__global__ void k_field_out(const float* __restrict__ p, float* __restrict__ d, Geom g) {
    long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nvox = (long long)g.N * g.N * g.N;
    if (v >= nvox) return;
    int x = (int)(v % g.N);
    long long line = v / g.N;
    d[v] = p[line * g.P + x];
}
__global__ void k_fill(float* p, long long n, float v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

int prof_begin(gell_ctx* c, const char* name) {
    if (!c->prof_on) return -1;
    cudaEvent_t a, b;
    if (c->ev_pool.size() >= 2) {
        a = c->ev_pool.back(); c->ev_pool.pop_back();
        b = c->ev_pool.back(); c->ev_pool.pop_back();
    } else {
        if (cudaEventCreate(&a) != cudaSuccess) return -1;
        if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -1; }
    }
    cudaEventRecord(a, c->stream);
    c->prof.push_back({name, a, b});
    return (int)c->prof.size() - 1;
}

void prof_end(gell_ctx* c, int slot) {
    if (slot < 0) return;
    cudaEventRecord(c->prof[slot].b, c->stream);
}

}  // namespace gell

// ------------------------------------------------------------------ C ABI

extern "C" {

int gell_abi_version(void) { return GELL_ABI_VERSION; }

const char* gell_status_string(gell_status s) {
    switch (s) {
        case GELL_OK: return "ok";
        case GELL_ERR_INVALID_ARG: return "invalid argument";
        case GELL_ERR_CAPACITY: return "capacity exceeded";
        case GELL_ERR_CUDA: return "CUDA error";
        case GELL_ERR_NO_DEVICE: return "no CUDA device";
        case GELL_ERR_TIMEOUT: return "device wait timed out";
        case GELL_ERR_STATE: return "invalid state";
        case GELL_ERR_UNSUPPORTED: return "unsupported";
        case GELL_ERR_ALLOC: return "allocation failed";
    }
    return "unknown status";
}

const char* gell_last_error(gell_ctx* c) { return c ? c->err.c_str() : "null context"; }

// include/Definitions.h:7-47 (and the literals of include/Cells.cuh, include/RandomFunctions.cuh:21)
void gell_params_default(gell_params* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->voxel_num = 100;
    p->voxel_length = 25.f;
    p->max_cell_num = 2 * 1000 * 1000;
    p->mechanics_dt = 0.1f;
    p->diffusion_dt = 0.01f;
    p->biology_dt = 6.f;
    p->ccca = 0.4f;
    p->cccr = 10.f;
    p->ra_ratio = 1.25;
    p->cc_max_dist = 25.f;
    p->dead_uptake_factor = 0.1f;
    p->default_v = 2494.f;
    p->o2_prolif_thres = 5.f;
    p->o2_prolif_sat = 10.f;
    p->o2_necrosis_thres = 5.f;
    p->o2_necrosis_max = 2.5f;
    p->necrosis_rate = 1.0 / 6.0 / 60.0;
    p->apoptosis_rate = 1.0 / 7.0 / 24.0 / 60.0;
    p->proliferation_rate = 1.0 / 8.5 / 60.0;
    p->duration_pre2post = 13.f * 60;
    p->duration_post2q = 2.5f * 60;
    p->o2_substrate = 0;
    p->rng_mode = GELL_RNG_XORWOW;
    p->mech_mode = GELL_MECH_REFERENCE;
    p->seed = 123;
}

// include/Definitions.h:21-24
void gell_substrate_oxygen(gell_substrate* s) {
    if (!s) return;
    s->boundary = 38.f;
    s->diffusion = 100000.f;
    s->decay = 0.1f;
    s->uptake = -10.f;
    s->init = 38.f;
}

static void free_all(gell_ctx* c) {
    auto f = [](void* p) { if (p) cudaFree(p); };
    for (int b = 0; b < 2; ++b) {
        f(c->sign.b[b]); f(c->mesh.b[b]); f(c->posr.b[b]); f(c->force.b[b]); f(c->oldf.b[b]);
        f(c->V.b[b]); f(c->Vf.b[b]); f(c->Vcs.b[b]); f(c->Vns.b[b]); f(c->clock.b[b]);
        f(c->phase.b[b]);
        f(c->sort.keys[b]); f(c->sort.vals[b]);
    }
    f(c->sort.hist);
    f(c->bins);
    f(c->dev_epoch);
    for (auto& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    surrogate_free(c);
    for (auto& s : c->subs) { f(s.p); f(s.rate); f(s.EF); f(s.FRS); f(s.line_flag); f(s.line_list); f(s.line_count); }
    f(c->xorwow); f(c->flags); f(c->scan_tmp); f(c->dev_count); f(c->dev_err);
    f(c->staging);
    for (auto& p : c->prof) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->xfer) cudaStreamDestroy(c->xfer);
    for (int s = 0; s < 8; ++s) {
        if (c->sub_stream[s]) cudaStreamDestroy(c->sub_stream[s]);
        if (c->sub_join[s]) cudaEventDestroy(c->sub_join[s]);
    }
    if (c->sub_fork) cudaEventDestroy(c->sub_fork);
    if (c->cells_ev) cudaEventDestroy(c->cells_ev);
    if (c->xfer_ev) cudaEventDestroy(c->xfer_ev);
}

gell_status gell_create(const gell_params* params, gell_ctx** out) {
    if (!params || !out) return GELL_ERR_INVALID_ARG;
    *out = nullptr;
    const gell_params& P = *params;
    if (P.voxel_num < 4 || P.voxel_num > 1023) return GELL_ERR_UNSUPPORTED;
    if (!(P.voxel_length > 0.f) || P.max_cell_num < 1 || P.max_cell_num > (1 << 30))
        return GELL_ERR_INVALID_ARG;
    if (P.rng_mode != GELL_RNG_XORWOW && P.rng_mode != GELL_RNG_PHILOX) return GELL_ERR_INVALID_ARG;
    if (P.mech_mode != GELL_MECH_REFERENCE) return GELL_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return GELL_ERR_NO_DEVICE;
    }
    gell_ctx* c = new (std::nothrow) gell_ctx;
    if (!c) return GELL_ERR_ALLOC;
    c->P = P;
    cudaGetDevice(&c->device);
    const int N = P.voxel_num;
    c->g.N = N;
    c->g.P = (N + 3) / 4 * 4;
    c->g.PN = (long long)c->g.P * N;
    c->g.len = P.voxel_length;
    c->nvox = (long long)N * N * N;
    c->nvox_p = (long long)c->g.P * N * N;
    c->cap = P.max_cell_num;
    const size_t cap = (size_t)c->cap;

    gell_status st = GELL_OK;
    auto A = [&](void** p, size_t bytes) {
        if (st != GELL_OK) return;
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) st = cuda_fail(c, e, "cudaMalloc");
    };
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return GELL_ERR_CUDA;
    }
    c->stream = c->own_stream;
    if (cudaStreamCreateWithFlags(&c->xfer, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->cells_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->xfer_ev, cudaEventDisableTiming) != cudaSuccess) {
        free_all(c);
        delete c;
        return GELL_ERR_CUDA;
    }
    for (int b = 0; b < 2; ++b) {
        A((void**)&c->sign.b[b], cap);
        A((void**)&c->mesh.b[b], cap * 4);
        A((void**)&c->posr.b[b], cap * 16);
        A((void**)&c->force.b[b], cap * 16);
        A((void**)&c->oldf.b[b], cap * 16);
        A((void**)&c->V.b[b], cap * 4);
        A((void**)&c->Vf.b[b], cap * 4);
        A((void**)&c->Vcs.b[b], cap * 4);
        A((void**)&c->Vns.b[b], cap * 4);
        A((void**)&c->clock.b[b], cap * 4);
        A((void**)&c->phase.b[b], cap * 4);
        A((void**)&c->sort.keys[b], cap * 4);
        A((void**)&c->sort.vals[b], cap * 4);
    }
    A((void**)&c->sort.hist, sort_hist_entries(c->cap) * 4);
    A((void**)&c->bins, (size_t)c->nvox * sizeof(int4));
    A((void**)&c->dev_epoch, sizeof(int));
    A((void**)&c->flags, (cap + 1) * 4);
    A((void**)&c->scan_tmp, ((cap + 4095) / 4096 + 64) * 4 * 2);
    A((void**)&c->dev_count, 64);
    A((void**)&c->dev_err, 64);
    A((void**)&c->staging, cap * sizeof(gell_cell));
    if (P.rng_mode == GELL_RNG_XORWOW) A((void**)&c->xorwow, cap * sizeof(curandState));
    if (st != GELL_OK) {
        free_all(c);
        delete c;
        return st;
    }
    cudaMemsetAsync(c->bins, 0, (size_t)c->nvox * sizeof(int4), c->stream);
    if (c->dev_epoch) cudaMemsetAsync(c->dev_epoch, 0, sizeof(int), c->stream);
    cudaMemsetAsync(c->dev_err, 0, 64, c->stream);
    if (P.rng_mode == GELL_RNG_XORWOW) {
        st = init_xorwow(c);
        if (st != GELL_OK) {
            free_all(c);
            delete c;
            return st;
        }
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        free_all(c);
        delete c;
        return GELL_ERR_CUDA;
    }
    *out = c;
    return GELL_OK;
}

gell_status gell_destroy(gell_ctx* c) {
    if (!c) return GELL_ERR_INVALID_ARG;
    // queued kernels, replayed graphs and transfers into the caller's host buffers finish first
    cudaStreamSynchronize(c->stream);
    if (c->xfer) cudaStreamSynchronize(c->xfer);
    if (c->own_stream && c->own_stream != c->stream) cudaStreamSynchronize(c->own_stream);
    free_all(c);
    delete c;
    return GELL_OK;
}

gell_status gell_set_stream(gell_ctx* c, void* stream) {
    if (!c) return GELL_ERR_INVALID_ARG;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return GELL_OK;
}

gell_status gell_sync(gell_ctx* c) {
    if (!c) return GELL_ERR_INVALID_ARG;
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->xfer_pending) GELL_CUDA(c, cudaStreamSynchronize(c->xfer));
    int herr = 0;
    GELL_CUDA(c, cudaMemcpy(&herr, c->dev_err, 4, cudaMemcpyDeviceToHost));
    if (herr) {
        // reported once: the word is cleared so that the context can go on
        GELL_CUDA(c, cudaMemsetAsync(c->dev_err, 0, 4, c->stream));  // ordered before the next kernels
        return fail(c, GELL_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(herr) + ")");
    }
    return GELL_OK;
}

// Mesh_struct::Mesh_initialize (include/LODkernel.cuh:239-259): host LU prefactor in float, each
// operation rounded once (host code is compiled with -ffp-contract=off).
static void mesh_init(int N, float len, float D, float decay, float dt, std::vector<float>& E,
                      std::vector<float>& F) {
    E.assign(N, 0.f);
    F.assign(N, 0.f);
    float side = -dt * D / (len * len);
    float corner = 1.f + dt * decay / 3.f - side;
    float diag = corner - side;
    E[0] = 0.f;
    F[0] = corner;
    for (int i = 1; i < N - 1; ++i) {
        E[i] = side / F[i - 1];
        F[i] = diag - E[i] * side;
    }
    E[N - 1] = side / F[N - 2];
    F[N - 1] = corner - E[N - 1] * side;
}

// RN(1/f): the float nearest to 1/f.  The product of two floats is exact in double, so
// |1 - y*f| ranks the candidates exactly; 1/f of a float is never halfway between two floats.
static uint32_t bits_of(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

static float recip_rn(float f) {
    const float y0 = (float)(1.0 / (double)f);
    float best = y0;
    double berr = fabs(1.0 - (double)y0 * (double)f);
    const float cand[2] = {nextafterf(y0, -INFINITY), nextafterf(y0, INFINITY)};
    for (float y : cand) {
        const double e = fabs(1.0 - (double)y * (double)f);
        if (e < berr) { best = y; berr = e; }
    }
    return best;
}

// TMA maps of a pitched field: x boxes [32 lines][32 elements] with the 128-byte swizzle over
// (P, N*N); y boxes [32 elements][32 lines] over (P, N, N); z boxes over (P*N, N).
static gell_status make_tensor_maps(gell_ctx* c, Substrate& sub) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(c, GELL_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t N = (cuuint64_t)c->g.N, P = (cuuint64_t)c->g.P;
    const cuuint32_t box2[2] = {32, 32}, box3[3] = {32, 32, 1}, es[3] = {1, 1, 1};
    const cuuint64_t dx[2] = {P, N * N}, sx[1] = {P * 4};
    const cuuint64_t dy[3] = {P, N, N}, sy[2] = {P * 4, P * N * 4};
    const cuuint64_t dz[2] = {P * N, N}, sz[1] = {P * N * 4};
    CUresult r = encode(&sub.tmap[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, sub.p, dx, sx, box2, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = encode(&sub.tmap[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, sub.p, dy, sy, box3, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = encode(&sub.tmap[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, sub.p, dz, sz, box2, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, GELL_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return GELL_OK;
}

gell_status gell_substrate_add(gell_ctx* c, const gell_substrate* s, int* index_out) {
    if (!c || !s) return GELL_ERR_INVALID_ARG;
    if (c->subs.size() >= 8) return fail(c, GELL_ERR_UNSUPPORTED, "at most 8 substrates");
    Substrate sub;
    sub.s = *s;
    mesh_init(c->g.N, c->g.len, s->diffusion, s->decay, c->P.diffusion_dt, sub.E, sub.F);
    sub.side = sub.E[1] * sub.F[0];
    size_t fb = (size_t)c->nvox_p * 4;
    size_t nl = (size_t)c->g.N * c->g.N;
    cudaError_t e = cudaMalloc(&sub.p, fb);
    if (e == cudaSuccess) e = cudaMalloc(&sub.rate, fb);
    if (e == cudaSuccess) e = cudaMalloc(&sub.EF, (size_t)c->g.N * 3 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sub.line_flag, nl * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sub.line_list, nl * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sub.line_count, 4);
    if (e != cudaSuccess) {
        for (void* q : {(void*)sub.p, (void*)sub.rate, (void*)sub.EF, (void*)sub.line_flag,
                        (void*)sub.line_list, (void*)sub.line_count})
            if (q) cudaFree(q);
        return cuda_fail(c, e, "cudaMalloc(substrate)");
    }
    GELL_CUDA(c, cudaMemsetAsync(sub.line_flag, 0, nl * 4, c->stream));
    GELL_CUDA(c, cudaMemsetAsync(sub.line_count, 0, 4, c->stream));
    {
        gell_status ts = make_tensor_maps(c, sub);
        if (ts != GELL_OK) {
            for (void* q : {(void*)sub.p, (void*)sub.rate, (void*)sub.EF, (void*)sub.line_flag,
                            (void*)sub.line_list, (void*)sub.line_count})
                cudaFree(q);
            return ts;
        }
    }
    // device table: E, F and RN(1/F) for the division on the back-substitution chain
    std::vector<float> efr(3 * (size_t)c->g.N);
    for (int i = 0; i < c->g.N; ++i) {
        efr[i] = sub.E[i];
        efr[c->g.N + i] = sub.F[i];
        efr[2 * c->g.N + i] = recip_rn(sub.F[i]);
    }
    // stream-ordered uploads (the context's stream is non-blocking, so a plain cudaMemcpy would not
    // be ordered before the sweeps that read these), finished before the host vectors go away
    GELL_CUDA(c, cudaMemcpyAsync(sub.EF, efr.data(), efr.size() * 4, cudaMemcpyHostToDevice, c->stream));
    {
        const int Na = (c->g.N + 31) / 32 * 32;
        std::vector<float4> frs((size_t)Na);
        for (int j = 0; j < Na; ++j) {
            const bool in = j >= 1 && j <= c->g.N - 2;
            const float rj = efr[2 * c->g.N + j];
            frs[j] = in ? make_float4(sub.F[j], rj, sub.side, sub.side * rj) : make_float4(1.f, 1.f, 0.f, 0.f);
        }
        const int N = c->g.N;
        const uint32_t eb = bits_of(sub.E[N - 2]), fb2 = bits_of(sub.F[N - 2]);
        for (int g = 0; 32 * g < N; ++g) {
            bool uni = 32 * g >= 1 && 32 * g + 31 <= N - 2;
            for (int j = 32 * g; uni && j < 32 * g + 32; ++j) uni = bits_of(sub.E[j]) == eb && bits_of(sub.F[j]) == fb2;
            if (uni) sub.uniform_groups |= 1u << g;
        }
        sub.conv_R = recip_rn(sub.F[N - 2]);
        GELL_CUDA(c, cudaMalloc(&sub.FRS, frs.size() * sizeof(float4)));
        GELL_CUDA(c, cudaMemcpyAsync(sub.FRS, frs.data(), frs.size() * sizeof(float4), cudaMemcpyHostToDevice,
                                     c->stream));
        GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    GELL_KERNEL(c, "k_fill", k_fill<<<blocks_for(c->nvox_p, 256), 256, 0, c->stream>>>(sub.p, c->nvox_p, s->init));
    GELL_CUDA(c, cudaMemsetAsync(sub.rate, 0, fb, c->stream));
    // the new map must cover the current cells before the next LOD substep
    c->rate_valid = false;
    c->subs.push_back(sub);
    if (index_out) *index_out = (int)c->subs.size() - 1;
    // rate maps of the existing substrates stay; rebuild all on the next prelod
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    // a second substrate: create the substrate streams now, before any graph capture uses them
    if (c->lod_streams && c->subs.size() >= 2) {
        const int s = (int)c->subs.size() - 1;
        if (s < 8 && !c->sub_stream[s]) {
            bool ok = (c->sub_fork || cudaEventCreateWithFlags(&c->sub_fork, cudaEventDisableTiming) == cudaSuccess) &&
                      cudaStreamCreateWithFlags(&c->sub_stream[s], cudaStreamNonBlocking) == cudaSuccess &&
                      cudaEventCreateWithFlags(&c->sub_join[s], cudaEventDisableTiming) == cudaSuccess;
            if (!ok) {
                cudaGetLastError();
                c->lod_streams = 0;  // fall back to one stream
            }
        }
    }
    return GELL_OK;
}

}  // extern "C"

// Work on `stream` that uses the cells first waits for the queued transfers, and afterwards marks
// the point the next queued transfer has to wait for.
namespace gell {
gell_status cells_begin(gell_ctx* c) {
    if (c->xfer_pending) GELL_CUDA(c, cudaStreamWaitEvent(c->stream, c->xfer_ev, 0));
    return GELL_OK;
}
gell_status cells_end(gell_ctx* c, gell_status st) {
    if (st != GELL_OK) return st;
    GELL_CUDA(c, cudaEventRecord(c->cells_ev, c->stream));
    return GELL_OK;
}
}  // namespace gell

extern "C" {

gell_status gell_cells_import(gell_ctx* c, const gell_cell* cells, int n, int on_device) {
    GELL_RANGE("gell_cells_import");
    if (!c || (n > 0 && !cells) || n < 0) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    if (n > c->cap) return fail(c, GELL_ERR_CAPACITY, "more cells than max_cell_num");
    const gell_cell* src = cells;
    if (!on_device && n > 0) {
        GELL_CUDA(c, cudaMemcpyAsync(c->staging, cells, (size_t)n * sizeof(gell_cell),
                                     cudaMemcpyHostToDevice, c->stream));
        src = c->staging;
    }
    if (n > 0) {
        GELL_KERNEL(c, "k_import", k_import<<<blocks_for(n, 256), 256, 0, c->stream>>>(src, c->cur(), n, c->g));
    }
    c->n = n;
    c->sorted_valid = false;
    c->rate_valid = false;
    return cells_end(c, GELL_OK);
}

gell_status gell_cells_export(gell_ctx* c, gell_cell* cells, int capacity, int* n_out, int on_device) {
    GELL_RANGE("gell_cells_export");
    if (!c || (c->n > 0 && !cells)) return GELL_ERR_INVALID_ARG;
    if (capacity < c->n) return fail(c, GELL_ERR_CAPACITY, "export buffer too small");
    if (gell_status b = cells_begin(c)) return b;
    int n = c->n;
    if (n > 0) {
        gell_cell* dst = on_device ? cells : c->staging;
        GELL_KERNEL(c, "k_export", k_export<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->cur(), dst, n));
        if (!on_device) {
            GELL_CUDA(c, cudaMemcpyAsync(cells, c->staging, (size_t)n * sizeof(gell_cell),
                                         cudaMemcpyDeviceToHost, c->stream));
            GELL_CUDA(c, cudaStreamSynchronize(c->stream));
        }
    }
    if (n_out) *n_out = n;
    return cells_end(c, GELL_OK);
}

gell_status gell_cells_import_async(gell_ctx* c, const gell_cell* cells, int n) {
    GELL_RANGE("gell_cells_import_async");
    if (!c || (n > 0 && !cells) || n < 0) return GELL_ERR_INVALID_ARG;
    if (n > c->cap) return fail(c, GELL_ERR_CAPACITY, "more cells than max_cell_num");
    GELL_CUDA(c, cudaStreamWaitEvent(c->xfer, c->cells_ev, 0));
    if (n > 0) {
        GELL_CUDA(c, cudaMemcpyAsync(c->staging, cells, (size_t)n * sizeof(gell_cell), cudaMemcpyHostToDevice,
                                     c->xfer));
        k_import<<<blocks_for(n, 256), 256, 0, c->xfer>>>(c->staging, c->cur(), n, c->g);
        c->launches++;
        GELL_LAUNCH(c, "k_import");
    }
    GELL_CUDA(c, cudaEventRecord(c->xfer_ev, c->xfer));
    c->xfer_pending = true;
    c->n = n;
    c->sorted_valid = false;
    c->rate_valid = false;
    return GELL_OK;
}

gell_status gell_cells_export_async(gell_ctx* c, gell_cell* cells, int capacity, int* n_out) {
    GELL_RANGE("gell_cells_export_async");
    if (!c || (c->n > 0 && !cells)) return GELL_ERR_INVALID_ARG;
    if (capacity < c->n) return fail(c, GELL_ERR_CAPACITY, "export buffer too small");
    const int n = c->n;
    GELL_CUDA(c, cudaStreamWaitEvent(c->xfer, c->cells_ev, 0));
    if (n > 0) {
        k_export<<<blocks_for(n, 256), 256, 0, c->xfer>>>(c->cur(), c->staging, n);
        c->launches++;
        GELL_LAUNCH(c, "k_export");
        GELL_CUDA(c, cudaMemcpyAsync(cells, c->staging, (size_t)n * sizeof(gell_cell), cudaMemcpyDeviceToHost,
                                     c->xfer));
    }
    GELL_CUDA(c, cudaEventRecord(c->xfer_ev, c->xfer));
    c->xfer_pending = true;
    if (n_out) *n_out = n;
    return GELL_OK;
}

gell_status gell_wait_transfers(gell_ctx* c) {
    if (!c) return GELL_ERR_INVALID_ARG;
    return cells_begin(c);
}

gell_status gell_cell_count(gell_ctx* c, int* n_out) {
    if (!c || !n_out) return GELL_ERR_INVALID_ARG;
    *n_out = c->n;
    return GELL_OK;
}

gell_status gell_field_import(gell_ctx* c, int sub, const float* field, int on_device) {
    if (!c || !field || sub < 0 || sub >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    const size_t bytes = (size_t)c->nvox * 4;
    if (on_device) {
        GELL_KERNEL(c, "k_field_in", k_field_in<<<blocks_for(c->nvox, 256), 256, 0, c->stream>>>(field, c->subs[sub].p, c->g));
        return GELL_OK;
    }
    // a dense staging copy on the device, freed in stream order on every path
    float* tmp = nullptr;
    GELL_CUDA(c, cudaMallocAsync((void**)&tmp, bytes, c->stream));
    cudaError_t e = cudaMemcpyAsync(tmp, field, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        k_field_in<<<blocks_for(c->nvox, 256), 256, 0, c->stream>>>(tmp, c->subs[sub].p, c->g);
        c->launches++;
        e = cudaGetLastError();
    }
    cudaFreeAsync(tmp, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "gell_field_import");
    return GELL_OK;
}

gell_status gell_field_export(gell_ctx* c, int sub, float* field, int on_device) {
    if (!c || !field || sub < 0 || sub >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    const size_t bytes = (size_t)c->nvox * 4;
    if (on_device) {
        GELL_KERNEL(c, "k_field_out", k_field_out<<<blocks_for(c->nvox, 256), 256, 0, c->stream>>>(c->subs[sub].p, field, c->g));
        return GELL_OK;
    }
    float* tmp = nullptr;
    GELL_CUDA(c, cudaMallocAsync((void**)&tmp, bytes, c->stream));
    k_field_out<<<blocks_for(c->nvox, 256), 256, 0, c->stream>>>(c->subs[sub].p, tmp, c->g);
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(field, tmp, bytes, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(tmp, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "gell_field_export");
    return GELL_OK;
}

gell_status gell_profile_enable(gell_ctx* c, int on) {
    if (!c) return GELL_ERR_INVALID_ARG;
    c->prof_on = on != 0;
    return GELL_OK;
}

gell_status gell_profile_read(gell_ctx* c, gell_profile_record* out, int max_records, int* count, int reset) {
    if (!c || !count || (max_records > 0 && !out)) return GELL_ERR_INVALID_ARG;
    GELL_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<gell_profile_record> recs;
    for (auto& p : c->prof) {
        float ms = 0.f;
        GELL_CUDA(c, cudaEventElapsedTime(&ms, p.a, p.b));
        gell_profile_record* r = nullptr;
        for (auto& q : recs)
            if (strncmp(q.name, p.name, sizeof q.name) == 0) r = &q;
        if (!r) {
            gell_profile_record z;
            memset(&z, 0, sizeof z);
            strncpy(z.name, p.name, sizeof z.name - 1);
            recs.push_back(z);
            r = &recs.back();
        }
        r->launches += 1;
        r->total_ms += ms;
    }
    *count = (int)recs.size();
    for (int i = 0; i < (int)recs.size() && i < max_records; ++i) out[i] = recs[i];
    if (reset) {
        for (auto& p : c->prof) { c->ev_pool.push_back(p.a); c->ev_pool.push_back(p.b); }
        c->prof.clear();
    }
    return GELL_OK;
}

gell_status gell_selftest_division(gell_ctx* c, int64_t samples, uint64_t seed, int64_t* mismatches) {
    if (!c || !mismatches || samples < 0) return GELL_ERR_INVALID_ARG;
    long long m = 0;
    gell_status st = selftest_division(c, samples, seed, &m);
    *mismatches = m;
    return st;
}

gell_status gell_selftest_timeout(gell_ctx* c, int polls) {
    if (!c || polls < 1) return GELL_ERR_INVALID_ARG;
    if (gell_status st = selftest_timeout(c, polls)) return st;
    return gell_sync(c);
}

gell_status gell_set_option(gell_ctx* c, int option, int64_t value) {
    if (!c) return GELL_ERR_INVALID_ARG;
    switch (option) {
        case GELL_OPT_EXACT_CHAIN: c->exact_chain = value != 0; return GELL_OK;
        case GELL_OPT_SWEEP_WARPS:
            if (value < 0 || value > 4) return fail(c, GELL_ERR_INVALID_ARG, "sweep warps outside 0..4");
            c->sweep_warps = (int)value;
            return GELL_OK;
        case GELL_OPT_CONV_RING: c->conv_ring = value != 0; return GELL_OK;
        case GELL_OPT_SWEEP_RING:
            if (value < -1 || value > 8) return fail(c, GELL_ERR_INVALID_ARG, "sweep ring outside -1..8");
            c->sweep_ring = (int)value;
            return GELL_OK;
        case GELL_OPT_SWEEP_L2HINT: c->sweep_l2hint = value != 0; return GELL_OK;
        case GELL_OPT_LOD_STREAMS:
            c->lod_streams = value != 0;
            // the streams exist before any capture that uses them
            if (c->lod_streams) {
                bool ok = c->sub_fork || cudaEventCreateWithFlags(&c->sub_fork, cudaEventDisableTiming) == cudaSuccess;
                for (int s = 1; ok && s < (int)c->subs.size() && s < 8; ++s)
                    if (!c->sub_stream[s])
                        ok = cudaStreamCreateWithFlags(&c->sub_stream[s], cudaStreamNonBlocking) == cudaSuccess &&
                             cudaEventCreateWithFlags(&c->sub_join[s], cudaEventDisableTiming) == cudaSuccess;
                if (!ok) {
                    cudaGetLastError();
                    c->lod_streams = false;
                    return fail(c, GELL_ERR_CUDA, "substrate streams");
                }
            }
            return GELL_OK;
        case GELL_OPT_SURROGATE_INPUT:
            if (value < 0 || value > 1) return fail(c, GELL_ERR_INVALID_ARG, "surrogate input outside 0..1");
            c->sur_input = (int)value;
            return GELL_OK;
        case GELL_OPT_SWEEP_RING_LAG:
            if (value < 0 || value > 7) return fail(c, GELL_ERR_INVALID_ARG, "sweep ring lag outside 0..7");
            c->sweep_ring_lag = (int)value;
            return GELL_OK;
        default: return fail(c, GELL_ERR_INVALID_ARG, "unknown option");
    }
}

gell_status gell_launch_count(gell_ctx* c, int64_t* count) {
    if (!c || !count) return GELL_ERR_INVALID_ARG;
    *count = c->launches;
    return GELL_OK;
}

gell_status gell_fm_update(gell_ctx* c) {
    GELL_RANGE("gell_fm_update");
    if (!c) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    return cells_end(c, fm_update(c));
}

gell_status gell_prelod(gell_ctx* c, int sub) {
    GELL_RANGE("gell_prelod");
    if (!c || sub < -1 || sub >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    return cells_end(c, prelod(c, sub));
}

gell_status gell_lod_solver(gell_ctx* c, int sub, int substeps) {
    GELL_RANGE("gell_lod_solver");
    if (!c || sub < -1 || sub >= (int)c->subs.size() || substeps < 0) return GELL_ERR_INVALID_ARG;
    return lod_solver(c, sub, substeps);
}

gell_status gell_cell_birth(gell_ctx* c, int* n_out) {
    GELL_RANGE("gell_cell_birth");
    if (!c) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    return cells_end(c, birth(c, n_out));
}

gell_status gell_cell_death(gell_ctx* c, int* n_out) {
    GELL_RANGE("gell_cell_death");
    if (!c) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    return cells_end(c, death(c, n_out));
}

gell_status gell_mechanics_step(gell_ctx* c, int substeps) {
    GELL_RANGE("gell_mechanics_step");
    if (!c || substeps < 0) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    gell_status s = fm_update(c);
    if (s == GELL_OK) s = prelod(c, -1);
    s = cells_end(c, s);
    if (s == GELL_OK) s = lod_solver(c, -1, substeps);
    if (s == GELL_OK) c->stepped = true;
    return s;
}

}  // extern "C"

// Which buffer of each double-buffered cell field is current: a captured graph is only valid for
// the assignment it was captured with.
namespace gell {
uint32_t buffer_parity(const gell_ctx* c) {
    return (uint32_t)(c->sign.c | c->mesh.c << 1 | c->posr.c << 2 | c->force.c << 3 | c->oldf.c << 4 |
                      c->V.c << 5 | c->Vf.c << 6 | c->Vcs.c << 7 | c->Vns.c << 8 | c->clock.c << 9 |
                      c->phase.c << 10);
}

gell_status one_mechanics_step(gell_ctx* c, int substeps) {
    gell_status s = fm_update(c);
    if (s == GELL_OK) s = prelod(c, -1);
    if (s == GELL_OK) s = lod_solver(c, -1, substeps);
    return s;
}

// Capture two mechanics steps on the context's stream into cache entry `gs`.
}  // namespace gell

static gell_status capture_step_graph(gell_ctx* c, gell_ctx::StepGraph& gs, int substeps) {
    if (gs.exec) {
        cudaGraphExecDestroy(gs.exec);
        gs.exec = nullptr;
    }
    const uint32_t parity = buffer_parity(c);
    const long long l0 = c->launches;
    GELL_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    gell_status st = one_mechanics_step(c, substeps);
    if (st == GELL_OK) st = one_mechanics_step(c, substeps);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    // nothing ran during the capture: the launches are counted when the graph is replayed
    gs.launches = c->launches - l0;
    c->launches = l0;
    if (st != GELL_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&gs.exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        gs.exec = nullptr;
        return cuda_fail(c, ei, "cudaGraphInstantiate");
    }
    gs.n = c->n;
    gs.substeps = substeps;
    gs.nsub = (int)c->subs.size();
    gs.parity = parity;
    return GELL_OK;
}

extern "C" {

gell_status gell_run_mechanics(gell_ctx* c, int steps, int substeps) {
    GELL_RANGE("gell_run_mechanics");
    if (!c || steps < 0 || substeps < 0) return GELL_ERR_INVALID_ARG;
    if (steps == 0) return GELL_OK;
    if (gell_status b = cells_begin(c)) return b;
    int left = steps;
    gell_status st = GELL_OK;
    if (!c->stepped) {
        // the first step of a context runs outside any capture (first-use set-up of the kernels)
        st = one_mechanics_step(c, substeps);
        --left;
        c->stepped = st == GELL_OK;
    }
    if (st == GELL_OK && left >= 2 && !c->prof_on && c->n > 0) {
        const uint32_t par = buffer_parity(c);
        gell_ctx::StepGraph* gs = nullptr;
        for (auto& e : c->graphs)
            if (e.exec && e.n == c->n && e.substeps == substeps && e.nsub == (int)c->subs.size() && e.parity == par)
                gs = &e;
        if (!gs) {
            gs = c->graphs[0].used <= c->graphs[1].used ? &c->graphs[0] : &c->graphs[1];
            st = capture_step_graph(c, *gs, substeps);
        }
        gs->used = ++c->graph_clock;
        for (; left >= 2 && st == GELL_OK && gs->exec; left -= 2) {
            const cudaError_t e = cudaGraphLaunch(gs->exec, c->stream);
            if (e != cudaSuccess) st = cuda_fail(c, e, "cudaGraphLaunch");
            c->launches += gs->launches;
        }
    }
    for (; left > 0 && st == GELL_OK; --left) st = one_mechanics_step(c, substeps);
    if (st == GELL_OK) c->stepped = true;
    return cells_end(c, st);
}

gell_status gell_debug_dump(gell_ctx* c, int what, int arg, void* out, size_t bytes) {
    if (!c || !out) return GELL_ERR_INVALID_ARG;
    if (gell_status b = cells_begin(c)) return b;
    const int n = c->n;
    switch (what) {
        case GELL_DUMP_KEYS:
        case GELL_DUMP_PERM: {
            if (bytes < (size_t)n * 4) return GELL_ERR_INVALID_ARG;
            if (!c->sorted_valid) return fail(c, GELL_ERR_STATE, "no fm_update since the cells changed");
            const uint32_t* src = what == GELL_DUMP_KEYS ? c->sort.keys[c->sort.which] : c->sort.vals[c->sort.which];
            GELL_CUDA(c, cudaMemcpyAsync(out, src, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
            GELL_CUDA(c, cudaStreamSynchronize(c->stream));
            if (what == GELL_DUMP_KEYS) {
                int32_t* k = (int32_t*)out;
                for (int i = 0; i < n; ++i) k[i] = (int32_t)((uint32_t)k[i] - 1u);  // 0 -> -1
            }
            return GELL_OK;
        }
        case GELL_DUMP_SE: {
            if (bytes < (size_t)c->nvox * 8) return GELL_ERR_INVALID_ARG;
            if (!c->sorted_valid) return fail(c, GELL_ERR_STATE, "no fm_update since the cells changed");
            return dump_se(c, (int*)out);
        }
        case GELL_DUMP_RATE: {
            if (arg < 0 || arg >= (int)c->subs.size() || bytes < (size_t)c->nvox * 4) return GELL_ERR_INVALID_ARG;
            float* tmp = nullptr;
            GELL_CUDA(c, cudaMallocAsync((void**)&tmp, (size_t)c->nvox * 4, c->stream));
            GELL_KERNEL(c, "k_field_out", k_field_out<<<blocks_for(c->nvox, 256), 256, 0, c->stream>>>(c->subs[arg].rate, tmp, c->g));
            GELL_CUDA(c, cudaMemcpyAsync(out, tmp, (size_t)c->nvox * 4, cudaMemcpyDeviceToHost, c->stream));
            GELL_CUDA(c, cudaFreeAsync(tmp, c->stream));
            GELL_CUDA(c, cudaStreamSynchronize(c->stream));
            return GELL_OK;
        }
        case GELL_DUMP_EF: {
            if (arg < 0 || arg >= (int)c->subs.size() || bytes < (size_t)c->g.N * 8) return GELL_ERR_INVALID_ARG;
            memcpy(out, c->subs[arg].E.data(), c->g.N * 4);
            memcpy((float*)out + c->g.N, c->subs[arg].F.data(), c->g.N * 4);
            return GELL_OK;
        }
    }
    return GELL_ERR_INVALID_ARG;
}

}  // extern "C"
