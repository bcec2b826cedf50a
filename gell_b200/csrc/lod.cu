// lod.cu — LOD reaction-diffusion of the substrates (include/LODkernel.cuh:12-136,183-300).
//
// One substep of the reference (Mesh_struct::LODsolver) is Setboundary, meshupdatekernel and the
// three Thomas sweeps LODkernel_x/y/z, each a separate launch over one thread per line.  Here a
// substep is three launches, all substrates in each:
//   k_sweep_x        boundary layers + implicit uptake source + x sweep, fused per x-line
//   k_sweep_strided  y sweep (axis 1) and z sweep (axis 2)
// Every line is staged in shared memory by bulk asynchronous copies (the Blackwell TMA engine)
// completing on an mbarrier; each lane then runs one line's recurrence out of shared memory.
// x-lines are contiguous rows (one bulk copy per line, tile [32 lines][S]); y- and z-lines are
// strided, so a tile is 32 neighbouring lines and each bulk copy moves one 128-byte row of it
// (tile [N rows][32 lanes]), which makes every global access a full, coalesced row.
//
// Arithmetic per line, identical to the reference kernels with nvcc's multiply-add fusion:
//   Y0 = b; Y_i = fma(-E_i, Y_{i-1}, p_i) (i = 1..N-2); x_{N-1} = b;
//   x_i = fma(-s, x_{i+1}, Y_i) / F_i (i = N-2..1); x_0 = b;  s = E[1]*F[0]
// and the source p /= fma(-rate, dt, 1).  Division is IEEE round-to-nearest.
#include "gell_internal.cuh"

namespace gell {

namespace {

constexpr int kMaxSub = 8;
constexpr int kChunks = 4;  // mbarriers per strided tile, so the forward pass starts early
constexpr unsigned FULL = 0xffffffffu;

struct SubDev {
    float* p;
    const float* rate;
    const uint32_t* line_flag;
    const float* EF;
    float b;
    float side;
};

struct LodArgs {
    SubDev sub[kMaxSub];
    int nsub;
    Geom g;
    float dt;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded, warp-uniform wait on an mbarrier phase: every lane polls until all lanes see the phase
// complete; after a fixed number of polls the warp gives up together, records `code` in the
// context's error word and returns false (the host then reports GELL_ERR_TIMEOUT).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int* err, int code) {
    for (int it = 0; it < (1 << 22); ++it)
        if (__all_sync(FULL, mbar_try_wait(b, parity))) return true;
    if ((threadIdx.x & 31) == 0) atomicExch(err, code);
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__host__ __device__ inline int align128(int b) { return (b + 127) / 128 * 128; }

// Shared-memory row stride of an x-tile: >= P, a multiple of 4 floats (16-byte rows for the bulk
// copies) with an odd number of 16-byte units, so that 32 lanes reading float4 element c of their
// own rows hit distinct banks.
__host__ __device__ inline int xrow_stride(int P) { return ((P / 4) % 2 == 1) ? P : P + 4; }

__device__ __forceinline__ void load_ef(float* sEF, const LodArgs& a) {
    const int N = a.g.N;
    for (int i = threadIdx.x; i < a.nsub * 2 * N; i += blockDim.x) {
        int s = i / (2 * N), r = i - s * 2 * N;
        sEF[i] = a.sub[s].EF[r];
    }
}

// Thomas recurrence of one line held in shared memory (row), in place, float4 at a time.
__device__ __forceinline__ void thomas_row(float* row, const float* E, const float* F, float s,
                                           float b, int N) {
    float4* r4 = reinterpret_cast<float4*>(row);
    float Y = b;
    const int cmax = (N - 2) / 4;  // last chunk holding an element <= N-2
    for (int c = 0; c <= cmax; ++c) {
        float4 q = r4[c];
        float e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int i = 4 * c + k;
            if (i >= 1 && i <= N - 2) {
                Y = __fmaf_rn(-E[i], Y, e[k]);
                e[k] = Y;
            }
        }
        r4[c] = make_float4(e[0], e[1], e[2], e[3]);
    }
    float x = b;
    for (int c = cmax; c >= 0; --c) {
        float4 q = r4[c];
        float e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            int i = 4 * c + k;
            if (i >= 1 && i <= N - 2) {
                x = __fdiv_rn(__fmaf_rn(-s, x, e[k]), F[i]);
                e[k] = x;
            }
        }
        r4[c] = make_float4(e[0], e[1], e[2], e[3]);
    }
    row[0] = b;
    row[N - 1] = b;
}

// Boundary layers + source + x sweep.  A warp owns 32 consecutive x-lines (line = y + z*N).
__global__ void __launch_bounds__(512) k_sweep_x(LodArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    const Geom g = a.g;
    const int N = g.N, P = g.P, S = xrow_stride(P);
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* sEF = reinterpret_cast<float*>(sm);
    const int efb = align128(a.nsub * 2 * N * 4);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + efb);
    float* tile = reinterpret_cast<float*>(sm + efb + align128(warps * 8)) + (size_t)warp * 32 * S;
    uint64_t* bar = bars + warp;
    load_ef(sEF, a);
    if (lane == 0) mbar_init(bar, 1);
    fence_mbar_init();
    __syncthreads();

    const long long nlines = (long long)N * N;
    const long long per_sub = (nlines + 31) / 32;
    const long long total = per_sub * a.nsub;
    uint32_t parity = 0;
    for (long long t = (long long)blockIdx.x * warps + warp; t < total; t += (long long)gridDim.x * warps) {
        const int s = (int)(t / per_sub);
        const long long tt = t - s * per_sub;
        const SubDev sd = a.sub[s];
        const float* E = sEF + s * 2 * N;
        const float* F = E + N;
        const long long line = tt * 32 + lane;
        const bool valid = line < nlines;
        const int y = valid ? (int)(line % N) : 0, z = valid ? (int)(line / N) : 0;
        // every voxel of a line in the two outer layers of a y or z face is set to b
        const bool bline = !valid || y < 2 || y >= N - 2 || z < 2 || z >= N - 2;
        float* gl = sd.p + line * P;
        const unsigned m = __ballot_sync(FULL, !bline);
        if (m) {
            if (lane == 0) mbar_arrive_expect(bar, (uint32_t)__popc(m) * P * 4);
            __syncwarp();
            if (!bline) bulk_g2s(tile + lane * S, gl, P * 4, bar);
            if (!mbar_wait(bar, parity, a.err, 1)) return;
            parity ^= 1;
        }
        // Setboundary (include/LODkernel.cuh:112-136) and meshupdatekernel (:24-31), one line at
        // a time across the warp; the uptake map is read only on lines that hold cells.
        for (int r = 0; r < 32; ++r) {
            const long long ln = tt * 32 + r;
            if (ln >= nlines) break;
            const int yr = (int)(ln % N), zr = (int)(ln / N);
            const bool blr = yr < 2 || yr >= N - 2 || zr < 2 || zr >= N - 2;
            const bool fl = sd.line_flag[ln] != 0;
            const float* rl = sd.rate + ln * P;
            float* row = tile + r * S;
            for (int i = lane; i < N; i += 32) {
                float v = (blr || i < 2 || i >= N - 2) ? sd.b : row[i];
                if (fl) v = __fdiv_rn(v, __fmaf_rn(-rl[i], a.dt, 1.f));
                row[i] = v;
            }
        }
        __syncwarp();
        if (valid) thomas_row(tile + lane * S, E, F, sd.side, sd.b, N);
        fence_proxy_async();
        __syncwarp();
        if (valid) {
            bulk_s2g(gl, tile + lane * S, P * 4);
            bulk_commit();
            bulk_wait_read0();
        }
        __syncwarp();
    }
}

// y sweep (axis 1: lines (x, z), element stride P) or z sweep (axis 2: lines (x, y) flattened to
// x + y*P, element stride P*N).  A warp owns 32 neighbouring lines: row j of its tile is the
// 128-byte run of element j of those lines.
__global__ void __launch_bounds__(512) k_sweep_strided(LodArgs a, int axis) {
    extern __shared__ __align__(128) unsigned char sm[];
    const Geom g = a.g;
    const int N = g.N, P = g.P;
    const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* sEF = reinterpret_cast<float*>(sm);
    const int efb = align128(a.nsub * 2 * N * 4);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + efb) + warp * kChunks;
    float* tile = reinterpret_cast<float*>(sm + efb + align128(warps * kChunks * 8)) + (size_t)warp * N * 32;
    load_ef(sEF, a);
    if (lane < kChunks) mbar_init(bar + lane, 1);
    fence_mbar_init();
    __syncthreads();

    const int ntx = (P + 31) / 32;
    const long long per_sub = axis == 1 ? (long long)ntx * N : (g.PN + 31) / 32;
    const long long total = per_sub * a.nsub;
    const int R = (N - 2 + kChunks - 1) / kChunks;  // rows per chunk over rows 1..N-2
    uint32_t parity = 0;
    for (long long t = (long long)blockIdx.x * warps + warp; t < total; t += (long long)gridDim.x * warps) {
        const int s = (int)(t / per_sub);
        const long long tt = t - s * per_sub;
        const SubDev sd = a.sub[s];
        const float* E = sEF + s * 2 * N;
        const float* F = E + N;
        float* base;
        long long rs;
        int width;
        bool valid;
        if (axis == 1) {
            const int z = (int)(tt / ntx), x0 = (int)(tt - (long long)z * ntx) * 32;
            base = sd.p + x0 + (long long)z * g.PN;
            rs = P;
            width = min(32, P - x0);
            valid = x0 + lane < N;
        } else {
            const long long L0 = tt * 32;
            base = sd.p + L0;
            rs = g.PN;
            width = (int)min(32LL, g.PN - L0);
            const long long L = L0 + lane;
            valid = L < g.PN && (int)(L % P) < N;
        }
        if (lane == 0) {
            for (int c = 0; c < kChunks; ++c) {
                const int lo = 1 + c * R, hi = min(N - 1, lo + R);
                if (hi > lo) mbar_arrive_expect(bar + c, (uint32_t)(hi - lo) * width * 4);
            }
        }
        __syncwarp();
        for (int j = 1 + lane; j <= N - 2; j += 32)
            bulk_g2s(tile + j * 32, base + j * rs, width * 4, bar + (j - 1) / R);
        // forward elimination, chunk by chunk as the rows land
        float Y = sd.b;
        for (int c = 0; c < kChunks; ++c) {
            const int lo = 1 + c * R, hi = min(N - 1, lo + R);
            if (hi <= lo) break;
            if (!mbar_wait(bar + c, (parity >> c) & 1u, a.err, 2)) return;
            parity ^= 1u << c;
            for (int j = lo; j < hi; ++j) {
                Y = __fmaf_rn(-E[j], Y, tile[j * 32 + lane]);
                tile[j * 32 + lane] = Y;
            }
        }
        // back substitution, written straight to global memory (a 128-byte row per element)
        float x = sd.b;
        float* gp = base + lane;
        if (valid) gp[(long long)(N - 1) * rs] = x;
        for (int j = N - 2; j >= 1; --j) {
            x = __fdiv_rn(__fmaf_rn(-sd.side, x, tile[j * 32 + lane]), F[j]);
            if (valid) gp[(long long)j * rs] = x;
        }
        if (valid) gp[0] = sd.b;
        fence_proxy_async();
        __syncwarp();
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

// Clear the lines flagged by the previous map (oxy_consumption_reset, include/LODkernel.cuh:183-190,
// restricted to the lines that can be nonzero).
__global__ void k_rate_reset(PreArgs a) {
    const int P = a.g.P;
    for (int s = 0; s < a.nsub; ++s) {
        const int cnt = *a.count[s];
        for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < (long long)cnt * P;
             w += (long long)gridDim.x * blockDim.x) {
            const int li = (int)(w / P), x = (int)(w - (long long)li * P);
            const int line = a.list[s][li];
            a.rate[s][(long long)line * P + x] = 0.f;
            if (x == 0) a.flag[s][line] = 0;
        }
    }
}

// oxy_consumption_update (include/LODkernel.cuh:12-22) with Cell::O2_consume (include/Cells.cuh:74-89)
// at O2 = 1: rate[mesh_idx] += coef * (V/len/len/len) (times the dead factor for phase >= 3).
__global__ void k_rate_accum(CellsSoA c, int n, PreArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

gell_status lod_solver(gell_ctx* c, int sub, int substeps) {
    if (c->subs.empty() || substeps == 0) return GELL_OK;
    LodArgs a{};
    int s0 = sub < 0 ? 0 : sub, s1 = sub < 0 ? (int)c->subs.size() : sub + 1;
    for (int s = s0; s < s1; ++s) {
        const Substrate& S = c->subs[s];
        a.sub[a.nsub++] = SubDev{S.p, S.rate, S.line_flag, S.EF, S.s.boundary, S.side};
    }
    a.g = c->g;
    a.dt = c->P.diffusion_dt;
    a.err = c->dev_err;
    const int N = c->g.N;
    const int efb = align128(a.nsub * 2 * N * 4);
    const int smem_cap = 227 * 1024;
    // x: [32][S] per warp
    const int xtile = 32 * xrow_stride(c->g.P) * 4;
    int wx = (smem_cap - efb - 128) / xtile;
    wx = wx > 16 ? 16 : wx;
    // y/z: [N][32] per warp
    const int stile = N * 32 * 4;
    int ws = (smem_cap - efb - 128 * 2) / stile;
    ws = ws > 16 ? 16 : ws;
    if (wx < 1 || ws < 1) return fail(c, GELL_ERR_UNSUPPORTED, "grid edge too large for the shared-memory line tiles");
    const int smx = efb + align128(wx * 8) + wx * xtile;
    const int sms = efb + align128(ws * kChunks * 8) + ws * stile;
    static int configured = 0;
    if (!configured) {
        GELL_CUDA(c, cudaFuncSetAttribute(k_sweep_x, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        GELL_CUDA(c, cudaFuncSetAttribute(k_sweep_strided, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
        configured = 1;
    }
    const long long nlines = (long long)N * N;
    const long long xt = (nlines + 31) / 32 * a.nsub;
    const long long yt = (long long)((c->g.P + 31) / 32) * N * a.nsub;
    const long long zt = (c->g.PN + 31) / 32 * a.nsub;
    auto grid = [&](long long tiles, int w, int smem) {
        int per_sm = smem_cap / (smem + 1024);
        if (per_sm < 1) per_sm = 1;
        long long want = (tiles + w - 1) / w;
        long long cap = (long long)num_sms() * per_sm;
        return (int)(want < cap ? want : cap);
    };
    const int gx = grid(xt, wx, smx), gy = grid(yt, ws, sms), gz = grid(zt, ws, sms);
    for (int k = 0; k < substeps; ++k) {
        GELL_KERNEL(c, "k_sweep_x", k_sweep_x<<<gx, wx * 32, smx, c->stream>>>(a));
        GELL_KERNEL(c, "k_sweep_strided(y)", k_sweep_strided<<<gy, ws * 32, sms, c->stream>>>(a, 1));
        GELL_KERNEL(c, "k_sweep_strided(z)", k_sweep_strided<<<gz, ws * 32, sms, c->stream>>>(a, 2));
    }
    return GELL_OK;
}

}  // namespace gell
