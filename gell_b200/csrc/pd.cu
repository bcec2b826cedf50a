// pd.cu — stochastic birth and death (include/PDkernel.cuh:27-117, include/Cells.cuh:91-223,
// include/RandomFunctions.cuh:13-31).
//
// Birth: k_birth_update draws u for each live cell, updates its volume and Ki-67 phase and flags
// the cells that divide; an exclusive scan of the flags gives each mother, in slot order, the slot
// of its daughter (the reference takes slots from atomicAdd, so its order varies run to run);
// k_birth_divide halves the mother and writes the daughter.  Death: stable compaction of the cells
// whose sign is set, like thrust::remove_if(isDeadCell).
//
// Draws: GELL_RNG_XORWOW keeps one curand XORWOW state per slot initialised with
// curand_init(seed, slot, 0) and draws exactly as the reference does (u, then two draws for the
// division direction of a mother that gets a slot).  GELL_RNG_PHILOX draws the same three
// numbers from Philox4x32-10 with counter (slot, biology step, 0, 0) and key (seed).
#include "gell_internal.cuh"

namespace gell {

namespace {

__global__ void k_init_xorwow(curandState* st, int cap, unsigned long long seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    curand_init(seed, (unsigned long long)i, 0ull, &st[i]);
}

struct BioParams {
    float bio_dt;
    float default_v;
    float o2_pt, o2_ps, o2_nt, o2_nm;
    double necrosis_rate, apoptosis_rate, prolif_rate;
    float dur_pre2post, dur_post2q;
};

// Cell::Volume_update (include/Cells.cuh:91-143): Vx' = Vx*(1 - dt*rx) + (rx*dt)*Vx_0 with the
// reference's device rounding.  1 - dt*rx and rx*dt are rounded once each; the fluid compartment,
// whose target V*ff varies per cell, fuses Vf*(1 - dt*rf) into the sum, while the nuclear and
// cytoplasmic compartments, whose targets are per-phase constants, fuse (rx*dt)*Vx_0 instead
// (measured against the reference's own device build on every phase).  V = (Vf + Vns) + Vcs,
// r = cbrt-by-pow in double.
__device__ __forceinline__ float relax_fluid(float v, float rx, float v0, float dt) {
    const float k = __fsub_rn(1.f, __fmul_rn(dt, rx));
    return __fmaf_rn(v, k, __fmul_rn(__fmul_rn(rx, dt), v0));
}
__device__ __forceinline__ float relax_const_target(float v, float rx, float v0, float dt) {
    const float k = __fsub_rn(1.f, __fmul_rn(dt, rx));
    return __fmaf_rn(__fmul_rn(rx, dt), v0, __fmul_rn(v, k));
}

__device__ void volume_update(int ph, float& V, float& Vf, float& Vcs, float& Vns, float& r) {
    const float dt = 6.f;  // Biology_dt as the reference's Cell model uses it
    float ff = (float)0.7502;
    float rf = 3.f / 60.f;
    float rcs = 0.33f / 60.f;
    float rns = 0.33f / 60.f;
    float Vns_0 = 135.f;
    if (ph == 1) {
        Vns_0 = 270.f;
        rcs = (float)(0.27 / 60);
    } else if (ph == 3) {
        ff = 0.f;
        Vns_0 = 0.f;
        rns = (float)(0.35 / 60);
        rcs = 1.f / 60;
    } else if (ph == 4) {
        ff = 1.f;
        rf = (float)(0.67 / 60);
        Vns_0 = 0.f;
        rns = (float)(0.013 / 60);
        rcs = (float)(0.0032 / 60);
    } else if (ph == 5) {
        ff = 0.f;
        rf = (float)(0.05 / 60);
        Vns_0 = 0.f;
        rns = (float)(0.013 / 60);
        rcs = (float)(0.0032 / 60);
    }
    const float Vf_0 = __fmul_rn(V, ff);
    const float Vcs_0 = __fmul_rn(Vns_0, 3.615f);
    Vf = relax_fluid(Vf, rf, Vf_0, dt);
    Vns = relax_const_target(Vns, rns, Vns_0, dt);
    Vcs = relax_const_target(Vcs, rcs, Vcs_0, dt);
    V = __fadd_rn(__fadd_rn(Vf, Vns), Vcs);
    r = (float)pow(0.23873241 * (double)V, 1.0 / 3);
}

// Cell::Phase_update_ki67adv (include/Cells.cuh:145-223); the probabilities are evaluated in
// double where the reference's rates are double-typed macros.  Returns true on mitosis.
__device__ bool phase_update(const BioParams& B, float rnd, float o2, int& phase, float& clock,
                             uint8_t& sign, float V, float Vcs) {
    const double dt = (double)B.bio_dt;
    clock = __fadd_rn(clock, B.bio_dt);
    bool proliferate = false;
    const float apop = __double2float_rn(__dmul_rn(B.apoptosis_rate, dt));
    float prolif = __double2float_rn(__dmul_rn(
        __dmul_rn((double)__fdiv_rn(__fsub_rn(o2, B.o2_pt), __fsub_rn(B.o2_ps, B.o2_pt)), B.prolif_rate), dt));
    if (o2 > B.o2_ps) prolif = __double2float_rn(__dmul_rn(B.prolif_rate, dt));
    else if (o2 < B.o2_pt) prolif = 0.f;
    float necro = __double2float_rn(__dmul_rn(
        __dmul_rn((double)__fdiv_rn(__fsub_rn(B.o2_nt, o2), __fsub_rn(B.o2_nt, B.o2_nm)), B.necrosis_rate), dt));
    if (o2 > B.o2_nt) necro = 0.f;
    else if (o2 < B.o2_nm) necro = __double2float_rn(__dmul_rn(B.necrosis_rate, dt));

    if (phase >= 3) {
        if (phase == 4 && V >= __fmul_rn(B.default_v, 2.f)) {
            phase = 5;
            clock = 0.f;
        }
        if (Vcs <= __fmul_rn(0.05f, 488.f)) {
            sign = 0;
            clock = 0.f;
        }
    } else {
        if (phase == 1 && clock >= B.dur_pre2post) {
            phase = 2;
            proliferate = true;
            clock = 0.f;
        }
        if (phase == 2 && clock >= B.dur_post2q) {
            phase = 0;
            clock = 0.f;
        }
        if (phase == 0) {
            const float pa = __fadd_rn(prolif, apop);
            if (rnd <= prolif) {
                phase = 1;
                clock = 0.f;
            } else if (rnd <= pa) {
                phase = 3;
                clock = 0.f;
            } else if (rnd <= __fadd_rn(pa, necro)) {
                phase = 4;
                clock = 0.f;
            }
        }
    }
    return proliferate;
}

struct BirthArgs {
    CellsSoA c;
    int n;
    int cap;
    const float* field;  // substrate driving the cell model (pitched), or null (O2 = 0)
    Geom g;
    BioParams B;
    int rng;              // gell_rng_mode
    curandState* xorwow;
    uint2 key;
    uint32_t step;
    uint32_t* flags;
    const uint32_t* rank;
};

__device__ __forceinline__ float field_at(const BirthArgs& a, float4 pr) {
    if (!a.field) return 0.f;
    int3 b = find_bin(pr.x, pr.y, pr.z, a.g.len);
    // the reference indexes p with Find_Index (which only prints when out of range); a cell
    // outside the grid reads the nearest voxel here
    b.x = min(max(b.x, 0), a.g.N - 1);
    b.y = min(max(b.y, 0), a.g.N - 1);
    b.z = min(max(b.z, 0), a.g.N - 1);
    return a.field[b.x + (long long)b.y * a.g.P + (long long)b.z * a.g.PN];
}

__global__ void k_birth_update(BirthArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    uint8_t sg = a.c.sign[i];
    if (!sg) {
        a.flags[i] = 0;
        return;
    }
    float u;
    if (a.rng == GELL_RNG_XORWOW) {
        curandState st = a.xorwow[i];
        u = curand_uniform(&st);
        a.xorwow[i] = st;
    } else {
        u = u01(philox4x32_10(make_uint4((uint32_t)i, a.step, 0u, 0u), a.key).x);
    }
    const float4 pr = a.c.posr[i];
    const float o2 = field_at(a, pr);
    float V = a.c.V[i], Vf = a.c.Vf[i], Vcs = a.c.Vcs[i], Vns = a.c.Vns[i], r;
    int ph = a.c.phase[i];
    float clock = a.c.clock[i];
    volume_update(ph, V, Vf, Vcs, Vns, r);
    const bool proli = phase_update(a.B, u, o2, ph, clock, sg, V, Vcs);
    a.c.V[i] = V;
    a.c.Vf[i] = Vf;
    a.c.Vcs[i] = Vcs;
    a.c.Vns[i] = Vns;
    a.c.posr[i] = make_float4(pr.x, pr.y, pr.z, r);
    a.c.phase[i] = ph;
    a.c.clock[i] = clock;
    a.c.sign[i] = sg;
    a.flags[i] = proli ? 1u : 0u;
}

// RandomFunctions.cuh:23-31
__device__ __forceinline__ float3 random_vect(float u, float v) {
    const float theta = __fmul_rn(__fmul_rn(2.f, u), 3.1415926f);
    const float phi = acosf(__fmaf_rn(2.f, v, -1.f));
    const float sp = sinf(phi);
    return make_float3(__fmul_rn(sinf(theta), sp), __fmul_rn(cosf(theta), sp), cosf(phi));
}

__global__ void k_birth_divide(BirthArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n || !a.flags[i]) return;
    const long long slot = (long long)a.n + a.rank[i];
    if (slot >= (long long)a.cap - 1) return;  // the reference stops placing daughters at Max_Cell_num-1
    float u1, v1;
    if (a.rng == GELL_RNG_XORWOW) {
        curandState st = a.xorwow[i];
        u1 = curand_uniform(&st);
        v1 = curand_uniform(&st);
        a.xorwow[i] = st;
    } else {
        const uint4 q = philox4x32_10(make_uint4((uint32_t)i, a.step, 0u, 0u), a.key);
        u1 = u01(q.y);
        v1 = u01(q.z);
    }
    const float3 dir = random_vect(u1, v1);
    const float4 pr = a.c.posr[i];
    const float dist = __fmul_rn(0.2063f, pr.w);
    const float rm = __fmul_rn(pr.w, 0.7937f);
    const float V = __fdiv_rn(a.c.V[i], 2.f), Vf = __fdiv_rn(a.c.Vf[i], 2.f);
    const float Vcs = __fdiv_rn(a.c.Vcs[i], 2.f), Vns = __fdiv_rn(a.c.Vns[i], 2.f);
    a.c.posr[i] = make_float4(__fmaf_rn(-dir.x, dist, pr.x), __fmaf_rn(-dir.y, dist, pr.y),
                              __fmaf_rn(-dir.z, dist, pr.z), rm);
    a.c.phase[i] = 2;
    a.c.clock[i] = 0.f;
    a.c.V[i] = V;
    a.c.Vf[i] = Vf;
    a.c.Vcs[i] = Vcs;
    a.c.Vns[i] = Vns;
    const int k = (int)slot;
    a.c.sign[k] = 1;
    a.c.mesh[k] = -1;
    a.c.posr[k] = make_float4(__fmaf_rn(dir.x, dist, pr.x), __fmaf_rn(dir.y, dist, pr.y),
                              __fmaf_rn(dir.z, dist, pr.z), rm);
    a.c.force[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    a.c.oldf[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    a.c.V[k] = V;
    a.c.Vf[k] = Vf;
    a.c.Vcs[k] = Vcs;
    a.c.Vns[k] = Vns;
    a.c.phase[k] = 2;
    a.c.clock[k] = 0.f;
}

__global__ void k_sign_flags(const uint8_t* sign, int n, uint32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = sign[i] ? 1u : 0u;
}

__global__ void k_compact(CellsSoA s, CellsSoA d, const uint32_t* __restrict__ pos, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !s.sign[i]) return;
    const int k = (int)pos[i];
    d.sign[k] = 1;
    d.mesh[k] = s.mesh[i];
    d.posr[k] = s.posr[i];
    d.force[k] = s.force[i];
    d.oldf[k] = s.oldf[i];
    d.V[k] = s.V[i];
    d.Vf[k] = s.Vf[i];
    d.Vcs[k] = s.Vcs[i];
    d.Vns[k] = s.Vns[i];
    d.clock[k] = s.clock[i];
    d.phase[k] = s.phase[i];
}

}  // namespace

gell_status init_xorwow(gell_ctx* c) {
    GELL_KERNEL(c, "k_init_xorwow", k_init_xorwow<<<blocks_for(c->cap, 256), 256, 0, c->stream>>>(c->xorwow, c->cap, c->P.seed));
    return GELL_OK;
}

gell_status birth(gell_ctx* c, int* n_out) {
    const int n = c->n;
    // the reference's Birthkernel returns at once when the count is at capacity (PDkernel.cuh:31)
    if (n > 0 && n < c->cap) {
        BirthArgs a{};
        a.c = c->cur();
        a.n = n;
        a.cap = c->cap;
        const int o2 = c->P.o2_substrate;
        a.field = (o2 >= 0 && o2 < (int)c->subs.size()) ? c->subs[o2].p : nullptr;
        a.g = c->g;
        a.B = BioParams{c->P.biology_dt, c->P.default_v, c->P.o2_prolif_thres, c->P.o2_prolif_sat,
                        c->P.o2_necrosis_thres, c->P.o2_necrosis_max, c->P.necrosis_rate,
                        c->P.apoptosis_rate, c->P.proliferation_rate, c->P.duration_pre2post,
                        c->P.duration_post2q};
        a.rng = c->P.rng_mode;
        a.xorwow = c->xorwow;
        a.key = make_uint2((uint32_t)c->P.seed, (uint32_t)(c->P.seed >> 32));
        a.step = c->bio_step;
        a.flags = c->flags;
        GELL_KERNEL(c, "k_birth_update", k_birth_update<<<blocks_for(n, 256), 256, 0, c->stream>>>(a));
        // daughter ranks: the sort payload buffer is free between mechanics steps
        uint32_t* ranks = c->sort.vals[1];
        gell_status st = scan_u32(c, c->flags, ranks, n, c->dev_count);
        if (st != GELL_OK) return st;
        a.rank = ranks;
        GELL_KERNEL(c, "k_birth_divide", k_birth_divide<<<blocks_for(n, 256), 256, 0, c->stream>>>(a));
        int total = 0;
        GELL_CUDA(c, cudaMemcpyAsync(&total, c->dev_count, 4, cudaMemcpyDeviceToHost, c->stream));
        GELL_CUDA(c, cudaStreamSynchronize(c->stream));
        long long room = (long long)c->cap - 1 - n;
        if (room < 0) room = 0;
        c->n = n + (int)(total < room ? total : room);
    }
    c->bio_step += 1;
    c->sorted_valid = false;
    c->rate_valid = false;
    if (n_out) *n_out = c->n;
    return GELL_OK;
}

gell_status death(gell_ctx* c, int* n_out) {
    const int n = c->n;
    if (n > 0) {
        GELL_KERNEL(c, "k_sign_flags", k_sign_flags<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->sign.cur(), n, c->flags));
        uint32_t* pos = c->sort.vals[0];
        gell_status st = scan_u32(c, c->flags, pos, n, c->dev_count);
        if (st != GELL_OK) return st;
        GELL_KERNEL(c, "k_compact", k_compact<<<blocks_for(n, 256), 256, 0, c->stream>>>(c->cur(), c->alt(), pos, n));
        int total = 0;
        GELL_CUDA(c, cudaMemcpyAsync(&total, c->dev_count, 4, cudaMemcpyDeviceToHost, c->stream));
        GELL_CUDA(c, cudaStreamSynchronize(c->stream));
        c->swap_all();
        c->n = total;
    }
    c->sorted_valid = false;
    c->rate_valid = false;
    if (n_out) *n_out = c->n;
    return GELL_OK;
}

}  // namespace gell
