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
#include "mech_body.cuh"

namespace gell {

namespace {

__global__ void k_keys(CellsSoA c, int n, Geom g, uint32_t* __restrict__ keys, int* __restrict__ epoch) {
    keys_body(c, n, g, keys, epoch, blockIdx.x);
}

__global__ void k_gather(CellsSoA s, CellsSoA d, const uint32_t* __restrict__ keys,
                         const uint32_t* __restrict__ perm, int n, int4* __restrict__ bins,
                         const int* __restrict__ epoch_p) {
    gather_body(s, d, keys, perm, n, bins, epoch_p, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_force_move(MechArgs a) { force_move_body(a, blockIdx.x); }

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

// ------------------------------------------------------------------ ensembles: batched mechanics
//
// One FM_update and one PreLOD of every member of an ensemble as one launch per kernel: keys, the
// sort's three kernels per digit pass, the gather, the force and move, the uptake map.  A batched
// launch's blocks are the members' own blocks laid end to end; block b runs the kernel body (the
// same device code as the member's own launch, mech_body.cuh) for block b - start[m] of the member
// m whose range holds b.  The arguments travel by value in the launch (at most kBatchMembers
// members), so a captured graph holds them and no device table is kept.  Members keep their own
// digit widths and pass counts (their grids differ); a member with fewer passes sits out the last
// ones.  The host swaps each member's buffers exactly as fm_update and prelod do.

namespace {

constexpr int kBatchMembers = 64;
constexpr int kBatchSub = 4;

struct BlockMap {
    int nm;
    int start[kBatchMembers + 1];  // member m owns blocks [start[m], start[m+1])
};

// member of block b (binary search over the starts) and the block's index inside the member
__device__ __forceinline__ int member_of(const BlockMap& bm, int b, int& local) {
    int lo = 0, hi = bm.nm;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (bm.start[mid] <= b) lo = mid;
        else hi = mid;
    }
    local = b - bm.start[lo];
    return lo;
}

struct KeysJob {
    CellsSoA c;
    uint32_t* keys;
    int* epoch;
    Geom g;
    int n;
};
struct KeysBatch {
    BlockMap map;
    KeysJob job[kBatchMembers];
};
__global__ void k_keys_batch(const __grid_constant__ KeysBatch b) {
    int local;
    const KeysJob& j = b.job[member_of(b.map, blockIdx.x, local)];
    keys_body(j.c, j.n, j.g, j.keys, j.epoch, local);
}

struct SortJob {
    const uint32_t* kin;
    const uint32_t* vin;
    uint32_t* kout;
    uint32_t* vout;
    uint32_t* hist;
    int n, nb, shift, R, iota;
};
struct SortBatch {
    BlockMap tiles, digits;
    SortJob job[kBatchMembers];
};
__global__ void __launch_bounds__(kSortThreads) k_hist_batch(const __grid_constant__ SortBatch b) {
    int local;
    const SortJob& j = b.job[member_of(b.tiles, blockIdx.x, local)];
    hist_body(j.kin, j.n, j.shift, j.R, j.hist, j.nb, local);
}
__global__ void __launch_bounds__(kSortThreads) k_digit_scan_batch(const __grid_constant__ SortBatch b) {
    int local;
    const SortJob& j = b.job[member_of(b.digits, blockIdx.x, local)];
    digit_scan_body(j.hist, j.nb, j.hist + (size_t)j.R * j.nb, local);
}
__global__ void __launch_bounds__(kSortThreads) k_scatter_batch(const __grid_constant__ SortBatch b) {
    int local;
    const SortJob& j = b.job[member_of(b.tiles, blockIdx.x, local)];
    scatter_body(j.kin, j.vin, j.kout, j.vout, j.n, j.shift, j.R, j.hist, j.nb, j.hist + (size_t)j.R * j.nb, j.iota,
                 local);
}

struct GatherJob {
    CellsSoA s, d;
    const uint32_t* keys;
    const uint32_t* perm;
    int4* bins;
    const int* epoch;
    int n;
};
struct GatherBatch {
    BlockMap map;
    GatherJob job[kBatchMembers];
};
__global__ void k_gather_batch(const __grid_constant__ GatherBatch b) {
    int local;
    const GatherJob& j = b.job[member_of(b.map, blockIdx.x, local)];
    gather_body(j.s, j.d, j.keys, j.perm, j.n, j.bins, j.epoch, local);
}

struct ForceBatch {
    BlockMap map;
    MechArgs job[kBatchMembers];
};
__global__ void __launch_bounds__(256) k_force_move_batch(const __grid_constant__ ForceBatch b) {
    int local;
    const MechArgs& j = b.job[member_of(b.map, blockIdx.x, local)];
    force_move_body(j, local);
}

// the uptake map's arguments (lod.cu's PreArgs for at most kBatchSub substrates) and the cells
struct PreJob {
    float* rate[kBatchSub];
    uint32_t* flag[kBatchSub];
    int* list[kBatchSub];
    int* count[kBatchSub];
    float coef[kBatchSub];
    CellsSoA c;
    Geom g;
    float dead;
    int nsub;
    int n;
};
struct PreBatch {
    BlockMap map;  // k_rate_accum blocks
    PreJob job[kBatchMembers];
};
constexpr int kResetBlocks = 8;  // k_rate_reset blocks per member (a grid-stride loop over its listed lines)
__global__ void k_rate_reset_batch(const __grid_constant__ PreBatch b) {
    rate_reset_body(b.job[blockIdx.y], blockIdx.x, gridDim.x);
}
__global__ void k_zero_counts_batch(const __grid_constant__ PreBatch b) {
    const int m = threadIdx.x / kBatchSub, s = threadIdx.x % kBatchSub;
    if (m < b.map.nm && s < b.job[m].nsub) *b.job[m].count[s] = 0;
}
__global__ void k_rate_accum_batch(const __grid_constant__ PreBatch b) {
    int local;
    const PreJob& j = b.job[member_of(b.map, blockIdx.x, local)];
    rate_accum_body(j.c, j.n, j, local);
}

static_assert(sizeof(KeysBatch) <= 32000 && sizeof(SortBatch) <= 32000 && sizeof(GatherBatch) <= 32000 &&
                  sizeof(ForceBatch) <= 32000 && sizeof(PreBatch) <= 32000,
              "batched arguments exceed the kernel parameter limit");
static_assert(kBatchMembers * kBatchSub <= 256, "k_zero_counts_batch runs one thread per (member, substrate)");

// start[] of a map over blocks[i] blocks per entry; total blocks
int fill_map(BlockMap& m, const std::vector<int>& blocks) {
    m.nm = (int)blocks.size();
    int t = 0;
    for (size_t i = 0; i < blocks.size(); ++i) {
        m.start[i] = t;
        t += blocks[i];
    }
    m.start[blocks.size()] = t;
    return t;
}

}  // namespace

bool mech_batch_ok(const std::vector<gell_ctx*>& ms) {
    if (ms.empty() || ms.size() > (size_t)kBatchMembers) return false;
    for (const gell_ctx* c : ms)
        if (c->subs.size() > (size_t)kBatchSub) return false;
    return true;
}

gell_status mech_batch_step(const std::vector<gell_ctx*>& ms, cudaStream_t st) {
    if (!mech_batch_ok(ms)) return GELL_ERR_UNSUPPORTED;
    gell_ctx* c0 = ms[0];  // the batched launches are counted (and profiled) on the first member

    // FM_update of the members that hold cells
    std::vector<gell_ctx*> fm;
    for (gell_ctx* c : ms)
        if (c->n > 0) fm.push_back(c);
    if (!fm.empty()) {
        const int nf = (int)fm.size();
        std::vector<int> blocks(nf);
        for (int i = 0; i < nf; ++i) blocks[i] = blocks_for(fm[i]->n, 256);

        KeysBatch kb{};
        const int kblocks = fill_map(kb.map, blocks);
        for (int i = 0; i < nf; ++i) {
            gell_ctx* c = fm[i];
            kb.job[i] = KeysJob{c->cur(), c->sort.keys[0], c->dev_epoch, c->g, c->n};
        }
        GELL_KERNEL(c0, "k_keys_batch", k_keys_batch<<<kblocks, 256, 0, st>>>(kb));

        // the sort: each member's own digit width and pass count (radix_sort's rule)
        std::vector<int> passes(nf), dbits(nf), in(nf, 0), iota(nf, 1);
        int maxp = 0;
        for (int i = 0; i < nf; ++i) {
            const int bits = key_bits(fm[i]->g.N);
            passes[i] = (bits + 7) / 8 < 1 ? 1 : (bits + 7) / 8;
            dbits[i] = (bits + passes[i] - 1) / passes[i];
            maxp = passes[i] > maxp ? passes[i] : maxp;
        }
        for (int p = 0; p < maxp; ++p) {
            SortBatch sb{};
            std::vector<int> tiles, digits, who;
            for (int i = 0; i < nf; ++i) {
                if (p >= passes[i]) continue;
                gell_ctx* c = fm[i];
                SortScratch& S = c->sort;
                const int nb = (c->n + kSortTile - 1) / kSortTile;
                const int R = 1 << dbits[i];
                sb.job[who.size()] = SortJob{S.keys[in[i]], S.vals[in[i]], S.keys[in[i] ^ 1], S.vals[in[i] ^ 1], S.hist,
                                             c->n, nb, p * dbits[i], R, iota[i]};
                tiles.push_back(nb);
                digits.push_back(R);
                who.push_back(i);
            }
            const int ntiles = fill_map(sb.tiles, tiles);
            const int ndigits = fill_map(sb.digits, digits);
            GELL_KERNEL(c0, "k_hist_batch", k_hist_batch<<<ntiles, kSortThreads, 0, st>>>(sb));
            GELL_KERNEL(c0, "k_digit_scan_batch", k_digit_scan_batch<<<ndigits, kSortThreads, 0, st>>>(sb));
            GELL_KERNEL(c0, "k_scatter_batch", k_scatter_batch<<<ntiles, kSortThreads, 0, st>>>(sb));
            for (int i : who) {
                in[i] ^= 1;
                iota[i] = 0;
            }
        }

        GatherBatch gb{};
        const int gblocks = fill_map(gb.map, blocks);
        for (int i = 0; i < nf; ++i) {
            gell_ctx* c = fm[i];
            c->sort.which = in[i];
            gb.job[i] = GatherJob{c->cur(), c->alt(), c->sort.keys[in[i]], c->sort.vals[in[i]], c->bins, c->dev_epoch,
                                  c->n};
            c->swap_all();
        }
        GELL_KERNEL(c0, "k_gather_batch", k_gather_batch<<<gblocks, 256, 0, st>>>(gb));

        ForceBatch fb{};
        const int fblocks = fill_map(fb.map, blocks);
        for (int i = 0; i < nf; ++i) {
            gell_ctx* c = fm[i];
            MechArgs& a = fb.job[i];
            a.cur = c->cur();
            a.alt = c->alt();
            a.bins = c->bins;
            a.epoch = c->dev_epoch;
            a.n = c->n;
            a.g = c->g;
            a.max_dist = c->P.cc_max_dist;
            a.cccr = c->P.cccr;
            a.ccca = c->P.ccca;
            a.ra_ratio = c->P.ra_ratio;
            a.half_dt = c->P.mechanics_dt / 2.f;
            c->sign.swap();
            c->mesh.swap();
            c->posr.swap();
            c->force.swap();
            c->oldf.swap();
        }
        GELL_KERNEL(c0, "k_force_move_batch", k_force_move_batch<<<fblocks, 256, 0, st>>>(fb));
    }
    for (gell_ctx* c : ms) {
        c->sorted_valid = true;
        c->rate_valid = false;
    }

    // PreLOD of every member with substrates: clear the lines of the last map, reset the line
    // counts, accumulate the new map
    std::vector<gell_ctx*> pm;
    for (gell_ctx* c : ms)
        if (!c->subs.empty()) pm.push_back(c);
    if (!pm.empty()) {
        PreBatch pb{};
        std::vector<int> blocks;
        for (size_t i = 0; i < pm.size(); ++i) {
            gell_ctx* c = pm[i];
            PreJob& j = pb.job[i];
            for (size_t s = 0; s < c->subs.size(); ++s) {
                Substrate& S = c->subs[s];
                j.rate[s] = S.rate;
                j.flag[s] = S.line_flag;
                j.list[s] = S.line_list;
                j.count[s] = S.line_count;
                j.coef[s] = S.s.uptake;
            }
            j.nsub = (int)c->subs.size();
            j.c = c->cur();
            j.g = c->g;
            j.dead = c->P.dead_uptake_factor;
            j.n = c->n;
            // a member without cells launches no k_rate_accum block
            blocks.push_back(c->n > 0 ? blocks_for(c->n, 256) : 0);
        }
        const int ablocks = fill_map(pb.map, blocks);
        GELL_KERNEL(c0, "k_rate_reset_batch",
                    k_rate_reset_batch<<<dim3(kResetBlocks, (unsigned)pm.size()), 256, 0, st>>>(pb));
        GELL_KERNEL(c0, "k_zero_counts_batch", k_zero_counts_batch<<<1, 256, 0, st>>>(pb));
        if (ablocks > 0) GELL_KERNEL(c0, "k_rate_accum_batch", k_rate_accum_batch<<<ablocks, 256, 0, st>>>(pb));
        for (gell_ctx* c : pm) c->rate_valid = true;
    }
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
