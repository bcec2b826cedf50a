// io.cu — host-side input/output around the hot path: the reference's CSV snapshots, a binary
// checkpoint that resumes a run bit for bit, and the reference's initial spheroid.
//
//   gell_write_cells_csv / gell_save_cells_csv   savecsv_cell (include/FileSave.cuh:24-33)
//   gell_save_field_csv                          savecsv_mesh (include/FileSave.cuh:35-49)
//   gell_save_field_slice_csv                    savecsv_meshslice of the slice GPU_Get_Slice takes,
//                                                z = N/2 (include/FileSave.cuh:50-64,
//                                                include/LODkernel.cuh:174-181)
//   gell_checkpoint_save / _load                 no counterpart (the reference writes CSV only)
//   gell_reference_spheroid                      Cell_sphere_Initialization
//                                                (include/Initialization.cuh:15-43)
// The CSV writers print with the reference's format strings, so equal data gives equal files.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "gell_internal.cuh"

namespace gell {
namespace {

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

// The C library's rand() as the reference's host build calls it (glibc's default generator: an
// additive lagged-Fibonacci sequence o_i = o_{i-3} + o_{i-31} mod 2^32 over a table filled by the
// Lehmer generator 16807 x mod (2^31 - 1), the first 310 outputs discarded, results shifted right
// by one), kept in an object of its own so no process-wide state is touched.
class LibcRand {
public:
    explicit LibcRand(uint32_t seed) {
        int32_t r[34];
        r[0] = seed == 0 ? 1 : (int32_t)seed;
        for (int i = 1; i < 31; ++i) {
            // 16807 * r mod (2^31 - 1) without overflow (Schrage's decomposition)
            const int32_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
            int32_t w = 16807 * lo - 2836 * hi;
            if (w < 0) w += 2147483647;
            r[i] = w;
        }
        for (int i = 0; i < 31; ++i) t_[i] = (uint32_t)r[i];
        k_ = 3;  // the first sum is t[3] += t[0]
        for (int i = 0; i < 310; ++i) next();
    }
    int next() {
        // ring of the last 31 values: t_[k_] is o_{i-31}, t_[(k_ + 28) % 31] is o_{i-3}
        const uint32_t o = t_[k_] + t_[(k_ + 28) % 31];
        t_[k_] = o;
        k_ = (k_ + 1) % 31;
        return (int)(o >> 1);
    }

private:
    uint32_t t_[31];
    int k_;
};

constexpr char kMagic[8] = {'G', 'E', 'L', 'L', 'C', 'K', 'P', '1'};

// Field by field: the record has a hole before the double-typed rates that callers need not clear.
bool same_params(const gell_params& a, const gell_params& b) {
    return a.voxel_num == b.voxel_num && a.voxel_length == b.voxel_length && a.max_cell_num == b.max_cell_num &&
           a.mechanics_dt == b.mechanics_dt && a.diffusion_dt == b.diffusion_dt && a.biology_dt == b.biology_dt &&
           a.ccca == b.ccca && a.cccr == b.cccr && a.ra_ratio == b.ra_ratio && a.cc_max_dist == b.cc_max_dist &&
           a.dead_uptake_factor == b.dead_uptake_factor && a.default_v == b.default_v &&
           a.o2_prolif_thres == b.o2_prolif_thres && a.o2_prolif_sat == b.o2_prolif_sat &&
           a.o2_necrosis_thres == b.o2_necrosis_thres && a.o2_necrosis_max == b.o2_necrosis_max &&
           a.necrosis_rate == b.necrosis_rate && a.apoptosis_rate == b.apoptosis_rate &&
           a.proliferation_rate == b.proliferation_rate && a.duration_pre2post == b.duration_pre2post &&
           a.duration_post2q == b.duration_post2q && a.o2_substrate == b.o2_substrate && a.rng_mode == b.rng_mode &&
           a.mech_mode == b.mech_mode && a.seed == b.seed;
}

}  // namespace
}  // namespace gell

using namespace gell;

extern "C" {

gell_status gell_write_cells_csv(const gell_cell* cells, int n, const char* path) {
    if (!path || n < 0 || (n > 0 && !cells)) return GELL_ERR_INVALID_ARG;
    File out(path, "w");
    if (!out.f) return GELL_ERR_INVALID_ARG;
    std::fprintf(out.f, "%s,%s,%s,%s,%s,%s,%s,%s,%s,%s\n", "Index", "Sign", "Phase", "x", "y", "z", "r", "V", "Vns",
                 "Vcs");
    for (int i = 0; i < n; ++i) {
        const gell_cell& c = cells[i];
        std::fprintf(out.f, "%d,%d,%d,%f,%f,%f,%f,%f,%f,%f\n", i, (int)(c.sign != 0), c.phase, c.pos[0], c.pos[1],
                     c.pos[2], c.r, c.V, c.Vns, c.Vcs);
    }
    return std::ferror(out.f) ? GELL_ERR_INVALID_ARG : GELL_OK;
}

gell_status gell_save_cells_csv(gell_ctx* c, const char* path) {
    if (!c || !path) return GELL_ERR_INVALID_ARG;
    std::vector<gell_cell> cells((size_t)(c->n > 0 ? c->n : 1));
    int n = 0;
    gell_status st = gell_cells_export(c, cells.data(), (int)cells.size(), &n, 0);
    if (st != GELL_OK) return st;
    return gell_write_cells_csv(cells.data(), n, path);
}

gell_status gell_save_field_csv(gell_ctx* c, int substrate, const char* path) {
    if (!c || !path || substrate < 0 || substrate >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    const int N = c->g.N;
    std::vector<float> f((size_t)c->nvox);
    gell_status st = gell_field_export(c, substrate, f.data(), 0);
    if (st != GELL_OK) return st;
    File out(path, "w");
    if (!out.f) return fail(c, GELL_ERR_INVALID_ARG, "cannot open the CSV file");
    std::fprintf(out.f, "%s,%s,%s,%s\n", "i", "j", "k", "Concentration");
    size_t idx = 0;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) std::fprintf(out.f, "%d,%d,%d,%f\n", i, j, k, f[idx++]);
    return GELL_OK;
}

gell_status gell_save_field_slice_csv(gell_ctx* c, int substrate, const char* path) {
    if (!c || !path || substrate < 0 || substrate >= (int)c->subs.size()) return GELL_ERR_INVALID_ARG;
    const int N = c->g.N;
    std::vector<float> f((size_t)c->nvox);
    gell_status st = gell_field_export(c, substrate, f.data(), 0);
    if (st != GELL_OK) return st;
    File out(path, "w");
    if (!out.f) return fail(c, GELL_ERR_INVALID_ARG, "cannot open the CSV file");
    std::fprintf(out.f, "%s,%s,%s\n", "x", "y", "Concentration");
    const size_t z = (size_t)(N / 2);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) std::fprintf(out.f, "%d,%d,%f\n", i, j, f[(size_t)i + (size_t)j * N + z * N * N]);
    return GELL_OK;
}

// Layout: magic, the gell_params record, substrate count and records, cell count, the device
// epoch and biology step, the cells (72-byte records), every field (N^3 floats, x fastest), and
// with XORWOW draws the generator state of every slot.
gell_status gell_checkpoint_save(gell_ctx* c, const char* path) {
    GELL_RANGE("gell_checkpoint_save");
    if (!c || !path) return GELL_ERR_INVALID_ARG;
    if (gell_status st = gell_sync(c)) return st;
    const int32_t nsub = (int32_t)c->subs.size(), n = c->n;
    int32_t epoch = 0;
    GELL_CUDA(c, cudaMemcpy(&epoch, c->dev_epoch, 4, cudaMemcpyDeviceToHost));
    std::vector<gell_cell> cells((size_t)(n > 0 ? n : 1));
    int got = 0;
    if (gell_status st = gell_cells_export(c, cells.data(), (int)cells.size(), &got, 0)) return st;
    File out(path, "wb");
    if (!out.f) return fail(c, GELL_ERR_INVALID_ARG, "cannot open the checkpoint file");
    bool ok = std::fwrite(kMagic, 8, 1, out.f) == 1 && std::fwrite(&c->P, sizeof(gell_params), 1, out.f) == 1 &&
              std::fwrite(&nsub, 4, 1, out.f) == 1;
    for (int s = 0; ok && s < nsub; ++s) ok = std::fwrite(&c->subs[s].s, sizeof(gell_substrate), 1, out.f) == 1;
    const uint32_t bio = c->bio_step;
    ok = ok && std::fwrite(&n, 4, 1, out.f) == 1 && std::fwrite(&epoch, 4, 1, out.f) == 1 &&
         std::fwrite(&bio, 4, 1, out.f) == 1;
    if (ok && n > 0) ok = std::fwrite(cells.data(), sizeof(gell_cell), (size_t)n, out.f) == (size_t)n;
    std::vector<float> f((size_t)c->nvox);
    for (int s = 0; ok && s < nsub; ++s) {
        if (gell_status st = gell_field_export(c, s, f.data(), 0)) return st;
        ok = std::fwrite(f.data(), 4, f.size(), out.f) == f.size();
    }
    if (ok && c->xorwow) {
        std::vector<curandState> states((size_t)c->cap);
        GELL_CUDA(c, cudaMemcpy(states.data(), c->xorwow, states.size() * sizeof(curandState), cudaMemcpyDeviceToHost));
        ok = std::fwrite(states.data(), sizeof(curandState), states.size(), out.f) == states.size();
    }
    if (!ok) return fail(c, GELL_ERR_INVALID_ARG, "writing the checkpoint failed");
    return GELL_OK;
}

gell_status gell_checkpoint_load(gell_ctx* c, const char* path) {
    GELL_RANGE("gell_checkpoint_load");
    if (!c || !path) return GELL_ERR_INVALID_ARG;
    File in(path, "rb");
    if (!in.f) return fail(c, GELL_ERR_INVALID_ARG, "cannot open the checkpoint file");
    char magic[8];
    gell_params P;
    int32_t nsub = 0;
    if (std::fread(magic, 8, 1, in.f) != 1 || std::memcmp(magic, kMagic, 8) != 0 ||
        std::fread(&P, sizeof(P), 1, in.f) != 1 || std::fread(&nsub, 4, 1, in.f) != 1)
        return fail(c, GELL_ERR_INVALID_ARG, "not a gell_b200 checkpoint");
    if (!same_params(P, c->P)) return fail(c, GELL_ERR_STATE, "checkpoint parameters differ from the context's");
    if (nsub != (int32_t)c->subs.size()) return fail(c, GELL_ERR_STATE, "checkpoint substrate count differs");
    for (int s = 0; s < nsub; ++s) {
        gell_substrate d;
        if (std::fread(&d, sizeof(d), 1, in.f) != 1) return fail(c, GELL_ERR_INVALID_ARG, "checkpoint truncated");
        if (std::memcmp(&d, &c->subs[s].s, sizeof(d)) != 0)
            return fail(c, GELL_ERR_STATE, "checkpoint substrate differs from the context's");
    }
    int32_t n = 0, epoch = 0;
    uint32_t bio = 0;
    if (std::fread(&n, 4, 1, in.f) != 1 || std::fread(&epoch, 4, 1, in.f) != 1 || std::fread(&bio, 4, 1, in.f) != 1 ||
        n < 0 || n > c->cap)
        return fail(c, GELL_ERR_INVALID_ARG, "checkpoint truncated or too many cells");
    std::vector<gell_cell> cells((size_t)(n > 0 ? n : 1));
    if (n > 0 && std::fread(cells.data(), sizeof(gell_cell), (size_t)n, in.f) != (size_t)n)
        return fail(c, GELL_ERR_INVALID_ARG, "checkpoint truncated");
    std::vector<float> f((size_t)c->nvox);
    std::vector<std::vector<float>> fields;
    for (int s = 0; s < nsub; ++s) {
        if (std::fread(f.data(), 4, f.size(), in.f) != f.size()) return fail(c, GELL_ERR_INVALID_ARG, "checkpoint truncated");
        fields.push_back(f);
    }
    std::vector<curandState> states;
    if (c->xorwow) {
        states.resize((size_t)c->cap);
        if (std::fread(states.data(), sizeof(curandState), states.size(), in.f) != states.size())
            return fail(c, GELL_ERR_INVALID_ARG, "checkpoint truncated");
    }
    if (gell_status st = gell_cells_import(c, cells.data(), n, 0)) return st;
    for (int s = 0; s < nsub; ++s)
        if (gell_status st = gell_field_import(c, s, fields[s].data(), 0)) return st;
    if (c->xorwow)
        GELL_CUDA(c, cudaMemcpyAsync(c->xorwow, states.data(), states.size() * sizeof(curandState),
                                     cudaMemcpyHostToDevice, c->stream));
    GELL_CUDA(c, cudaMemcpyAsync(c->dev_epoch, &epoch, 4, cudaMemcpyHostToDevice, c->stream));
    c->bio_step = bio;
    return gell_sync(c);
}

gell_status gell_reference_spheroid(const gell_params* p, int n, float cell_radius, uint32_t seed, gell_cell* out) {
    if (!p || n < 0 || (n > 0 && !out)) return GELL_ERR_INVALID_ARG;
    const int N = p->voxel_num;
    const float len = p->voxel_length;
    const float middle = N * len / 2;
    const float radius = cell_radius;
    const float ballr = (float)(radius * std::pow((double)n, 1.0 / 3) / 1.612 * 1.87);
    LibcRand rng(seed);
    for (int i = 0; i < n;) {
        const float x = 2.f * ((float)rng.next()) / 2147483647 - 1.f;
        const float y = 2.f * ((float)rng.next()) / 2147483647 - 1.f;
        const float z = 2.f * ((float)rng.next()) / 2147483647 - 1.f;
        if (x * x + y * y + z * z < 1) {
            gell_cell& c = out[i];
            std::memset(&c, 0, sizeof(c));
            c.sign = 1;
            c.pos[0] = middle + x * ballr;
            c.pos[1] = middle + y * ballr;
            c.pos[2] = middle + z * ballr;
            c.r = radius;
            c.phase = 0;
            c.V = p->default_v;
            c.Vf = 1871;
            c.Vns = 135;
            c.Vcs = 489;
            c.cell_clock = 0.f;
            const int bx = (int)(c.pos[0] / len), by = (int)(c.pos[1] / len), bz = (int)(c.pos[2] / len);
            c.mesh_idx = bx + by * N + bz * N * N;
            ++i;
        }
    }
    return GELL_OK;
}

}  // extern "C"
