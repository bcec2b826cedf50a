// gell_compat.hpp — the reference's host-loop vocabulary on top of the C ABI (gell.h).
//
// The reference (PhantomOtter/Gell) drives its hot path from Main.cu through these names:
//   MechanicsMesh_struct MecMesh;            MecMesh.FM_update(GpuCell, currentnum);
//   Mesh_struct O2Mesh(conc, D, decay);      O2Mesh.PreLOD(GC, n);  O2Mesh.LODsolver(GC, n);
//   currentnum = CellBirth_kernel(O2Mesh.p, GpuCell, curand_states, currentnum, gcurrentnum);
//   currentnum = CellDeath_kernel(GpuCell, curand_states, currentnum, gcurrentnum);
// (Main.cu:63-128, include/FMkernel.cuh:160-202, include/LODkernel.cuh:192-300,
//  include/PDkernel.cuh:88-117).  Here the cells, the meshes and the RNG states live in one
// gell::Context; the classes below keep the reference's names and call order so a
// reference-shaped loop keeps its shape.  Errors throw gell::Error (the reference has none).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "gell.h"

namespace gell {

struct Error : std::runtime_error {
    gell_status status;
    Error(gell_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(gell_status s, gell_ctx* c, const char* what) {
    if (s != GELL_OK) {
        std::string msg = std::string(what) + ": " + gell_status_string(s);
        if (c) msg += std::string(" (") + gell_last_error(c) + ")";
        throw Error(s, msg);
    }
}

// The reference's compile-time parameter set (include/Definitions.h), at run time.
inline gell_params reference_params() {
    gell_params p;
    gell_params_default(&p);
    return p;
}

// Owns the device state: cells (up to max_cell_num), substrates, RNG states, cell list.
class Context {
public:
    explicit Context(const gell_params& p) : params_(p) { check(gell_create(&p, &h_), nullptr, "gell_create"); }
    ~Context() {
        if (h_) gell_destroy(h_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    gell_ctx* get() const { return h_; }
    const gell_params& params() const { return params_; }
    size_t voxels() const { return (size_t)params_.voxel_num * params_.voxel_num * params_.voxel_num; }

    // GpuCell = CpuCell (Main.cu:91-92)
    void cells_from_host(const std::vector<gell_cell>& cells) {
        check(gell_cells_import(h_, cells.data(), (int)cells.size(), 0), h_, "gell_cells_import");
    }
    void cells_from_device(const gell_cell* dev, int n) {
        check(gell_cells_import(h_, dev, n, 1), h_, "gell_cells_import");
    }
    // CpuCell = GpuCell (Main.cu:151)
    std::vector<gell_cell> cells_to_host() const {
        int n = count();
        std::vector<gell_cell> out((size_t)n);
        check(gell_cells_export(h_, out.data(), n, &n, 0), h_, "gell_cells_export");
        out.resize((size_t)n);
        return out;
    }
    int count() const {
        int n = 0;
        check(gell_cell_count(h_, &n), h_, "gell_cell_count");
        return n;
    }
    void sync() const { check(gell_sync(h_), h_, "gell_sync"); }

private:
    gell_params params_;
    gell_ctx* h_ = nullptr;
};

// MechanicsMesh_struct (include/FMkernel.cuh:160-212): the cell list lives in the context.
class MechanicsMesh_struct {
public:
    explicit MechanicsMesh_struct(Context& c) : c_(c) {}
    // FM_update(GpuCell, num): the context knows the cells and their count
    void FM_update(int /*num*/ = 0) { check(gell_fm_update(c_.get()), c_.get(), "FM_update"); }

private:
    Context& c_;
};

// Mesh_struct (include/LODkernel.cuh:192-300) for one substrate.  The reference fixes the
// boundary value and uptake to oxygen's; here they are arguments (oxygen's by default).
class Mesh_struct {
public:
    Mesh_struct(Context& c, float concentration, float D, float decay, float boundary = 38.f,
                float uptake = -10.f)
        : c_(c) {
        gell_substrate s{boundary, D, decay, uptake, concentration};
        check(gell_substrate_add(c_.get(), &s, &index_), c_.get(), "Mesh_struct");
    }
    int index() const { return index_; }
    void PreLOD(int /*num*/ = 0) { check(gell_prelod(c_.get(), index_), c_.get(), "PreLOD"); }
    // one LODsolver call = one substep (the reference's loop calls it per Diffusion_dt)
    void LODsolver(int /*num*/ = 0) { check(gell_lod_solver(c_.get(), index_, 1), c_.get(), "LODsolver"); }
    void LODsolver_substeps(int k) { check(gell_lod_solver(c_.get(), index_, k), c_.get(), "LODsolver"); }
    // move_to_CPU / move_to_GPU (include/LODkernel.cuh:302-309): the dense N^3 field, x fastest
    std::vector<float> move_to_CPU() const {
        std::vector<float> f(c_.voxels());
        check(gell_field_export(c_.get(), index_, f.data(), 0), c_.get(), "move_to_CPU");
        return f;
    }
    void move_to_GPU(const std::vector<float>& f) {
        if (f.size() != c_.voxels()) throw Error(GELL_ERR_INVALID_ARG, "move_to_GPU: field size is not N^3");
        check(gell_field_import(c_.get(), index_, f.data(), 0), c_.get(), "move_to_GPU");
    }

private:
    Context& c_;
    int index_ = -1;
};

// `steps` mechanics steps of FM_update, PreLOD and `substeps` LOD substeps (Main.cu:114-124 with an
// integer count), pairs of them replayed from a captured CUDA graph.
inline void run_mechanics(Context& c, int steps, int substeps = 10) {
    check(gell_run_mechanics(c.get(), steps, substeps), c.get(), "run_mechanics");
}

// CellBirth_kernel / CellDeath_kernel (include/PDkernel.cuh:88-117): return the new count.
inline int CellBirth_kernel(Context& c) {
    int n = 0;
    check(gell_cell_birth(c.get(), &n), c.get(), "CellBirth_kernel");
    return n;
}
inline int CellDeath_kernel(Context& c) {
    int n = 0;
    check(gell_cell_death(c.get(), &n), c.get(), "CellDeath_kernel");
    return n;
}

// The reference's time loop (Main.cu:108-128) with integer counts: every biology step is birth,
// then `mech_per_bio` mechanics steps (each with `substeps` LOD substeps of every substrate), then
// death.  Returns the final cell count.
inline int run(Context& c, int bio_steps, int mech_per_bio = 60, int substeps = 10) {
    int n = c.count();
    for (int b = 0; b < bio_steps; ++b) {
        CellBirth_kernel(c);
        run_mechanics(c, mech_per_bio, substeps);
        n = CellDeath_kernel(c);
    }
    return n;
}

}  // namespace gell
