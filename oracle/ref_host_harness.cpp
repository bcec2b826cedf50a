// ref_host_harness.cpp — TEST INFRASTRUCTURE ONLY.
//
// The reference's own kernel bodies and façades for mechanics and diffusion (PhantomOtter/Gell,
// include/FMkernel.cuh and include/LODkernel.cuh), compiled for the HOST with g++ -fopenmp: the
// CPU baseline of the large workload.  The reference has no CPU path; this is its GPU code run on
// the host cores, each kernel launch an OpenMP loop over the launch's (block, thread) pairs.
//
// Nothing is copied into this repository.  oracle/make_ref_host.py reads the two headers in place,
// rewrites only the launch syntax (kernel<<<grid, block>>>(args) becomes a call of
// gref_host_launch, oracle/host_shim/gref_host_launch.h) and pipes this file, with those two
// headers spliced in at the marker below, to g++.  The other headers are included unmodified;
// oracle/host_shim/ stands in for the CUDA runtime, curand and Thrust headers.  As in
// ref_harness.cu, Definitions.h is included first and its macros are redefined for the parameter
// set (Voxel_num, Voxel_length, Max_Cell_num, the substrate's boundary value and uptake).
#include "Definitions.h"

#ifdef GREF_N
#undef Voxel_num
#define Voxel_num GREF_N
#endif
#ifdef GREF_LEN
#undef Voxel_length
#define Voxel_length GREF_LEN
#endif
#ifdef GREF_CAP
#undef Max_Cell_num
#define Max_Cell_num GREF_CAP
#endif
#ifdef GREF_BOUNDARY
#undef O2_Default_Concentration
#define O2_Default_Concentration GREF_BOUNDARY
#endif
#ifdef GREF_UPTAKE
#undef Tumor_O2_consumption
#define Tumor_O2_consumption GREF_UPTAKE
#endif

#include "BasicFunctions.cuh"
#include "RandomFunctions.cuh"
#include "Cells.cuh"

// @REFERENCE_HEADERS_WITH_HOST_LAUNCHES@

#include <omp.h>

namespace {
struct HRef {
    Mesh_struct* mesh = nullptr;
    MechanicsMesh_struct* mech = nullptr;
    thrust::device_vector<Cell>* cells = nullptr;
    int n = 0;
};
}  // namespace

extern "C" {

void gref_build_params(int* out_int4, float* out_float4) {
    out_int4[0] = Voxel_num;
    out_int4[1] = Max_Cell_num;
    out_int4[2] = (int)sizeof(Cell);
    out_int4[3] = omp_get_max_threads();
    out_float4[0] = (float)Voxel_length;
    out_float4[1] = O2_Default_Concentration;
    out_float4[2] = Tumor_O2_consumption;
    out_float4[3] = Diffusion_dt;
}

int gref_threads() { return omp_get_max_threads(); }

// Main.cu:63-95 without the RNG states (no random draws on this path)
void* gref_create(float conc, float D, float decay) {
    HRef* g = new HRef;
    g->mesh = new Mesh_struct(conc, D, decay);
    g->mech = new MechanicsMesh_struct();
    g->cells = new thrust::device_vector<Cell>(Max_Cell_num);
    return g;
}

int gref_destroy(void* h) {
    HRef* g = (HRef*)h;
    if (!g) return 0;
    delete g->cells;
    delete g->mech;
    delete g->mesh;
    delete g;
    return 0;
}

int gref_set_cells(void* h, const Cell* cells, int n) {
    HRef* g = (HRef*)h;
    if (n < 0 || n > Max_Cell_num) return -1;
    std::memcpy(static_cast<void*>(g->cells->data()), cells, sizeof(Cell) * (size_t)n);
    g->n = n;
    return 0;
}

int gref_get_cells(void* h, Cell* cells, int n) {
    HRef* g = (HRef*)h;
    if (n < 0 || n > Max_Cell_num) return -1;
    std::memcpy(static_cast<void*>(cells), g->cells->data(), sizeof(Cell) * (size_t)n);
    return 0;
}

int gref_count(void* h) { return ((HRef*)h)->n; }
void* gref_cells_ptr(void* h) { return ((HRef*)h)->cells->data(); }

// MechanicsMesh_struct::FM_update (include/FMkernel.cuh:181-202)
int gref_fm_update(void* h) {
    HRef* g = (HRef*)h;
    g->mech->FM_update(*g->cells, g->n);
    return 0;
}
// Mesh_struct::PreLOD (include/LODkernel.cuh:270-278), on this handle's cells or another's
int gref_prelod(void* h) {
    HRef* g = (HRef*)h;
    g->mesh->PreLOD(g->cells->data(), g->n);
    return 0;
}
int gref_prelod_ptr(void* h, void* cells, int n) {
    ((HRef*)h)->mesh->PreLOD(static_cast<Cell*>(cells), n);
    return 0;
}
// Mesh_struct::LODsolver (include/LODkernel.cuh:280-300), integer substep count
int gref_lodsolver(void* h, int substeps) {
    HRef* g = (HRef*)h;
    for (int s = 0; s < substeps; ++s) g->mesh->LODsolver(g->cells->data(), g->n);
    return 0;
}
int gref_get_field(void* h, float* out) {
    std::memcpy(out, ((HRef*)h)->mesh->p, sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num);
    return 0;
}
int gref_set_field(void* h, const float* in) {
    std::memcpy(((HRef*)h)->mesh->p, in, sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num);
    return 0;
}

}  // extern "C"
