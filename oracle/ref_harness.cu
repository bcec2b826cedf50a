// ref_harness.cu — TEST INFRASTRUCTURE ONLY.
//
// Builds the reference's own kernels and façades (PhantomOtter/Gell, header-only CUDA C++ under
// the reference's include/) into a shared library with a C ABI, so the tests can run the
// reference on the same inputs as gell_b200 and compare.  Nothing in the reference is copied or
// edited: every reference header starts with `#pragma once`, so including Definitions.h first
// and then redefining its macros (Voxel_num, Voxel_length, Max_Cell_num, the substrate's
// boundary value and uptake) sets the parameters every later header is compiled with.  One
// library is built per parameter set by oracle/Makefile into oracle/_ref/.
//
// The host-callable reference functions (Morton code, bin lookup, the Cell model) run on the CPU
// and need no GPU; everything else runs the reference's kernels on the current CUDA device.
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
#include "FMkernel.cuh"
#include "LODkernel.cuh"
#include "PDkernel.cuh"
#include "FileSave.cuh"
#include "Initialization.cuh"

#include <cstdio>
#include <cstring>

namespace {
struct GRef {
    Mesh_struct* mesh = nullptr;
    MechanicsMesh_struct* mech = nullptr;
    thrust::device_vector<Cell>* cells = nullptr;
    curandState* states = nullptr;
    int* gcount = nullptr;
    int n = 0;
};
int ok(cudaError_t e) { return e == cudaSuccess ? 0 : -(int)e; }
}  // namespace

extern "C" {

// ---- parameters this library was built with
void gref_build_params(int* out_int4, float* out_float4) {
    out_int4[0] = Voxel_num;
    out_int4[1] = Max_Cell_num;
    out_int4[2] = (int)sizeof(Cell);
    out_int4[3] = (int)sizeof(curandState);
    out_float4[0] = (float)Voxel_length;
    out_float4[1] = O2_Default_Concentration;
    out_float4[2] = Tumor_O2_consumption;
    out_float4[3] = Diffusion_dt;
}

// ---- host-side reference functions (CPU, no GPU needed)
int gref_morton(int i, int j, int k) { return Morton_encode(i, j, k); }
void gref_find_mesh(const float* pos, int* ijk) {
    int3 r = Find_Mesh(make_float3(pos[0], pos[1], pos[2]), Voxel_length);
    ijk[0] = r.x; ijk[1] = r.y; ijk[2] = r.z;
}
int gref_inside(int i, int j, int k) { return Check_Inside(i, j, k) ? 1 : 0; }
float gref_o2_consume(const Cell* c) { Cell t = *c; return t.O2_consume(); }
void gref_volume_update(Cell* c) { c->Volume_update(); }
int gref_phase_update(Cell* c, float rnd, float o2) { return c->Phase_update_ki67adv(rnd, o2) ? 1 : 0; }
void gref_radius_update(Cell* c) { c->Radius_update(); }

// ---- the reference's snapshot writers and initial spheroid (host code)
int gref_savecsv_cell(const Cell* cells, int n, const char* path) {
    thrust::host_vector<Cell> h(cells, cells + n);
    savecsv_cell(h, n, std::string(path));
    return 0;
}
int gref_init_sphere(unsigned seed, int n, Cell* out) {
    srand(seed);
    thrust::host_vector<Cell> h(n);
    Cell_sphere_Initialization(h, n);
    for (int i = 0; i < n; ++i) out[i] = h[i];
    return 0;
}

// ---- the same Cell member function compiled for and run on the GPU
static __global__ void gref_k_volume(Cell* c, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i].Volume_update();
}
int gref_volume_update_device(Cell* host, int n) {
    Cell* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(Cell) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(d, host, sizeof(Cell) * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        gref_k_volume<<<(n + 255) / 256, 256>>>(d, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(host, d, sizeof(Cell) * (size_t)n, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    return (int)e;
}

// ---- the reference's device state: meshes, cells, RNG (Main.cu:63-95)
void* gref_create(float conc, float D, float decay) {
    GRef* g = new GRef;
    g->mesh = new Mesh_struct(conc, D, decay);
    g->mech = new MechanicsMesh_struct();
    g->cells = new thrust::device_vector<Cell>(Max_Cell_num);
    if (cudaMalloc(&g->states, sizeof(curandState) * (size_t)Max_Cell_num) != cudaSuccess) return nullptr;
    set_random_states<<<(Max_Cell_num + BlockWidth1d - 1) / BlockWidth1d, BlockWidth1d>>>(g->states);
    if (cudaMalloc(&g->gcount, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
    return g;
}

int gref_destroy(void* h) {
    GRef* g = (GRef*)h;
    if (!g) return 0;
    delete g->cells;
    delete g->mech;
    delete g->mesh;
    cudaFree(g->states);
    cudaFree(g->gcount);
    delete g;
    return ok(cudaDeviceSynchronize());
}

int gref_set_cells(void* h, const Cell* host, int n) {
    GRef* g = (GRef*)h;
    if (n < 0 || n > Max_Cell_num) return -1;
    Cell* d = thrust::raw_pointer_cast(g->cells->data());
    int e = ok(cudaMemcpy(d, host, sizeof(Cell) * (size_t)n, cudaMemcpyHostToDevice));
    g->n = n;
    if (!e) e = ok(cudaMemcpy(g->gcount, &n, sizeof(int), cudaMemcpyHostToDevice));
    return e;
}

int gref_get_cells(void* h, Cell* host, int n) {
    GRef* g = (GRef*)h;
    if (n < 0 || n > Max_Cell_num) return -1;
    Cell* d = thrust::raw_pointer_cast(g->cells->data());
    return ok(cudaMemcpy(host, d, sizeof(Cell) * (size_t)n, cudaMemcpyDeviceToHost));
}

int gref_count(void* h) { return ((GRef*)h)->n; }

// MechanicsMesh_struct::FM_update (include/FMkernel.cuh:181-202)
int gref_fm_update(void* h) {
    GRef* g = (GRef*)h;
    g->mech->FM_update(*g->cells, g->n);
    return ok(cudaDeviceSynchronize());
}
int gref_get_keys(void* h, int* out, int n) {
    GRef* g = (GRef*)h;
    return ok(cudaMemcpy(out, g->mech->key, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
}
int gref_get_se(void* h, int* s, int* e) {
    GRef* g = (GRef*)h;
    size_t nb = sizeof(int) * (size_t)Voxel_num * Voxel_num * Voxel_num;
    int r = ok(cudaMemcpy(s, g->mech->Mech_Mesh_s, nb, cudaMemcpyDeviceToHost));
    if (!r) r = ok(cudaMemcpy(e, g->mech->Mech_Mesh_e, nb, cudaMemcpyDeviceToHost));
    return r;
}

// Mesh_struct::PreLOD / LODsolver (include/LODkernel.cuh:270-300), integer substep count
int gref_prelod(void* h) {
    GRef* g = (GRef*)h;
    g->mesh->PreLOD(thrust::raw_pointer_cast(g->cells->data()), g->n);
    return ok(cudaDeviceSynchronize());
}
int gref_lodsolver(void* h, int substeps) {
    GRef* g = (GRef*)h;
    for (int s = 0; s < substeps; ++s) g->mesh->LODsolver(thrust::raw_pointer_cast(g->cells->data()), g->n);
    return ok(cudaDeviceSynchronize());
}
int gref_get_field(void* h, float* out) {
    GRef* g = (GRef*)h;
    size_t nb = sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num;
    return ok(cudaMemcpy(out, g->mesh->p, nb, cudaMemcpyDeviceToHost));
}
int gref_set_field(void* h, const float* in) {
    GRef* g = (GRef*)h;
    size_t nb = sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num;
    return ok(cudaMemcpy(g->mesh->p, in, nb, cudaMemcpyHostToDevice));
}
// Mesh_struct::PreLOD on cells held by another handle (a second substrate is a second build of the
// reference: its mesh takes the cells the first build's FM_update moved), and their device address
void* gref_cells_ptr(void* h) { return thrust::raw_pointer_cast(((GRef*)h)->cells->data()); }
int gref_prelod_ptr(void* h, void* dev_cells, int n) {
    GRef* g = (GRef*)h;
    g->mesh->PreLOD(static_cast<Cell*>(dev_cells), n);
    return ok(cudaDeviceSynchronize());
}

// CUDA events on the legacy default stream, where every reference façade runs
void* gref_event_create() {
    cudaEvent_t e = nullptr;
    return cudaEventCreate(&e) == cudaSuccess ? (void*)e : nullptr;
}
int gref_event_record(void* e) { return ok(cudaEventRecord((cudaEvent_t)e, 0)); }
float gref_event_elapsed_ms(void* a, void* b) {
    if (cudaEventSynchronize((cudaEvent_t)b) != cudaSuccess) return -1.f;
    float ms = -1.f;
    return cudaEventElapsedTime(&ms, (cudaEvent_t)a, (cudaEvent_t)b) == cudaSuccess ? ms : -1.f;
}
void gref_event_destroy(void* e) { cudaEventDestroy((cudaEvent_t)e); }
int gref_sync() { return ok(cudaDeviceSynchronize()); }
// page-locked host memory for the cells copied in and out around each step
void* gref_host_alloc(size_t bytes) {
    void* p = nullptr;
    return cudaMallocHost(&p, bytes) == cudaSuccess ? p : nullptr;
}
void gref_host_free(void* p) { cudaFreeHost(p); }

int gref_get_rate(void* h, float* out) {
    GRef* g = (GRef*)h;
    size_t nb = sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num;
    return ok(cudaMemcpy(out, g->mesh->p_rate, nb, cudaMemcpyDeviceToHost));
}
int gref_set_rate(void* h, const float* in) {
    GRef* g = (GRef*)h;
    size_t nb = sizeof(float) * (size_t)Voxel_num * Voxel_num * Voxel_num;
    return ok(cudaMemcpy(g->mesh->p_rate, in, nb, cudaMemcpyHostToDevice));
}
int gref_get_ef(void* h, float* E, float* F) {
    GRef* g = (GRef*)h;
    int r = ok(cudaMemcpy(E, g->mesh->E, sizeof(float) * Voxel_num, cudaMemcpyDeviceToHost));
    if (!r) r = ok(cudaMemcpy(F, g->mesh->F, sizeof(float) * Voxel_num, cudaMemcpyDeviceToHost));
    return r;
}

// CellBirth_kernel / CellDeath_kernel (include/PDkernel.cuh:88-117); return the new count
int gref_birth(void* h) {
    GRef* g = (GRef*)h;
    g->n = CellBirth_kernel(g->mesh->p, *g->cells, g->states, g->n, g->gcount);
    return g->n;
}
int gref_death(void* h) {
    GRef* g = (GRef*)h;
    g->n = CellDeath_kernel(*g->cells, g->states, g->n, g->gcount);
    return g->n;
}

// ---- timing of the façades with CUDA events (ms per call, mean over `iters` after `warm`)
static float time_it(int warm, int iters, void (*f)(GRef*), GRef* g) {
    for (int i = 0; i < warm; ++i) f(g);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    for (int i = 0; i < iters; ++i) f(g);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return iters > 0 ? ms / iters : 0.f;
}
static void f_fm(GRef* g) { g->mech->FM_update(*g->cells, g->n); }
static void f_prelod(GRef* g) { g->mesh->PreLOD(thrust::raw_pointer_cast(g->cells->data()), g->n); }
static void f_lod(GRef* g) { g->mesh->LODsolver(thrust::raw_pointer_cast(g->cells->data()), g->n); }
// savecsv_mesh / savecsv_meshslice of the mesh's current field (include/FileSave.cuh:35-64)
int gref_savecsv_mesh(void* h, const char* path) {
    GRef* g = (GRef*)h;
    g->mesh->move_to_CPU();
    savecsv_mesh(g->mesh, std::string(path));
    return (int)cudaGetLastError();
}
int gref_savecsv_meshslice(void* h, const char* path) {
    GRef* g = (GRef*)h;
    g->mesh->Slice_to_CPU();
    savecsv_meshslice(g->mesh, std::string(path));
    return (int)cudaGetLastError();
}
float gref_time_fm(void* h, int warm, int iters) { return time_it(warm, iters, f_fm, (GRef*)h); }
float gref_time_prelod(void* h, int warm, int iters) { return time_it(warm, iters, f_prelod, (GRef*)h); }
float gref_time_lod(void* h, int warm, int iters) { return time_it(warm, iters, f_lod, (GRef*)h); }

}  // extern "C"
