/*
 * gell.h — C ABI of gell_b200, a B200 (sm_100a) implementation of the Gell per-timestep hot path:
 * Morton-sorted cell-list mechanics (FM), LOD x/y/z Thomas reaction-diffusion with cell uptake
 * (LOD) and stochastic Ki-67 birth/death with stream compaction (PD).
 *
 * The reference (PhantomOtter/Gell) is a header-only CUDA C++ program with no FFI.  Its entry
 * points are C++ member functions and free functions that take thrust::device_vector<Cell>&;
 * each function below names the reference interface it replaces (file:line in the reference
 * project).  Everything here is plain C: opaque context, plain pointers and sizes, status codes.
 *
 * Conventions
 *   - Every call returns gell_status (0 = ok, negative = error).  The message of the last error
 *     of a context is available from gell_last_error().
 *   - Calls are ordered on the context's CUDA stream (gell_set_stream).  Calls that return a
 *     host-visible value (a cell count, an exported buffer on the host) synchronise that stream;
 *     the others do not.
 *   - A context is not thread-safe: one host thread drives it at a time.
 *   - Device pointers passed in must be on the context's device.
 */
#ifndef GELL_B200_GELL_H
#define GELL_B200_GELL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GELL_ABI_VERSION 1

typedef enum gell_status {
    GELL_OK = 0,
    GELL_ERR_INVALID_ARG = -1,   /* bad pointer, size or parameter */
    GELL_ERR_CAPACITY = -2,      /* more cells than max_cell_num */
    GELL_ERR_CUDA = -3,          /* a CUDA runtime call failed; see gell_last_error */
    GELL_ERR_NO_DEVICE = -4,     /* no CUDA device visible */
    GELL_ERR_TIMEOUT = -5,       /* a bounded device-side wait gave up */
    GELL_ERR_STATE = -6,         /* call not valid in the current context state */
    GELL_ERR_UNSUPPORTED = -7,   /* parameter outside what this build supports */
    GELL_ERR_ALLOC = -8          /* device or host allocation failed */
} gell_status;

/*
 * One cell, byte-for-byte the reference's `struct Cell` (include/Cells.cuh:9-47), 72 bytes:
 * sign@0 (bool), mesh_idx@4, pos@8, force@20, oldforce@32, r@44, V@48, Vf@52, Vcs@56, Vns@60,
 * phase@64, cell_clock@68.  Import/export use this layout so a reference host loop can hand its
 * thrust::device_vector<Cell> storage (or a host copy) straight to gell_cells_import/export.
 */
typedef struct gell_cell {
    uint8_t sign;          /* alive flag (reference: bool sign) */
    uint8_t _pad[3];
    int32_t mesh_idx;      /* x + y*N + z*N*N of the cell's voxel */
    float pos[3];          /* um */
    float force[3];
    float oldforce[3];
    float r;               /* radius, um */
    float V, Vf, Vcs, Vns; /* total, fluid, cytoplasmic, nuclear volume, um^3 */
    int32_t phase;         /* 0 quiescent,1 premitotic,2 postmitotic,3 apoptotic,4/5 necrotic,-1 unused */
    float cell_clock;      /* min */
} gell_cell;

/* RNG used by the birth step. */
typedef enum gell_rng_mode {
    GELL_RNG_XORWOW = 0,   /* curand XORWOW, one state per array slot, curand_init(seed, slot, 0):
                              the reference's draws (include/RandomFunctions.cuh:13-31) */
    GELL_RNG_PHILOX = 1    /* stateless Philox4x32-10 keyed by (seed), counter (slot, step, draw) */
} gell_rng_mode;

/* Mechanics neighbour search mode. */
typedef enum gell_mech_mode {
    GELL_MECH_REFERENCE = 0,  /* 27 bins of size voxel_length and the reference's order-dependent
                                 cutoff (include/FMkernel.cuh:56-118), reproduced exactly */
} gell_mech_mode;

/*
 * Runtime parameter set.  The reference has these as compile-time #defines
 * (include/Definitions.h:7-47 and the literals inside include/Cells.cuh); gell_params_default()
 * fills in exactly those values.  Types follow the reference: the rates that are double-typed
 * macros there are double here, because the reference evaluates their products in double.
 */
typedef struct gell_params {
    int32_t voxel_num;            /* Voxel_num: grid edge N, same on all axes (4..1023) */
    float voxel_length;           /* Voxel_length: voxel and mechanics bin edge, um */
    int32_t max_cell_num;         /* Max_Cell_num: cell capacity */
    float mechanics_dt;           /* Mechanics_dt, min */
    float diffusion_dt;           /* Diffusion_dt, min */
    float biology_dt;             /* Biology_dt, min */
    /* force law (include/FMkernel.cuh:56-118) */
    float ccca;                   /* Ccca: adhesion coefficient */
    float cccr;                   /* Cccr: repulsion coefficient */
    double ra_ratio;              /* Ra_ratio: interaction cutoff / (r_i + r_j) */
    float cc_max_dist;            /* Tumor_CC_Max_Dist: initial cutoff of each cell's scan */
    /* cell model (include/Cells.cuh:74-223) */
    float dead_uptake_factor;     /* Dead_O2_consumption_factor */
    float default_v;              /* Default_V */
    float o2_prolif_thres;        /* Tumor_O2_Proliferation_Thres */
    float o2_prolif_sat;          /* Tumor_O2_Proliferation_Sat */
    float o2_necrosis_thres;      /* Tumor_Necrosis_02_Thres */
    float o2_necrosis_max;        /* Tumor_Necrosis_02_Max */
    double necrosis_rate;         /* Tumor_Necrosis_Rate, 1/min */
    double apoptosis_rate;        /* Tumor_Apoptosis_rate, 1/min */
    double proliferation_rate;    /* Tumor_Proliferation_Rate, 1/min */
    float duration_pre2post;      /* duration_pre2post, min */
    float duration_post2q;        /* duration_post2q, min */
    /* which substrate drives the Ki-67 model (the reference's oxygen mesh) */
    int32_t o2_substrate;
    int32_t rng_mode;             /* gell_rng_mode */
    int32_t mech_mode;            /* gell_mech_mode */
    int32_t _reserved0;
    uint64_t seed;                /* 123 in the reference (include/RandomFunctions.cuh:21) */
} gell_params;

/*
 * One diffusing substrate.  The reference hard-wires oxygen: boundary and uptake come from
 * O2_Default_Concentration / Tumor_O2_consumption (include/LODkernel.cuh:41-49,80-88,100-108,288,
 * include/Cells.cuh:74-89); D and decay are the Mesh_struct constructor arguments
 * (include/LODkernel.cuh:205).
 */
typedef struct gell_substrate {
    float boundary;   /* Dirichlet value on the two outer layers of all six faces */
    float diffusion;  /* D, um^2/min */
    float decay;      /* lambda, 1/min */
    float uptake;     /* per-cell rate coefficient (negative = consumption), reference: -10 */
    float init;       /* initial field value */
} gell_substrate;

typedef struct gell_ctx gell_ctx;

/* Fill *p with the reference's compile-time values (include/Definitions.h:7-47). */
void gell_params_default(gell_params* p);
/* Oxygen as the reference defines it (include/Definitions.h:21-24). */
void gell_substrate_oxygen(gell_substrate* s);

/* Create a context on the current CUDA device: allocates every device buffer for
 * max_cell_num cells and the N^3 grid.  Replaces the constructors MechanicsMesh_struct()
 * (include/FMkernel.cuh:167-172) and the RNG set-up set_random_states (include/RandomFunctions.cuh:13,
 * Main.cu:72-74); when rng_mode is XORWOW the per-slot states are initialised here. */
gell_status gell_create(const gell_params* params, gell_ctx** out);
gell_status gell_destroy(gell_ctx* ctx);

/* Use `stream` (a cudaStream_t) for every later call; NULL selects the context's own stream. */
gell_status gell_set_stream(gell_ctx* ctx, void* stream);

/* Add a substrate field initialised to s->init.  Replaces Mesh_struct(float, float, float)
 * including its host LU prefactor Mesh_initialize (include/LODkernel.cuh:205-259). */
gell_status gell_substrate_add(gell_ctx* ctx, const gell_substrate* s, int* index_out);

/* Load n cells (72-byte gell_cell records) from host or device memory; replaces the
 * GpuCell = CpuCell copy of the reference host loop (Main.cu:91-92). */
gell_status gell_cells_import(gell_ctx* ctx, const gell_cell* cells, int n, int cells_on_device);
/* Write the current cells to `cells` (room for `capacity` records, host or device) and the
 * count to *n_out; replaces CpuCell = GpuCell (Main.cu:151). Synchronises when on host. */
gell_status gell_cells_export(gell_ctx* ctx, gell_cell* cells, int capacity, int* n_out,
                              int cells_on_device);
/* Queued host transfers of the cells: gell_cells_import / gell_cells_export with host memory, but
 * returning at once.  The copy runs on a transfer stream of the context, after the last queued work
 * that uses the cells (fm_update, prelod, birth, death, another transfer), and the next such work
 * waits for it; the LOD substeps do not use the cells, so a transfer queued after prelod overlaps
 * them.  `cells` should be pinned host memory for the copy to overlap.  It must stay valid (and,
 * for an import, unchanged) until the transfer has finished: after gell_sync, or in stream order
 * after gell_wait_transfers.  No counterpart in the reference (its host loop copies synchronously,
 * Main.cu:91-92,151). */
gell_status gell_cells_import_async(gell_ctx* ctx, const gell_cell* cells, int n);
gell_status gell_cells_export_async(gell_ctx* ctx, gell_cell* cells, int capacity, int* n_out);
/* Make the context's stream wait (without blocking the host) for every queued transfer. */
gell_status gell_wait_transfers(gell_ctx* ctx);

/* Current cell count (the reference's host `currentnum`).  No synchronisation. */
gell_status gell_cell_count(gell_ctx* ctx, int* n_out);

/* Dense N^3 float field, x fastest (index x + y*N + z*N*N): replaces move_to_GPU / move_to_CPU
 * (include/LODkernel.cuh:302-309). */
gell_status gell_field_import(gell_ctx* ctx, int substrate, const float* field, int on_device);
gell_status gell_field_export(gell_ctx* ctx, int substrate, float* field, int on_device);

/* One mechanics step: Morton keys, stable sort, cell list, forces and Adams-Bashforth move.
 * Replaces MechanicsMesh_struct::FM_update (include/FMkernel.cuh:181-202). */
gell_status gell_fm_update(gell_ctx* ctx);

/* Uptake map of every cell into substrate `substrate` (-1 = all substrates).
 * Replaces Mesh_struct::PreLOD (include/LODkernel.cuh:270-278). */
gell_status gell_prelod(gell_ctx* ctx, int substrate);

/* `substeps` LOD substeps (boundary, implicit source, x, y and z Thomas sweeps) of substrate
 * `substrate` (-1 = all substrates).  Replaces Mesh_struct::LODsolver (include/LODkernel.cuh:280-300),
 * called `substeps` times. */
gell_status gell_lod_solver(gell_ctx* ctx, int substrate, int substeps);

/* Biology step, part 1: volume and Ki-67 phase update of every live cell and division of the
 * cells that complete mitosis.  Replaces CellBirth_kernel (include/PDkernel.cuh:88-98).
 * Daughters are appended in the order of their mothers (the reference appends them in atomic
 * order).  Writes the new count to *n_out when n_out is not NULL (synchronises). */
gell_status gell_cell_birth(gell_ctx* ctx, int* n_out);

/* Biology step, part 2: stable removal of every cell whose sign is false.  Replaces
 * CellDeath_kernel (include/PDkernel.cuh:100-117).  Writes the new count when n_out != NULL. */
gell_status gell_cell_death(gell_ctx* ctx, int* n_out);

/* One mechanics step and its diffusion: gell_fm_update, gell_prelod(-1) and `substeps`
 * gell_lod_solver(-1) calls, as the reference host loop runs them (Main.cu:114-124). */
gell_status gell_mechanics_step(gell_ctx* ctx, int substeps);

/* `steps` mechanics steps, each gell_fm_update, gell_prelod(-1) and `substeps` gell_lod_solver(-1)
 * calls: the reference host loop between two biology steps (Main.cu:114-124), with an integer step
 * count.  Pairs of steps are replayed from a CUDA graph captured on the context's stream (two steps
 * bring every double buffer back to where it was); the graph is captured again when the cell count,
 * the substrates, `substeps` or the buffer assignment have changed, and not used while per-kernel
 * profiling is on.  Queued on the context's stream, no host synchronisation. */
gell_status gell_run_mechanics(gell_ctx* ctx, int steps, int substeps);

/* Wait for all work queued on the context's stream and for the queued transfers. */
gell_status gell_sync(gell_ctx* ctx);

/* Debug and parity support.  Copies the named internal array to host memory `out` (room for
 * `bytes` bytes).  GELL_DUMP_KEYS: int32[n] Morton keys of the last fm_update in sorted order
 * (-1 for cells outside the grid, as include/FMkernel.cuh:26-33).  GELL_DUMP_PERM: int32[n]
 * source index of each sorted position.  GELL_DUMP_SE: int32[2*N^3], the reference's
 * Mech_Mesh_s then Mech_Mesh_e arrays (include/FMkernel.cuh:38-53) rebuilt from the cell list.
 * GELL_DUMP_RATE: float[N^3] uptake map of substrate `arg`.  GELL_DUMP_EF: float[2*N]
 * Thomas factors E then F of substrate `arg` (include/LODkernel.cuh:239-259). */
enum {
    GELL_DUMP_KEYS = 1,
    GELL_DUMP_PERM = 2,
    GELL_DUMP_SE = 3,
    GELL_DUMP_RATE = 4,
    GELL_DUMP_EF = 5
};
gell_status gell_debug_dump(gell_ctx* ctx, int what, int arg, void* out, size_t bytes);

/* Per-kernel timing.  When enabled, every kernel this library launches is bracketed by CUDA events
 * on the context's stream; gell_profile_read synchronises and reports, per kernel name, the number
 * of launches and their summed device time since the last reset (replaces the host clock() timing
 * of the reference host loop, Main.cu:101-133).  Off by default. */
typedef struct gell_profile_record {
    char name[40];
    int32_t launches;
    float total_ms;
} gell_profile_record;
gell_status gell_profile_enable(gell_ctx* ctx, int on);
gell_status gell_profile_read(gell_ctx* ctx, gell_profile_record* out, int max_records, int* count,
                              int reset);
/* Self-test of the division the LOD back substitution uses (a Markstein division with a
 * precomputed reciprocal) against IEEE division, on `samples` random operands in the sweeps'
 * range; *mismatches = number of quotients that differ in any bit.  Synchronises. */
gell_status gell_selftest_division(gell_ctx* ctx, int64_t samples, uint64_t seed, int64_t* mismatches);

/* Self-test of the bounded device waits: a kernel waits on a barrier that nothing completes, gives
 * up after `polls` polls and records it, so this returns GELL_ERR_TIMEOUT (reported once; the
 * context stays usable).  This is the path a sweep takes when a TMA box never lands.  No
 * counterpart in the reference, which has no device-side waits. */
gell_status gell_selftest_timeout(gell_ctx* ctx, int polls);

/* Largest key count gell_sort_keys_noalloc accepts. */
#define GELL_NOALLOC_MAX_KEYS (1 << 20)

/* Stable sort of n int32 Morton keys (-1 = outside the grid, ordered first) into sorted_keys,
 * with perm[i] = input position of sorted position i: the sort FM_update performs, for callers
 * that cannot allocate device memory.  No counterpart in the reference (its thrust::sort_by_key
 * allocates temporary storage on every call, include/FMkernel.cuh:190).  Some callers cannot call
 * cudaMalloc when they need the sort: code that runs while a CUDA stream is being captured, hosts
 * that must keep to a memory budget reserved up front, C callers that only own their buffers.  So
 * this call allocates nothing: keys, sorted_keys and perm are the caller's device buffers, and the
 * scratch lives in one fixed device array inside the library (about 8.3 MB on every GPU that
 * loads it, kept until the process exits).  key_bits must be at least the bit length of
 * (largest key + 1), e.g. 27 on a 400^3 grid; a smaller value gives an unspecified order, with
 * status OK.  keys, sorted_keys and perm must not share any memory (GELL_ERR_INVALID_ARG
 * otherwise).  n above GELL_NOALLOC_MAX_KEYS returns GELL_ERR_CAPACITY.  A CUDA error already
 * pending on the calling thread when the call starts is returned as GELL_ERR_CUDA and left
 * pending.  The first call on a device (and under each further driver context of it) looks up the
 * scratch address and should come before any stream capture; after a cudaDeviceReset the entry
 * point must not be called again.  All calls share the scratch, so calls that overlap on the GPU
 * race.  Work is queued on `stream` (a cudaStream_t; NULL = the default stream) and not
 * synchronised. */
gell_status gell_sort_keys_noalloc(const int32_t* keys, int32_t* sorted_keys, int32_t* perm, int n,
                                   int key_bits, void* stream);

/* Options (none has a reference counterpart).  GELL_OPT_EXACT_CHAIN = 1 makes the LOD back
 * substitution run the exact division chain for every group instead of the speculative chain that
 * is checked against it; results are identical either way, this only makes the exact path testable. */
enum {
    GELL_OPT_EXACT_CHAIN = 1,
    GELL_OPT_SWEEP_WARPS = 3,
    GELL_OPT_CONV_RING = 4,
    GELL_OPT_SWEEP_RING = 5,
    GELL_OPT_SWEEP_L2HINT = 6,
    GELL_OPT_SWEEP_RING_LAG = 7,
    GELL_OPT_SURROGATE_INPUT = 9,
    GELL_OPT_LOD_STREAMS = 10
};
/* GELL_OPT_SWEEP_RING (-1..8, default -1): 1 runs the LOD sweeps as ring kernels (a few group
 * slots of shared memory per warp; back substitution re-reads each group from L2 and recomputes its
 * forward values from a per-group checkpoint), which fit twice as many warps per SM as whole line
 * tiles; 2..8 do the same with at most that many slots per warp; 0 keeps whole line tiles in shared
 * memory; -1 picks the ring when fewer than four line tiles fit per SM (long lines, N > 416).
 * GELL_OPT_SWEEP_L2HINT (0 or 1, default 0): the ring sweeps load groups they will read again with
 * priority to stay in L2.  GELL_OPT_SWEEP_RING_LAG (0..7, default 0 = 1): how many of its own
 * result stores a ring warp lets run before it refills a stored slot (capped at the slots less
 * one).  Results are identical for every value of these options.
 * GELL_OPT_SURROGATE_INPUT (0 or 1, default 0), for surrogates loaded (or trained) after it is set:
 * 0 gives the operator the field p / b and scales its output d by b (q = p + b d); 1 gives it the
 * change of one plain substep, (L(p) - p) / m with m its largest magnitude inside the shell, and
 * scales the output by m (q = p + m d).  A LOD substep is affine in the field, so the change over
 * the surrogate's substeps is a linear function of that one-substep change; in this form bf16
 * inputs quantise the change rather than the field.  Weights are trained for one form.
 * GELL_OPT_LOD_STREAMS (0 or 1, default 1): the LOD substeps of each substrate run on a stream of
 * their own (forked from and joined back to the context's stream), so that one substrate's sweep
 * fills the SMs another's leaves idle at its start and end.  Results are identical. */
/* GELL_OPT_CONV_RING (0 or 1, default 1): the surrogate's convolutions keep the input rows of
 * consecutive lines in a ring of shared-memory slots (each row read from L2 once per unit of 32
 * lines) instead of loading all nine rows per tile; the results are the same. */
/* GELL_OPT_SWEEP_WARPS (0..4, default 0): line tiles (compute warps) per CTA of the LOD sweeps;
 * 0 = as many as shared memory holds.  Fewer give more, smaller CTAs, which can fill the GPU
 * better for small grids run side by side (the ensemble tuner tries them).  Results do not change. */
gell_status gell_set_option(gell_ctx* ctx, int option, int64_t value);

/*
 * Snapshots in the reference's CSV formats, printed with its own format strings so that equal data
 * gives identical files.  gell_write_cells_csv: `n` records from host memory as savecsv_cell
 * (include/FileSave.cuh:24-33): Index,Sign,Phase,x,y,z,r,V,Vns,Vcs.  gell_save_cells_csv: the
 * context's current cells, the same way.  gell_save_field_csv: substrate `substrate` as savecsv_mesh
 * (include/FileSave.cuh:35-49), one i,j,k,Concentration row per voxel, x fastest.
 * gell_save_field_slice_csv: the plane z = N/2 as savecsv_meshslice writes the slice GPU_Get_Slice
 * takes (include/FileSave.cuh:50-64, include/LODkernel.cuh:174-181).  These synchronise.
 */
gell_status gell_write_cells_csv(const gell_cell* cells, int n, const char* path);
gell_status gell_save_cells_csv(gell_ctx* ctx, const char* path);
gell_status gell_save_field_csv(gell_ctx* ctx, int substrate, const char* path);
gell_status gell_save_field_slice_csv(gell_ctx* ctx, int substrate, const char* path);

/*
 * Checkpoint and resume (no counterpart in the reference, which writes CSV snapshots only).
 * gell_checkpoint_save writes the state between two calls: parameters, substrates, cells, fields,
 * the cell-list epoch, the biology step counter and, with XORWOW draws, every slot's generator
 * state.  gell_checkpoint_load restores it into a context created with the same parameters and
 * substrates (GELL_ERR_STATE otherwise); the run then continues exactly as it would have without
 * the interruption.  Both synchronise.
 */
gell_status gell_checkpoint_save(gell_ctx* ctx, const char* path);
gell_status gell_checkpoint_load(gell_ctx* ctx, const char* path);

/*
 * The reference's initial tumour (Cell_sphere_Initialization, include/Initialization.cuh:15-43):
 * n quiescent cells of radius `cell_radius` (Tumor_Cell_Radius, 8.4 um) drawn uniformly in a ball
 * of radius cell_radius * n^(1/3) / 1.612 * 1.87 at the centre of the grid, with the reference's
 * default volumes.  Positions come from the C library's rand() sequence for `seed` (the reference
 * never seeds it, which is seed 1), computed by a private copy of that generator.  Host only.
 */
gell_status gell_reference_spheroid(const gell_params* p, int n, float cell_radius, uint32_t seed, gell_cell* out);

/*
 * Ensembles: independent simulations stepped together (no counterpart in the reference, which runs
 * one tumour per process).  Members are ordinary contexts on the same device, each with its own
 * grid, cells and substrates.  gell_ensemble_run_mechanics runs `steps` mechanics steps of every
 * member: pairs of steps replay ONE captured CUDA graph in which the members run on `branches`
 * parallel streams, so the small kernels of many small grids share the GPU.  The graph is captured
 * again when a member's cell count, substrates or buffer assignment, the substep count or the
 * configuration changed.  Each member's own stream is ordered before and after the ensemble's work;
 * biology steps and transfers stay per member (gell_cell_birth / gell_cell_death, ...).
 * gell_ensemble_configure sets the branch count (1..64) and the sweeps' line tiles per CTA
 * (GELL_OPT_SWEEP_WARPS, 0..4) of every member.  gell_ensemble_tune times branch counts 1, 2, 4, ..
 * and tile widths 0, 2, 1, then the batched LOD, with real steps of the members (2 per trial, plus
 * one first step; the total is returned in *steps_taken) and keeps the fastest.  The members must
 * outlive the ensemble and live on the device that is current when it is created.
 * gell_ensemble_set_batched (0 or 1, default 0): every captured step runs the FM_update and PreLOD
 * of ALL members as one launch per kernel (keys, each radix-sort pass, gather, force and move,
 * uptake map; up to 64 members with up to 4 substrates each, larger ensembles run these on the
 * branches), then their LOD substeps as one launch per sweep axis (and one for the uptake source)
 * over a device-side list of every member's line tiles; grid edges up to 256.  Results are
 * identical either way.  gell_ensemble_get_batched reports the setting (after a tune, whether the
 * tuner chose it).
 */
typedef struct gell_ensemble gell_ensemble;
gell_status gell_ensemble_create(gell_ctx* const* members, int count, gell_ensemble** out);
gell_status gell_ensemble_destroy(gell_ensemble* ens);
gell_status gell_ensemble_configure(gell_ensemble* ens, int branches, int sweep_warps);
gell_status gell_ensemble_run_mechanics(gell_ensemble* ens, int steps, int substeps);
gell_status gell_ensemble_tune(gell_ensemble* ens, int substeps, int* steps_taken, int* best_branches,
                               int* best_sweep_warps);
gell_status gell_ensemble_sync(gell_ensemble* ens);
gell_status gell_ensemble_set_batched(gell_ensemble* ens, int on);
gell_status gell_ensemble_get_batched(const gell_ensemble* ens, int* on);

/* Learned surrogate of one substrate's LOD (no reference counterpart; the reference's plain solver,
 * LODsolver in include/LODkernel.cuh:280-300, is its fallback and the source of its training pairs).
 * A 3-D convolutional operator maps [p / b, uptake rate * rate_scale, boundary-shell mask] to the
 * field after `substeps` LOD substeps: conv 3->32 + ReLU, four residual blocks
 * h += conv(ReLU(conv(h))), conv 32->1 giving d; output p + b * d inside the four boundary layers
 * and b on them (b = the substrate's boundary value).  3x3x3 kernels, zero padding, bf16 weights and
 * activations, fp32 sums, hand-written tcgen05 kernels.
 *
 * gell_surrogate_load: `weights` holds gell_surrogate_weight_count() floats, layer by layer
 * (conv_in, conv_a/conv_b of blocks 1-4, conv_out), each the PyTorch conv3d weight
 * [cout][cin][3][3][3] followed by its bias [cout].  Allocates the operator's buffers (40 bytes per
 * voxel of bf16 activations, two fields) on the first load; a later load replaces the weights.
 * gell_lod_surrogate: one judged step of `substeps` LOD substeps of the substrate (the uptake map
 * must be current, as for gell_lod_solver).  The operator's field q is judged by one plain substep
 * L: r = max |L(q) - q| / b over the voxels inside the boundary layers.  r <= threshold keeps q
 * (*accepted = 1); otherwise the field is restored and the plain solver runs the substeps
 * (*accepted = 0).  Synchronises the stream once (the decision is taken on the host).
 * gell_surrogate_infer: the operator alone, field := q (no judge).
 * gell_surrogate_run_layers / gell_surrogate_read: the input packing and the first `layers` (0..10)
 * convolutions, and a copy of a buffer to the host (which: 0 = input planes, 2 x 16 bytes per voxel;
 * 1 = h, 2 = t, 4 x 16 bytes per voxel; 3 = the output field, pitched) — for tests.  Activations are
 * stored as planes of 8 channels: plane q holds channels 8q..8q+7 of voxel x + N*(y + N*z) as 8
 * bf16 values at byte 16*(voxel + q*N^3). */
/* Training with the library's own kernels (no reference counterpart).
 * gell_surrogate_train_init: loads `weights` as gell_surrogate_load does and keeps fp32 master
 * copies, Adam moments and every buffer of the backward pass (46 more planes of 16 bytes per voxel:
 * the stored activations and the gradient planes).
 * gell_surrogate_train_pair: one pair of the running model.  The plain solver advances the field by
 * `substeps` (the target); the operator runs from the field before them; the loss is the mean of
 * ((q - target) / b)^2 inside the boundary layers.  Its gradient goes back through the ten layers:
 * data gradients on the tensor cores; weight gradients on the tensor cores for the 32 -> 32
 * layers, on the CUDA cores for the first and last. Adam (0.9, 0.999, 1e-8) takes a step of rate
 * `lr` on the gradient clipped to global norm 1.  The field is left at the target.  *loss (if not
 * NULL) gets the loss before the step (synchronises).
 * gell_surrogate_train_read: which 0 = the master weights, 1 = the last gradient (count =
 * gell_surrogate_weight_count()), 2 = the last target field (count = pitched field floats). */
gell_status gell_surrogate_train_init(gell_ctx* ctx, int substrate, const float* weights, long long count, int substeps,
                                      float rate_scale);
gell_status gell_surrogate_train_pair(gell_ctx* ctx, int substrate, float lr, float* loss);
gell_status gell_surrogate_train_read(gell_ctx* ctx, int substrate, int which, float* host, long long count);
long long gell_surrogate_weight_count(void);
gell_status gell_surrogate_load(gell_ctx* ctx, int substrate, const float* weights, long long count, int substeps,
                                float rate_scale, float threshold);
gell_status gell_lod_surrogate(gell_ctx* ctx, int substrate, int* accepted, float* residual);
gell_status gell_surrogate_infer(gell_ctx* ctx, int substrate);
gell_status gell_surrogate_run_layers(gell_ctx* ctx, int substrate, int layers);
gell_status gell_surrogate_read(gell_ctx* ctx, int substrate, int which, void* host, long long bytes);

/* Number of kernels this context has launched (always counted). */
gell_status gell_launch_count(gell_ctx* ctx, int64_t* count);

const char* gell_status_string(gell_status s);
const char* gell_last_error(gell_ctx* ctx);
int gell_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GELL_B200_GELL_H */
