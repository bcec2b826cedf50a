/*
 * gell_oracle.h — TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's per-timestep hot
 * path (PhantomOtter/Gell: include/FMkernel.cuh, include/LODkernel.cuh, include/PDkernel.cuh,
 * include/Cells.cuh, include/BasicFunctions.cuh).  It is the checker of the gell_b200 CUDA path
 * and the timed CPU baseline; the product never links or calls it.
 *
 * Arithmetic contract (FP32 entry points).  The reference is compiled by nvcc, which contracts a
 * multiply feeding an add into one fused multiply-add.  This restatement writes each of those
 * contractions out as fmaf() and every other operation as one IEEE-754 single-precision operation
 * (compile with -ffp-contract=off), keeping the double-precision steps the reference has through
 * double literals and double-typed macros.  Each function states the sequence it uses.
 *
 * Parity pins: the host-callable reference functions (Morton code, bin lookup, cell model) are
 * compared with this file on CPU through fixtures under tests/golden/; the reference's kernels,
 * built from its unmodified sources for a B200, are compared with it on the GPU.
 */
#ifndef GELL_ORACLE_H
#define GELL_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's 72-byte struct Cell (include/Cells.cuh:9-47). */
typedef struct go_cell {
    uint8_t sign; uint8_t pad_[3];
    int32_t mesh_idx;
    float pos[3], force[3], oldforce[3];
    float r, V, Vf, Vcs, Vns;
    int32_t phase;
    float cell_clock;
} go_cell;

/* Parameters: the reference's #defines (include/Definitions.h:7-47), at run time. */
typedef struct go_params {
    int32_t N;                 /* Voxel_num */
    float len;                 /* Voxel_length */
    int32_t cap;               /* Max_Cell_num */
    float mech_dt, diff_dt, bio_dt;
    float ccca, cccr;
    double ra_ratio;
    float cc_max_dist;
    float dead_factor, default_v;
    float o2_pt, o2_ps, o2_nt, o2_nm;
    double necrosis_rate, apoptosis_rate, prolif_rate;
    float dur_pre2post, dur_post2q;
} go_params;

void go_params_reference(go_params* p);

/* ---- indexing (include/BasicFunctions.cuh) ---- */
int go_morton(int i, int j, int k);                                  /* :111-137 */
void go_find_mesh(const float pos[3], float len, int ijk[3]);       /* :60-66 */
int go_inside(int i, int j, int k, int N);                          /* :18-29 */

/* ---- LOD (include/LODkernel.cuh) ---- */
void go_mesh_init(int N, float len, float D, float decay, float dt, float* E, float* F); /* :239-259 */
void go_lod_substep(float* p, const float* rate, const float* E, const float* F, int N,
                    float dt, float boundary);                      /* :280-300 */
void go_lod_substep_f64(double* p, const double* rate, const double* E, const double* F, int N,
                        double dt, double boundary);
void go_mesh_init_f64(int N, double len, double D, double decay, double dt, double* E, double* F);
/* single sweep of one line (input p[0..N-1] with stride `stride`), in place */
void go_thomas_line(float* p, long stride, const float* E, const float* F, int N, float boundary);
float go_uptake(const go_cell* c, float coef, float len, float dead_factor); /* Cells.cuh:74-89 */
void go_prelod(const go_cell* cells, int n, int N, float len, float coef, float dead_factor,
               float* rate);                                        /* LODkernel.cuh:12-22,270-278 */

/* ---- FM (include/FMkernel.cuh) ---- */
/* keys (updateCellMeshIdx :22-36); returns nothing, writes keys[n] */
void go_update_keys(go_cell* cells, int n, const go_params* P, int* keys);
/* stable sort of (key, cell) by signed key; perm[i] = old index of sorted position i */
void go_stable_sort(go_cell* cells, int* keys, int n, int* perm);
/* Mech_Mesh_se_Reset + Mech_Mesh_se_Get (:38-53) into dense s,e of N^3 */
void go_cell_list(const go_cell* cells, int n, const go_params* P, int* s, int* e);
/* forcekernel (:56-118), writes cell.force of live cells */
void go_force(go_cell* cells, int n, const go_params* P, const int* s, const int* e);
/* force of one cell (same sequence), without writing */
void go_force_one(const go_cell* cells, int i, const go_params* P, const int* s, const int* e,
                  float out[3]);
/* movementkernel (:130-158) */
void go_move(go_cell* cells, int n, const go_params* P);
/* FP64 force and moved position of each live sorted cell (accuracy report, not parity) */
void go_force_move_f64(const go_cell* cells, int n, const go_params* P, const int* s, const int* e, double* force,
                       double* pos);
/* FM_update (:181-202): keys, sort, s/e, force, move.  keys/perm/s/e may be NULL. */
void go_fm_update(go_cell* cells, int n, const go_params* P, int* keys, int* perm, int* s, int* e);

/* ---- cell model (include/Cells.cuh) ---- */
enum { GO_VOL_HOST = 0, GO_VOL_DEVICE = 1, GO_VOL_DEVICE_FUSED = 2, GO_VOL_DEVICE_SWAP = 3, GO_VOL_DEVICE_SWAP_FUSED = 4,
       GO_VOL_DEVICE_REF = 5 };
void go_volume_update(go_cell* c);                                  /* :91-143 */
void go_volume_update_mode(go_cell* c, int mode);
void go_set_volume_mode(int mode);
void go_volume_update_modes(go_cell* c, int n, int mode);           /* n cells, one mode */
void go_radius_update(go_cell* c);                                  /* :69-71 */
int go_phase_update(go_cell* c, float rnd, float o2, const go_params* P); /* :145-223 */
void go_random_vect(float u, float v, float out[3]);                /* RandomFunctions.cuh:23-31 */

/* ---- PD (include/PDkernel.cuh) with Philox draws ---- */
void go_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float go_u01(uint32_t x);
/* Birthkernel + CellBirth_kernel (:27-98) with per-slot Philox draws; daughters appended in
 * the order of their mothers.  field = substrate driving the cell model (dense N^3).
 * Returns the new count. */
int go_birth_philox(go_cell* cells, int n, const go_params* P, const float* field,
                    uint64_t seed, uint32_t bio_step);
/* Birth with explicit draws: u[i] for slot i, and (u1[i], v1[i]) for its division direction */
int go_birth_draws(go_cell* cells, int n, const go_params* P, const float* field,
                   const float* u, const float* u1, const float* v1);
/* CellDeath_kernel (:100-117): stable compaction of sign != 0; returns the new count */
int go_death(go_cell* cells, int n);

/* threads used by the OpenMP loops (0 = runtime default) */
void go_set_threads(int t);
int go_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
