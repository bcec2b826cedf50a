/*
 * gell_oracle.c — TEST INFRASTRUCTURE ONLY (see gell_oracle.h).  CPU restatement of the
 * reference's hot path, used as the checker of the CUDA kernels and as the CPU baseline.
 * Build with -ffp-contract=off: each fused multiply-add the reference's nvcc build performs is
 * written as fmaf() below, every other float operation rounds once.
 */
#include "gell_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;
void go_set_threads(int t) { g_threads = t; }
int go_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}
#define OMP_THREADS num_threads(go_get_threads())

/* include/Definitions.h:7-47 and include/Cells.cuh literals */
void go_params_reference(go_params* p) {
    p->N = 100;
    p->len = 25.f;
    p->cap = 2 * 1000 * 1000;
    p->mech_dt = 0.1f;
    p->diff_dt = 0.01f;
    p->bio_dt = 6.f;
    p->ccca = 0.4f;
    p->cccr = 10.f;
    p->ra_ratio = 1.25;
    p->cc_max_dist = 25.f;
    p->dead_factor = 0.1f;
    p->default_v = 2494.f;
    p->o2_pt = 5.f;
    p->o2_ps = 10.f;
    p->o2_nt = 5.f;
    p->o2_nm = 2.5f;
    p->necrosis_rate = 1.0 / 6.0 / 60.0;        /* (1.f / 6.0 / 60.0) */
    p->apoptosis_rate = 1.0 / 7.0 / 24.0 / 60.0; /* (1.f / 7.0 / 24.0 / 60.0) */
    p->prolif_rate = 1.0 / 8.5 / 60.0;          /* (1.f/8.5/60.0) */
    p->dur_pre2post = 13.f * 60;
    p->dur_post2q = 2.5f * 60;
}

/* ------------------------------------------------------------------ indexing */

/* include/BasicFunctions.cuh:111-137: bit b of i goes to bit 3b, of j to 3b+1, of k to 3b+2,
 * for the 10 low bits of each coordinate.  Written as a loop over bits. */
int go_morton(int i, int j, int k) {
    unsigned out = 0;
    for (int b = 0; b < 10; ++b) {
        out |= ((unsigned)(i >> b) & 1u) << (3 * b);
        out |= ((unsigned)(j >> b) & 1u) << (3 * b + 1);
        out |= ((unsigned)(k >> b) & 1u) << (3 * b + 2);
    }
    return (int)out;
}

/* include/BasicFunctions.cuh:60-66: truncating conversion of pos/len */
void go_find_mesh(const float pos[3], float len, int ijk[3]) {
    ijk[0] = (int)(pos[0] / len);
    ijk[1] = (int)(pos[1] / len);
    ijk[2] = (int)(pos[2] / len);
}

int go_inside(int i, int j, int k, int N) {
    return !(i < 0 || i >= N || j < 0 || j >= N || k < 0 || k >= N);
}

static inline long vidx(int i, int j, int k, int N) { return i + (long)j * N + (long)k * N * N; }

/* ------------------------------------------------------------------ LOD */

/* include/LODkernel.cuh:239-259, host float arithmetic (no contraction on the host). */
void go_mesh_init(int N, float len, float D, float decay, float dt, float* E, float* F) {
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

void go_mesh_init_f64(int N, double len, double D, double decay, double dt, double* E, double* F) {
    double side = -dt * D / (len * len);
    double corner = 1.0 + dt * decay / 3.0 - side;
    double diag = corner - side;
    E[0] = 0.0;
    F[0] = corner;
    for (int i = 1; i < N - 1; ++i) {
        E[i] = side / F[i - 1];
        F[i] = diag - E[i] * side;
    }
    E[N - 1] = side / F[N - 2];
    F[N - 1] = corner - E[N - 1] * side;
}

/* One Dirichlet Thomas line (include/LODkernel.cuh:34-50, identical for y and z at :73-110):
 *   p[N-1] := b;  Y0 = b;  Y_i = fma(-E_i, Y_{i-1}, p_i)             i = 1..N-1
 *   x_i = fma(-s, x_{i+1}, Y_i) / F_i (from x_{N-1} = b)               i = N-2..1
 *   p[0] := b,  s = E[1]*F[0]  (the kernel's thomas_side). */
void go_thomas_line(float* p, long stride, const float* E, const float* F, int N, float b) {
    float Y[4096];
    float s = E[1] * F[0];
    p[(long)(N - 1) * stride] = b;
    Y[0] = b;
    for (int i = 1; i < N; ++i) Y[i] = fmaf(-E[i], Y[i - 1], p[(long)i * stride]);
    for (int i = N - 2; i > 0; --i)
        p[(long)i * stride] = fmaf(-s, p[(long)(i + 1) * stride], Y[i]) / F[i];
    p[0] = b;
}

/* Bundle of lines that run along `axis` over a plane, vectorised over the contiguous x index
 * where possible.  Same per-line arithmetic as go_thomas_line. */
static void sweep_x(float* p, const float* E, const float* F, int N, float b) {
    long NN = (long)N * N;
#pragma omp parallel for OMP_THREADS schedule(static)
    for (long l = 0; l < NN; ++l) go_thomas_line(p + l * N, 1, E, F, N, b);
}

/* lines along `stride` (N for y, N*N for z); outer index `o` chooses the plane */
static void sweep_strided(float* p, const float* E, const float* F, int N, float b, int axis) {
    long NN = (long)N * N;
    float s = E[1] * F[0];
#pragma omp parallel OMP_THREADS
    {
        float* Y = (float*)malloc(sizeof(float) * (size_t)N * N);
#pragma omp for schedule(static)
        for (int o = 0; o < N; ++o) {
            /* axis 1 (y): plane z = o, element j at x + j*N + o*NN
               axis 2 (z): plane y = o, element k at x + o*N + k*NN */
            long base = axis == 1 ? o * NN : (long)o * N;
            long st = axis == 1 ? N : NN;
            for (int x = 0; x < N; ++x) { p[base + x + (long)(N - 1) * st] = b; Y[x] = b; }
            for (int i = 1; i < N; ++i) {
                float* Yi = Y + (long)i * N;
                const float* Yp = Y + (long)(i - 1) * N;
                const float* pi = p + base + (long)i * st;
                float e = E[i];
                for (int x = 0; x < N; ++x) Yi[x] = fmaf(-e, Yp[x], pi[x]);
            }
            for (int i = N - 2; i > 0; --i) {
                float* pi = p + base + (long)i * st;
                const float* pn = p + base + (long)(i + 1) * st;
                const float* Yi = Y + (long)i * N;
                float f = F[i];
                for (int x = 0; x < N; ++x) pi[x] = fmaf(-s, pn[x], Yi[x]) / f;
            }
            for (int x = 0; x < N; ++x) p[base + x] = b;
        }
        free(Y);
    }
}

/* include/LODkernel.cuh:112-136 (Setboundary): layers 0,1,N-2,N-1 of every axis := b */
static void set_boundary(float* p, int N, float b) {
    int L[4] = {0, 1, N - 2, N - 1};
#pragma omp parallel for OMP_THREADS schedule(static)
    for (int a = 0; a < N; ++a)
        for (int c = 0; c < N; ++c)
            for (int l = 0; l < 4; ++l) {
                p[vidx(L[l], a, c, N)] = b;
                p[vidx(a, L[l], c, N)] = b;
                p[vidx(a, c, L[l], N)] = b;
            }
}

/* include/LODkernel.cuh:280-300: Setboundary, meshupdatekernel (:24-31) p /= 1 - rate*dt with
 * the product fused (fma(-rate, dt, 1)), then the x, y and z sweeps. */
void go_lod_substep(float* p, const float* rate, const float* E, const float* F, int N,
                    float dt, float b) {
    long NNN = (long)N * N * N;
    set_boundary(p, N, b);
#pragma omp parallel for OMP_THREADS schedule(static)
    for (long v = 0; v < NNN; ++v) p[v] = p[v] / fmaf(-rate[v], dt, 1.f);
    sweep_x(p, E, F, N, b);
    sweep_strided(p, E, F, N, b, 1);
    sweep_strided(p, E, F, N, b, 2);
}

/* FP64 restatement of the same substep (for accuracy reports, not parity). */
static void thomas_line_f64(double* p, long st, const double* E, const double* F, int N, double b,
                            double* Y) {
    double s = E[1] * F[0];
    p[(long)(N - 1) * st] = b;
    Y[0] = b;
    for (int i = 1; i < N; ++i) Y[i] = p[(long)i * st] - E[i] * Y[i - 1];
    for (int i = N - 2; i > 0; --i) p[(long)i * st] = (Y[i] - s * p[(long)(i + 1) * st]) / F[i];
    p[0] = b;
}

void go_lod_substep_f64(double* p, const double* rate, const double* E, const double* F, int N,
                        double dt, double b) {
    long NN = (long)N * N, NNN = NN * N;
    int L[4] = {0, 1, N - 2, N - 1};
    for (int a = 0; a < N; ++a)
        for (int c = 0; c < N; ++c)
            for (int l = 0; l < 4; ++l) {
                p[vidx(L[l], a, c, N)] = b;
                p[vidx(a, L[l], c, N)] = b;
                p[vidx(a, c, L[l], N)] = b;
            }
#pragma omp parallel for OMP_THREADS schedule(static)
    for (long v = 0; v < NNN; ++v) p[v] = p[v] / (1.0 - rate[v] * dt);
#pragma omp parallel OMP_THREADS
    {
        double* Y = (double*)malloc(sizeof(double) * (size_t)N);
#pragma omp for schedule(static)
        for (long l = 0; l < NN; ++l) thomas_line_f64(p + l * N, 1, E, F, N, b, Y);
#pragma omp for schedule(static)
        for (long l = 0; l < NN; ++l) {
            long x = l % N, z = l / N;
            thomas_line_f64(p + x + z * NN, N, E, F, N, b, Y);
        }
#pragma omp for schedule(static)
        for (long l = 0; l < NN; ++l) thomas_line_f64(p + l, NN, E, F, N, b, Y);
        free(Y);
    }
}

/* include/Cells.cuh:74-89 with O2 = 1: coef * (V/len/len/len) * 1, times the dead factor
 * for phase >= 3, zero for phase < 0. */
float go_uptake(const go_cell* c, float coef, float len, float dead_factor) {
    float vf = c->V / len / len / len;
    float rate = 0.f;
    if (c->phase >= 0 && c->phase <= 2) rate = coef * vf * 1.f;
    else if (c->phase >= 3) rate = coef * vf * 1.f * dead_factor;
    return rate;
}

/* include/LODkernel.cuh:12-22 and :270-278: zero the map, add each live cell's uptake at its
 * mesh_idx.  The reference adds with float atomics (order varies run to run); this sums in
 * cell order. */
void go_prelod(const go_cell* cells, int n, int N, float len, float coef, float dead_factor,
               float* rate) {
    long NNN = (long)N * N * N;
    memset(rate, 0, sizeof(float) * (size_t)NNN);
    for (int i = 0; i < n; ++i) {
        if (!cells[i].sign) continue;
        int m = cells[i].mesh_idx;
        if (m < 0 || m >= NNN) continue;
        rate[m] += go_uptake(&cells[i], coef, len, dead_factor);
    }
}

/* ------------------------------------------------------------------ FM */

/* include/FMkernel.cuh:22-36 */
void go_update_keys(go_cell* cells, int n, const go_params* P, int* keys) {
#pragma omp parallel for OMP_THREADS schedule(static)
    for (int i = 0; i < n; ++i) {
        int ijk[3];
        go_find_mesh(cells[i].pos, P->len, ijk);
        if (!go_inside(ijk[0], ijk[1], ijk[2], P->N)) {
            cells[i].sign = 0;
            keys[i] = -1;
            continue;
        }
        keys[i] = go_morton(ijk[0], ijk[1], ijk[2]);
        cells[i].mesh_idx = (int)vidx(ijk[0], ijk[1], ijk[2], P->N);
    }
}

/* Stable sort by signed key (thrust::sort_by_key at include/FMkernel.cuh:190 is a stable radix
 * sort; -1 orders first).  LSD radix over key+1 with two 16-bit digits. */
void go_stable_sort(go_cell* cells, int* keys, int n, int* perm) {
    unsigned* k0 = (unsigned*)malloc(sizeof(unsigned) * (size_t)(n > 0 ? n : 1));
    unsigned* k1 = (unsigned*)malloc(sizeof(unsigned) * (size_t)(n > 0 ? n : 1));
    int* p0 = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* p1 = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    size_t* cnt = (size_t*)malloc(sizeof(size_t) * 65537);
    for (int i = 0; i < n; ++i) { k0[i] = (unsigned)(keys[i] + 1); p0[i] = i; }
    for (int pass = 0; pass < 2; ++pass) {
        int sh = 16 * pass;
        memset(cnt, 0, sizeof(size_t) * 65537);
        for (int i = 0; i < n; ++i) cnt[((k0[i] >> sh) & 0xffff) + 1]++;
        for (int d = 0; d < 65536; ++d) cnt[d + 1] += cnt[d];
        for (int i = 0; i < n; ++i) {
            size_t o = cnt[(k0[i] >> sh) & 0xffff]++;
            k1[o] = k0[i];
            p1[o] = p0[i];
        }
        unsigned* tk = k0; k0 = k1; k1 = tk;
        int* tp = p0; p0 = p1; p1 = tp;
    }
    go_cell* tmp = (go_cell*)malloc(sizeof(go_cell) * (size_t)(n > 0 ? n : 1));
    memcpy(tmp, cells, sizeof(go_cell) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        cells[i] = tmp[p0[i]];
        keys[i] = (int)k0[i] - 1;
        if (perm) perm[i] = p0[i];
    }
    free(tmp); free(k0); free(k1); free(p0); free(p1); free(cnt);
}

/* include/FMkernel.cuh:38-53 */
void go_cell_list(const go_cell* cells, int n, const go_params* P, int* s, int* e) {
    long NNN = (long)P->N * P->N * P->N;
    for (long v = 0; v < NNN; ++v) { s[v] = P->cap + 1; e[v] = -1; }
    for (int i = 0; i < n; ++i) {
        if (!cells[i].sign) continue;
        int m = cells[i].mesh_idx;
        if (m < 0 || m >= NNN) continue;
        if (i > e[m]) e[m] = i;
        if (i < s[m]) s[m] = i;
    }
}

/* include/FMkernel.cuh:56-118 for one cell.  Per candidate j, in the reference's order
 * (xi, then yi, then zi bins, then ascending sorted index), with the stale cutoff `thres`:
 *   d   = sqrt(float(double(fma(dz,dz, fma(dx,dx, dy*dy))) + 0.0001))
 *   skip if d >= thres;  R = max(r2 + r1, 0.01);  thres = float(double(R) * ra_ratio)
 *   skip if d >= thres;  coefr = cccr*((1-d/R)^2/d) if d <= R;  coefa = ccca*((1-d/thres)^2/d)
 *   f += (p1 - p2) * (coefr - coefa)   as fma per component. */
void go_force_one(const go_cell* cells, int i, const go_params* P, const int* s, const int* e,
                  float out[3]) {
    const int N = P->N;
    float x1 = cells[i].pos[0], y1 = cells[i].pos[1], z1 = cells[i].pos[2];
    float r1 = cells[i].r;
    int b[3];
    go_find_mesh(cells[i].pos, P->len, b);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    float thres = P->cc_max_dist;
    for (int xi = b[0] - 1; xi <= b[0] + 1; ++xi)
        for (int yi = b[1] - 1; yi <= b[1] + 1; ++yi)
            for (int zi = b[2] - 1; zi <= b[2] + 1; ++zi) {
                if (!go_inside(xi, yi, zi, N)) continue;
                long m = vidx(xi, yi, zi, N);
                int cs = s[m], ce = e[m];
                if (ce < 0) continue;
                for (int j = cs; j <= ce; ++j) {
                    if (!cells[j].sign) continue;
                    float dx = x1 - cells[j].pos[0];
                    float dy = y1 - cells[j].pos[1];
                    float dz = z1 - cells[j].pos[2];
                    float ss = fmaf(dz, dz, fmaf(dx, dx, dy * dy));
                    float d = sqrtf((float)((double)ss + 0.0001));
                    if (d >= thres) continue;
                    float r2 = cells[j].r;
                    float rs = r2 + r1;
                    float R = rs > 0.01f ? rs : 0.01f;
                    thres = (float)((double)R * P->ra_ratio);
                    if (d >= thres) continue;
                    float coefr = 0.f, coefa = 0.f;
                    if (d <= R) {
                        float t = 1.f - d / R;
                        coefr = P->cccr * ((t * t) / d);
                    }
                    if (d <= thres) {
                        float t = 1.f - d / thres;
                        coefa = P->ccca * ((t * t) / d);
                    }
                    float c = coefr - coefa;
                    fx = fmaf(dx, c, fx);
                    fy = fmaf(dy, c, fy);
                    fz = fmaf(dz, c, fz);
                }
            }
    out[0] = fx; out[1] = fy; out[2] = fz;
}

void go_force(go_cell* cells, int n, const go_params* P, const int* s, const int* e) {
#pragma omp parallel for OMP_THREADS schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        if (!cells[i].sign) continue;
        float f[3];
        go_force_one(cells, i, P, s, e, f);
        cells[i].force[0] = f[0]; cells[i].force[1] = f[1]; cells[i].force[2] = f[2];
    }
}

/* include/FMkernel.cuh:130-158: pos += dt/2 * (3f - f_old) as fma(dt/2, fma(3, f, -f_old), pos);
 * a cell whose new bin is outside the grid only loses its sign. */
void go_move(go_cell* cells, int n, const go_params* P) {
    const float h = P->mech_dt / 2.f;
#pragma omp parallel for OMP_THREADS schedule(static)
    for (int i = 0; i < n; ++i) {
        go_cell* c = &cells[i];
        if (!c->sign) continue;
        float np[3];
        for (int a = 0; a < 3; ++a) np[a] = fmaf(h, fmaf(3.f, c->force[a], -c->oldforce[a]), c->pos[a]);
        int ijk[3];
        go_find_mesh(np, P->len, ijk);
        if (!go_inside(ijk[0], ijk[1], ijk[2], P->N)) { c->sign = 0; continue; }
        for (int a = 0; a < 3; ++a) {
            c->pos[a] = np[a];
            c->oldforce[a] = c->force[a];
            c->force[a] = 0.f;
        }
        c->mesh_idx = (int)vidx(ijk[0], ijk[1], ijk[2], P->N);
    }
}

/* FP64 restatement of forcekernel and movementkernel (include/FMkernel.cuh:56-118,130-158), for the
 * accuracy report rather than parity: the same bins, candidate order and stale cutoff as
 * go_force_one, every operation in double.  `cells` are sorted with `s`/`e` their cell list; writes
 * the force and the moved position (pos + dt/2 (3 f - oldforce)) of every live cell, zeros for
 * the others. */
void go_force_move_f64(const go_cell* cells, int n, const go_params* P, const int* s, const int* e, double* force,
                       double* pos) {
    const int N = P->N;
    const double h = (double)P->mech_dt / 2.0;
#pragma omp parallel for OMP_THREADS schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        double* f = force + 3L * i;
        double* q = pos + 3L * i;
        f[0] = f[1] = f[2] = q[0] = q[1] = q[2] = 0.0;
        if (!cells[i].sign) continue;
        const double x1 = cells[i].pos[0], y1 = cells[i].pos[1], z1 = cells[i].pos[2], r1 = cells[i].r;
        int b[3];
        go_find_mesh(cells[i].pos, P->len, b);
        double fx = 0.0, fy = 0.0, fz = 0.0, thres = P->cc_max_dist;
        for (int xi = b[0] - 1; xi <= b[0] + 1; ++xi)
            for (int yi = b[1] - 1; yi <= b[1] + 1; ++yi)
                for (int zi = b[2] - 1; zi <= b[2] + 1; ++zi) {
                    if (!go_inside(xi, yi, zi, N)) continue;
                    long m = vidx(xi, yi, zi, N);
                    if (e[m] < 0) continue;
                    for (int j = s[m]; j <= e[m]; ++j) {
                        if (!cells[j].sign) continue;
                        const double dx = x1 - cells[j].pos[0], dy = y1 - cells[j].pos[1], dz = z1 - cells[j].pos[2];
                        const double d = sqrt(dx * dx + dy * dy + dz * dz + 0.0001);
                        if (d >= thres) continue;
                        const double rs = cells[j].r + r1, R = rs > 0.01 ? rs : 0.01;
                        thres = R * P->ra_ratio;
                        if (d >= thres) continue;
                        double coefr = 0.0, coefa = 0.0;
                        if (d <= R) coefr = P->cccr * ((1.0 - d / R) * (1.0 - d / R) / d);
                        if (d <= thres) coefa = P->ccca * ((1.0 - d / thres) * (1.0 - d / thres) / d);
                        fx += dx * (coefr - coefa);
                        fy += dy * (coefr - coefa);
                        fz += dz * (coefr - coefa);
                    }
                }
        f[0] = fx; f[1] = fy; f[2] = fz;
        for (int a = 0; a < 3; ++a) q[a] = cells[i].pos[a] + h * (3.0 * f[a] - cells[i].oldforce[a]);
    }
}

void go_fm_update(go_cell* cells, int n, const go_params* P, int* keys, int* perm, int* s, int* e) {
    long NNN = (long)P->N * P->N * P->N;
    int* k = keys ? keys : (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* ss = s ? s : (int*)malloc(sizeof(int) * (size_t)NNN);
    int* ee = e ? e : (int*)malloc(sizeof(int) * (size_t)NNN);
    go_update_keys(cells, n, P, k);
    go_stable_sort(cells, k, n, perm);
    go_cell_list(cells, n, P, ss, ee);
    go_force(cells, n, P, ss, ee);
    go_move(cells, n, P);
    if (!keys) free(k);
    if (!s) free(ss);
    if (!e) free(ee);
}

/* ------------------------------------------------------------------ cell model */

/* include/Cells.cuh:91-143.  Each compartment relaxes as Vx' = Vx*(1 - dt*rx) + (rx*dt)*Vx_0.
 * The reference's host build (g++) rounds every operation; its device build (nvcc) fuses the
 * outer multiply-add.  mode GO_VOL_HOST: every operation rounded.  GO_VOL_DEVICE:
 * fma(Vx, 1 - dt*rx, (rx*dt)*Vx_0) with 1 - dt*rx and rx*dt rounded once each.
 * GO_VOL_DEVICE_FUSED: the inner 1 - dt*rx fused as well.  GO_VOL_DEVICE_SWAP(_FUSED): the other
 * product fused, fma(rx*dt, Vx_0, Vx*(1 - dt*rx)).  GO_VOL_DEVICE_REF: what the reference's device
 * build does, found by running it on every phase: the fluid compartment (target V*ff, per cell)
 * as GO_VOL_DEVICE, the nuclear and cytoplasmic ones (per-phase constant targets) as
 * GO_VOL_DEVICE_SWAP.  r from the double-precision pow. */
static int g_vol_mode = GO_VOL_DEVICE_REF;
void go_set_volume_mode(int mode) { g_vol_mode = mode; }
static inline float relax(float v, float rx, float v0, float dt, int mode) {
    if (mode == GO_VOL_HOST) return v * (1.f - dt * rx) + rx * dt * v0;
    const int fused = mode == GO_VOL_DEVICE_FUSED || mode == GO_VOL_DEVICE_SWAP_FUSED;
    const float k = fused ? fmaf(-dt, rx, 1.f) : 1.f - dt * rx;
    if (mode == GO_VOL_DEVICE_SWAP || mode == GO_VOL_DEVICE_SWAP_FUSED) return fmaf(rx * dt, v0, v * k);
    return fmaf(v, k, rx * dt * v0);
}
void go_volume_update_mode(go_cell* c, int mode) {
    const float dt = 6.f; /* Biology_dt */
    float ff = (float)0.7502;
    float rf = 3.f / 60.f;
    float rcs = 0.33f / 60.f;
    float rns = 0.33f / 60.f;
    float Vns_0 = 135.f;
    int ph = c->phase;
    if (ph == 0 || ph == 2) {
    } else if (ph == 1) {
        Vns_0 = Vns_0 * 2;
        rcs = (float)(0.27 / 60);
    } else if (ph == 3) {
        ff = 0;
        Vns_0 = 0;
        rns = (float)(0.35 / 60);
        rcs = 1.f / 60;
    } else if (ph == 4) {
        ff = 1;
        rf = (float)(0.67 / 60);
        Vns_0 = 0;
        rns = (float)(0.013 / 60);
        rcs = (float)(0.0032 / 60);
    } else if (ph == 5) {
        ff = 0;
        rf = (float)(0.05 / 60);
        Vns_0 = 0;
        rns = (float)(0.013 / 60);
        rcs = (float)(0.0032 / 60);
    }
    float Vf_0 = c->V * ff;
    float Vcs_0 = Vns_0 * 3.615f;
    const int mf = mode == GO_VOL_DEVICE_REF ? GO_VOL_DEVICE : mode;
    const int mc = mode == GO_VOL_DEVICE_REF ? GO_VOL_DEVICE_SWAP : mode;
    c->Vf = relax(c->Vf, rf, Vf_0, dt, mf);
    c->Vns = relax(c->Vns, rns, Vns_0, dt, mc);
    c->Vcs = relax(c->Vcs, rcs, Vcs_0, dt, mc);
    c->V = c->Vf + c->Vns + c->Vcs;
    c->r = (float)pow(0.23873241 * (double)c->V, 1.0 / 3);
}
void go_volume_update(go_cell* c) { go_volume_update_mode(c, g_vol_mode); }
void go_volume_update_modes(go_cell* c, int n, int mode) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) go_volume_update_mode(c + i, mode);
}

/* include/Cells.cuh:69-71 */
void go_radius_update(go_cell* c) { c->r = (float)pow(0.23873241 * (double)c->V, 1.0 / 3); }

/* include/Cells.cuh:145-223 */
int go_phase_update(go_cell* c, float rnd, float o2, const go_params* P) {
    const float dt = P->bio_dt;
    c->cell_clock = c->cell_clock + dt;
    int proliferate = 0;
    float apoptosis_prob = (float)(P->apoptosis_rate * (double)dt);
    float proliferation_prob =
        (float)((double)((o2 - P->o2_pt) / (P->o2_ps - P->o2_pt)) * P->prolif_rate * (double)dt);
    if (o2 > P->o2_ps) proliferation_prob = (float)(P->prolif_rate * (double)dt);
    else if (o2 < P->o2_pt) proliferation_prob = 0;
    float necrosis_prob =
        (float)((double)((P->o2_nt - o2) / (P->o2_nt - P->o2_nm)) * P->necrosis_rate * (double)dt);
    if (o2 > P->o2_nt) necrosis_prob = 0;
    else if (o2 < P->o2_nm) necrosis_prob = (float)(P->necrosis_rate * (double)dt);

    if (c->phase >= 3) {
        if (c->phase == 4 && c->V >= P->default_v * 2) {
            c->phase = 5;
            c->cell_clock = 0;
        }
        if (c->Vcs <= 0.05f * 488) {
            c->sign = 0;
            c->cell_clock = 0;
        }
    } else {
        if (c->phase == 1 && c->cell_clock >= P->dur_pre2post) {
            c->phase = 2;
            proliferate = 1;
            c->cell_clock = 0;
        }
        if (c->phase == 2 && c->cell_clock >= P->dur_post2q) {
            c->phase = 0;
            c->cell_clock = 0;
        }
        if (c->phase == 0) {
            if (rnd <= proliferation_prob) {
                c->phase = 1;
                c->cell_clock = 0;
            } else if (rnd <= proliferation_prob + apoptosis_prob) {
                c->phase = 3;
                c->cell_clock = 0;
            } else if (rnd <= proliferation_prob + apoptosis_prob + necrosis_prob) {
                c->phase = 4;
                c->cell_clock = 0;
            }
        }
    }
    return proliferate;
}

/* include/RandomFunctions.cuh:23-31 */
void go_random_vect(float u, float v, float out[3]) {
    float theta = 2 * u * 3.1415926f;
    float phi = acosf(fmaf(2.f, v, -1.f));
    out[0] = sinf(theta) * sinf(phi);
    out[1] = cosf(theta) * sinf(phi);
    out[2] = cosf(phi);
}

/* ------------------------------------------------------------------ PD */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11): ten rounds of two 32x32->64 multiplies with the Weyl key schedule. */
void go_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* uniform on (0, 1]: the top 24 bits plus one, times 2^-24 (exact in float) */
float go_u01(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

static float field_at(const float* field, const float pos[3], const go_params* P) {
    int b[3];
    go_find_mesh(pos, P->len, b);
    for (int a = 0; a < 3; ++a) b[a] = b[a] < 0 ? 0 : (b[a] >= P->N ? P->N - 1 : b[a]);
    return field[vidx(b[0], b[1], b[2], P->N)];
}

/* include/PDkernel.cuh:27-86 for one slot, given its draws; returns 1 if a daughter was written */
static int birth_one(go_cell* cells, int i, int slot_new, int can_place, const go_params* P,
                     const float* field, float u, float u1, float v1) {
    go_cell* c = &cells[i];
    float o2 = field_at(field, c->pos, P);
    go_volume_update(c);
    int proli = go_phase_update(c, u, o2, P);
    if (!(proli && can_place)) return 0;
    float dir[3];
    go_random_vect(u1, v1, dir);
    float rm = c->r;
    float dist = 0.2063f * rm;
    rm *= 0.7937f;
    float pd[3], pm[3];
    for (int a = 0; a < 3; ++a) {
        pd[a] = fmaf(dir[a], dist, c->pos[a]);
        pm[a] = fmaf(-dir[a], dist, c->pos[a]);
    }
    c->r = rm;
    for (int a = 0; a < 3; ++a) c->pos[a] = pm[a];
    c->phase = 2;
    c->cell_clock = 0;
    c->V = c->V / 2;
    c->Vf = c->Vf / 2;
    c->Vcs = c->Vcs / 2;
    c->Vns = c->Vns / 2;
    go_cell d;
    memset(&d, 0, sizeof d);
    d.sign = 1;
    d.mesh_idx = -1;
    for (int a = 0; a < 3; ++a) { d.pos[a] = pd[a]; d.force[a] = 0.f; d.oldforce[a] = 0.f; }
    d.phase = 2;
    d.cell_clock = 0;
    d.r = rm;
    d.V = c->V;
    d.Vf = c->Vf;
    d.Vcs = c->Vcs;
    d.Vns = c->Vns;
    cells[slot_new] = d;
    return 1;
}

/* Birth in slot order: a daughter is placed while the count stays below cap - 1, the
 * sequential reading of the reference's checks (include/PDkernel.cuh:31,51,54). */
int go_birth_draws(go_cell* cells, int n, const go_params* P, const float* field,
                   const float* u, const float* u1, const float* v1) {
    if (n >= P->cap) return n;
    int count = n;
    for (int i = 0; i < n; ++i) {
        if (!cells[i].sign) continue;
        int can = count < P->cap - 1;
        count += birth_one(cells, i, count, can, P, field, u[i], u1[i], v1[i]);
    }
    return count;
}

int go_birth_philox(go_cell* cells, int n, const go_params* P, const float* field,
                    uint64_t seed, uint32_t bio_step) {
    if (n >= P->cap) return n;
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    int count = n;
    for (int i = 0; i < n; ++i) {
        if (!cells[i].sign) continue;
        uint32_t ctr[4] = {(uint32_t)i, bio_step, 0u, 0u}, r[4];
        go_philox4x32_10(ctr, key, r);
        int can = count < P->cap - 1;
        count += birth_one(cells, i, count, can, P, field, go_u01(r[0]), go_u01(r[1]), go_u01(r[2]));
    }
    return count;
}

/* include/PDkernel.cuh:100-117: thrust::remove_if(sign == false) is stable */
int go_death(go_cell* cells, int n) {
    int k = 0;
    for (int i = 0; i < n; ++i)
        if (cells[i].sign) cells[k++] = cells[i];
    return k;
}
