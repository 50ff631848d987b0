/*
 * orc_interp.c -- oracle: particles to grid (test infrastructure).
 *
 * Restates src/particles.f90: PPART_DENS (742-801), VVEL_INTERP_SPH_VW (806-929),
 * KERNEL_FUNC (935-963), H_DISTANCE (276-350), FILL_H_ZEROS (398-430),
 * DDENS_INTERP_SPH (434-617), DENS_INTERP_TSC (16-127), VEL_INTERP_TSC (132-271),
 * called in the order of src/avism.f90:1159-1245.  Grids are inner NX^3,
 * column-major, 0-based in C (Fortran index i -> i-1).
 *
 * Order rules where the reference depends on thread timing:
 *   - DDENS / DENS_TSC: FP64 accumulation in particle order, then rounded;
 *   - VEL_TSC: FP32 accumulation in particle order (the reference uses FP32
 *     atomics, src/particles.f90:241-248, so its own result varies per run).
 * The scatter loops run in parallel over z-slabs of cells (slab_of), each
 * thread walking every particle in index order, so these orders hold.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "avism_oracle.h"

#define RAD(i) radx[(i) - g->rad_lo]

/* branch counters of the last orc_particles_to_grid: cells on the ball_search
 * fallback, FILL_H_ZEROS orphans, DDENS particles with NORM = 0 */
static int64_t g_path_counts[3];

void orc_path_counts(int64_t *out)
{
    for (int i = 0; i < 3; i++) out[i] = g_path_counts[i];
}

static inline int64_t cell_id(int nx, int i, int j, int k)   /* 1-based i,j,k */
{
    return (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (int64_t)(k - 1));
}

/* KERNEL_FUNC (src/particles.f90:935-963): returns W(dist; h) for KERNEL_MODE
 * 1 (M4 cubic spline) or 2 (Gaussian EXP(-Q**2)) */
static inline float kernel_w(int gauss, float h, float dist)
{
    const float q = dist / (h / 2.0f);
    if (gauss) return expf(-(q * q));
    if (q <= 1.0f) return 1.0f - (1.5f * (q * q)) * (1.0f - 0.5f * q);
    if (q <= 2.0f) { const float t = 2.0f - q; return 0.25f * ((t * t) * t); }
    return 0.0f;
}

/* HPART(j) = MAX(HPART(j), d) under OMP ATOMIC: floats >= 0 ordered as ints */
static inline void atomic_max_pos(float *a, float v)
{
    int32_t *ai = (int32_t *)a;
    int32_t nv; memcpy(&nv, &v, 4);
    int32_t cur = __atomic_load_n(ai, __ATOMIC_RELAXED);
    while (nv > cur) {
        if (__atomic_compare_exchange_n(ai, &cur, nv, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
    }
}

int orc_ppart_dens(const orc_kdtree *t, int64_t n, const float *x, const float *y,
                   const float *z, const float *m, int k, float *part_dens)
{
    if (k <= 0 || k > 1024) return AVISM_ERR_ARG;
    const double pi = acos(-1.0);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        int64_t idx[1024]; float d2[1024];
        orc_kd_knn(t, x[i], y[i], z[i], k, idx, d2);
        const float hk = sqrtf(d2[k - 1]);
        double bas8 = 0.0;
        for (int j = 0; j < k; j++) bas8 = bas8 + (double)m[idx[j]];
        part_dens[i] = (float)(bas8 / ((4.0 / 3.0) * pi * (double)((hk * hk) * hk)));
    }
    return AVISM_OK;
}

/* cell kNN with the ball fallback of src/particles.f90:868-878.  Returns the
 * neighbour count; idx/d2 point into the caller's growable buffers. */
static int64_t cell_neigh(const orc_kdtree *t, float tx, float ty, float tz, int k, float dx,
                          int64_t **idx, float **d2, int64_t *cap)
{
    if (*cap < k) {
        *cap = k + 64;
        *idx = (int64_t *)realloc(*idx, (size_t)*cap * sizeof(int64_t));
        *d2 = (float *)realloc(*d2, (size_t)*cap * sizeof(float));
    }
    orc_kd_knn(t, tx, ty, tz, k, *idx, *d2);
    if (sqrtf((*d2)[k - 1]) > dx) return k;
    __atomic_fetch_add(&g_path_counts[0], 1, __ATOMIC_RELAXED);
    return orc_kd_ball(t, tx, ty, tz, dx, idx, d2, cap);
}

int orc_vvel_interp_sph_vw(const orc_kdtree *t, const avism_grid *g, const float *radx,
                           int k, int64_t n, const float *m, const float *vx,
                           const float *vy, const float *vz, const float *part_dens,
                           const int8_t *smask, int gauss, float *hpart, float *u2, float *u3,
                           float *u4)
{
    (void)n;
    const int nx = g->nx;
    const float dx = g->dx;
    #pragma omp parallel
    {
        int64_t *idx = NULL; float *d2 = NULL; int64_t cap = 0;
        float *w = NULL; int64_t wcap = 0;
        #pragma omp for collapse(2) schedule(dynamic, 4)
        for (int kz = 1; kz <= nx; kz++)
            for (int jy = 1; jy <= nx; jy++)
                for (int ix = 1; ix <= nx; ix++) {
                    const int64_t c = cell_id(nx, ix, jy, kz);
                    if (smask && smask[c] == 0) continue;
                    const int64_t cnt = cell_neigh(t, RAD(ix), RAD(jy), RAD(kz), k, dx, &idx, &d2, &cap);
                    if (cnt > wcap) { wcap = cnt + 64; w = (float *)realloc(w, (size_t)wcap * sizeof(float)); }
                    for (int64_t i = 0; i < cnt; i++) {
                        w[i] = sqrtf(d2[i]);
                        atomic_max_pos(&hpart[idx[i]], w[i]);
                    }
                    const float hk = cnt > 0 ? w[cnt - 1] : 0.0f;
                    for (int64_t i = 0; i < cnt; i++) w[i] = kernel_w(gauss, hk, w[i]);
                    for (int64_t i = 0; i < cnt; i++) w[i] = w[i] * (m[idx[i]] / part_dens[idx[i]]);
                    double b = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
                    for (int64_t i = 0; i < cnt; i++) {
                        const double w8 = (double)w[i];
                        b = b + w8;
                        bx = bx + w8 * (double)vx[idx[i]];
                        by = by + w8 * (double)vy[idx[i]];
                        bz = bz + w8 * (double)vz[idx[i]];
                    }
                    u2[c] = (float)(bx / b);
                    u3[c] = (float)(by / b);
                    u4[c] = (float)(bz / b);
                }
        free(idx); free(d2); free(w);
    }
    return AVISM_OK;
}

int orc_h_distance(const orc_kdtree *t, const avism_grid *g, const float *radx, int k,
                   int64_t n, const int8_t *smask, float *hpart)
{
    (void)n;
    const int nx = g->nx;
    #pragma omp parallel
    {
        int64_t *idx = NULL; float *d2 = NULL; int64_t cap = 0;
        #pragma omp for collapse(2) schedule(dynamic, 4)
        for (int kz = 1; kz <= nx; kz++)
            for (int jy = 1; jy <= nx; jy++)
                for (int ix = 1; ix <= nx; ix++) {
                    const int64_t c = cell_id(nx, ix, jy, kz);
                    if (smask && smask[c] == 0) continue;
                    const int64_t cnt = cell_neigh(t, RAD(ix), RAD(jy), RAD(kz), k, g->dx, &idx, &d2, &cap);
                    for (int64_t i = 0; i < cnt; i++) atomic_max_pos(&hpart[idx[i]], sqrtf(d2[i]));
                }
        free(idx); free(d2);
    }
    return AVISM_OK;
}

int orc_fill_h_zeros(const orc_kdtree *t, int64_t n, const float *x, const float *y,
                     const float *z, int k, float *hpart)
{
    if (k <= 0 || k > 1024) return AVISM_ERR_ARG;
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        if (hpart[i] > 0.0f) continue;
        __atomic_fetch_add(&g_path_counts[1], 1, __ATOMIC_RELAXED);
        int64_t idx[1024]; float d2[1024];
        orc_kd_knn(t, x[i], y[i], z[i], k, idx, d2);
        hpart[i] = sqrtf(d2[k - 1]);
    }
    return AVISM_OK;
}

/* Cells are split into z-slabs, one per thread; every thread walks all the
 * particles in index order and adds only the contributions that fall in its
 * slab, so each cell still receives its terms in particle order (the rule that
 * replaces the reference's OpenMP atomics).  A particle whose support spans two
 * slabs has its NORM computed by both threads, identically. */
static void slab_of(int nx, int *k0, int *k1)
{
    int nt = 1, t = 0;
#ifdef _OPENMP
    nt = omp_get_num_threads();
    t = omp_get_thread_num();
#endif
    *k0 = 1 + (int)(((int64_t)nx * t) / nt);
    *k1 = (int)(((int64_t)nx * (t + 1)) / nt);
}

int orc_ddens_interp_sph(const avism_grid *g, const float *radx, int64_t n,
                         const float *x, const float *y, const float *z,
                         const float *hpart, const float *m, int gauss, float *u)
{
    const int nx = g->nx;
    const float dx = g->dx;
    const float rx1 = RAD(1);
    const int64_t nc = (int64_t)nx * nx * nx;
    double *u8 = (double *)calloc((size_t)nc, sizeof(double));
    if (!u8) return AVISM_ERR_OOM;
    #pragma omp parallel
    {
        int ks0, ks1;
        slab_of(nx, &ks0, &ks1);
        for (int64_t p = 0; p < n && ks0 <= ks1; p++) {
            const int ix = (int)((x[p] - rx1) / dx) + 1;
            const int jy = (int)((y[p] - rx1) / dx) + 1;
            const int kz = (int)((z[p] - rx1) / dx) + 1;
            const float h = hpart[p];
            const int inc = (int)((2.0f * h) / dx + 0.5f);
            if (kz + inc < ks0 || kz - inc > ks1) continue;
            const float inv_h = 2.0f / h;
            const float inv_h_sq = inv_h * inv_h;
            const float h2max = (4.0f * h) * h;
            float norm = 0.0f;
            for (int pass = 0; pass < 2; pass++) {
                for (int k2 = kz - inc; k2 <= kz + inc; k2++) {
                    if (k2 < 1 || k2 > nx) continue;
                    if (pass == 1 && (k2 < ks0 || k2 > ks1)) continue;
                    const float tz = z[p] - RAD(k2);
                    const float dz2 = tz * tz;
                    for (int j2 = jy - inc; j2 <= jy + inc; j2++) {
                        if (j2 < 1 || j2 > nx) continue;
                        const float ty = y[p] - RAD(j2);
                        const float dy2 = ty * ty;
                        for (int i2 = ix - inc; i2 <= ix + inc; i2++) {
                            if (i2 < 1 || i2 > nx) continue;
                            const float tx = x[p] - RAD(i2);
                            const float dx2 = tx * tx;
                            const float d2 = (dx2 + dy2) + dz2;
                            if (d2 > h2max) continue;
                            float w;
                            if (gauss) {
                                w = expf(-(d2 * inv_h_sq));           /* KERNEL_MODE = 2 */
                            } else {
                                const float q = sqrtf(d2) * inv_h;
                                if (q <= 1.0f) w = 1.0f - (1.5f * (q * q)) * (1.0f - 0.5f * q);
                                else if (q <= 2.0f) { const float s = 2.0f - q; w = 0.25f * ((s * s) * s); }
                                else w = 0.0f;
                            }
                            if (pass == 0) norm = norm + w;
                            else u8[cell_id(nx, i2, j2, k2)] += (double)((w * m[p]) / norm);
                        }
                    }
                }
                if (pass == 0 && norm == 0.0f) {
                    if (kz >= ks0 && kz <= ks1) __atomic_fetch_add(&g_path_counts[2], 1, __ATOMIC_RELAXED);
                    if (ix >= 1 && ix <= nx && jy >= 1 && jy <= nx && kz >= ks0 && kz <= ks1 && kz <= nx)
                        u8[cell_id(nx, ix, jy, kz)] += (double)m[p];
                    break;
                }
            }
        }
    }
    for (int64_t c = 0; c < nc; c++) u[c] = (float)u8[c];
    free(u8);
    return AVISM_OK;
}

/* TSC weights and the nearest cell of one coordinate, src/particles.f90:56-96 */
static inline void tsc_axis(const avism_grid *g, const float *radx, int periodic, float xt,
                            int *cell, float w[3])
{
    const float dx = g->dx;
    const float r1 = RAD(1) - 0.5f * dx;
    const float rn = RAD(g->nx) + 0.5f * dx;
    const float leng = rn - r1;
    if (periodic) {
        if (xt < r1) xt = xt + leng;
        if (xt >= rn) xt = xt - leng;
    }
    const int i = (int)(((xt - RAD(1)) / dx) + 0.49999f) + 1;
    float bas = fabsf(RAD(i - 1) - xt);
    float t = 1.5f - bas / dx;
    w[0] = 0.5f * (t * t);
    bas = fabsf(RAD(i) - xt);
    t = bas / dx;
    w[1] = 0.75f - t * t;
    bas = fabsf(RAD(i + 1) - xt);
    t = 1.5f - bas / dx;
    w[2] = 0.5f * (t * t);
    *cell = i;
}

static inline int tsc_wrap(int i, int nx, int periodic)
{
    if (periodic) { if (i < 1) i += nx; if (i > nx) i -= nx; }
    return i;
}

int orc_dens_interp_tsc(const avism_grid *g, const float *radx, int periodic, int64_t n,
                        const float *x, const float *y, const float *z, const float *m,
                        float *u)
{
    const int nx = g->nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    double *u8 = (double *)calloc((size_t)nc, sizeof(double));
    if (!u8) return AVISM_ERR_OOM;
    #pragma omp parallel
    {
    int ks0, ks1;
    slab_of(nx, &ks0, &ks1);
    for (int64_t p = 0; p < n && ks0 <= ks1; p++) {
        int ci, cj, ck; float wx[3], wy[3], wz[3];
        tsc_axis(g, radx, periodic, x[p], &ci, wx);
        tsc_axis(g, radx, periodic, y[p], &cj, wy);
        tsc_axis(g, radx, periodic, z[p], &ck, wz);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                for (int c = 0; c < 3; c++) {
                    const int i3 = tsc_wrap(ci + c - 1, nx, periodic);
                    const int j3 = tsc_wrap(cj + b - 1, nx, periodic);
                    const int k3 = tsc_wrap(ck + a - 1, nx, periodic);
                    /* non-periodic cells outside 1..NX: the reference writes out of
                       bounds there; the oracle drops the contribution */
                    if (i3 < 1 || i3 > nx || j3 < 1 || j3 > nx || k3 < 1 || k3 > nx) continue;
                    if (k3 < ks0 || k3 > ks1) continue;
                    const float inc = ((m[p] * wx[c]) * wy[b]) * wz[a];
                    u8[cell_id(nx, i3, j3, k3)] += (double)inc;
                }
    }
    }
    for (int64_t c = 0; c < nc; c++) u[c] = (float)u8[c];
    free(u8);
    return AVISM_OK;
}

int orc_vel_interp_tsc(const avism_grid *g, const float *radx, int periodic, int64_t n,
                       const float *x, const float *y, const float *z, const float *vx,
                       const float *vy, const float *vz, float *u2, float *u3, float *u4)
{
    const int nx = g->nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    float *wt = (float *)calloc((size_t)nc, sizeof(float));
    if (!wt) return AVISM_ERR_OOM;
    for (int64_t c = 0; c < nc; c++) { u2[c] = 0.0f; u3[c] = 0.0f; u4[c] = 0.0f; }
    #pragma omp parallel
    {
    int ks0, ks1;
    slab_of(nx, &ks0, &ks1);
    for (int64_t p = 0; p < n && ks0 <= ks1; p++) {
        int ci, cj, ck; float wx[3], wy[3], wz[3];
        tsc_axis(g, radx, periodic, x[p], &ci, wx);
        tsc_axis(g, radx, periodic, y[p], &cj, wy);
        tsc_axis(g, radx, periodic, z[p], &ck, wz);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                for (int c = 0; c < 3; c++) {
                    const int i3 = tsc_wrap(ci + c - 1, nx, periodic);
                    const int j3 = tsc_wrap(cj + b - 1, nx, periodic);
                    const int k3 = tsc_wrap(ck + a - 1, nx, periodic);
                    if (i3 < 1 || i3 > nx || j3 < 1 || j3 > nx || k3 < 1 || k3 > nx) continue;
                    if (k3 < ks0 || k3 > ks1) continue;
                    const float w = (wx[c] * wy[b]) * wz[a];
                    const int64_t id = cell_id(nx, i3, j3, k3);
                    u2[id] = u2[id] + vx[p] * w;
                    u3[id] = u3[id] + vy[p] * w;
                    u4[id] = u4[id] + vz[p] * w;
                    wt[id] = wt[id] + w;
                }
    }
    }
    for (int64_t c = 0; c < nc; c++) {
        float wei = wt[c];
        if (wei == 0.0f) wei = 1.0f;
        u2[c] = u2[c] / wei; u3[c] = u3[c] / wei; u4[c] = u4[c] / wei;
    }
    free(wt);
    return AVISM_OK;
}

int orc_particles_to_grid(const avism_params *p, int64_t n, const float *x, const float *y,
                          const float *z, const float *vx, const float *vy, const float *vz,
                          const float *m, const int8_t *smask, float *u_mass, float *u2,
                          float *u3, float *u4, float *hpart, float *part_dens)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    float *radx = (float *)malloc((size_t)(g.rad_hi - g.rad_lo + 1) * sizeof(float));
    orc_grid_setup(p, &g, radx);
    const int k = p->kneighbours;
    const int64_t nc = (int64_t)g.nx * g.nx * g.nx;
    /* particles outside [-L0/2, L0/2] stop the run (src/avism.f90:560-589) */
    const float half = p->lado0 / 2.0f;
    for (int64_t i = 0; i < n; i++)
        if (x[i] < -half || x[i] > half || y[i] < -half || y[i] > half || z[i] < -half || z[i] > half) {
            free(radx);
            return AVISM_ERR_OUT_OF_BOX;
        }
    for (int i = 0; i < 3; i++) g_path_counts[i] = 0;
    float *h = hpart ? hpart : (float *)malloc((size_t)n * sizeof(float));
    float *pd = part_dens ? part_dens : (float *)malloc((size_t)n * sizeof(float));
    for (int64_t i = 0; i < n; i++) { h[i] = 0.0f; pd[i] = 0.0f; }
    for (int64_t c = 0; c < nc; c++) { u_mass[c] = 0.0f; u2[c] = 0.0f; u3[c] = 0.0f; u4[c] = 0.0f; }
    orc_kdtree *t = NULL;
    if ((p->flag_vel_interp == 1 && !p->no_velocities) || p->flag_dens_interp == 1)
        t = orc_kd_build(n, x, y, z, p->periodic ? p->lado0 : 0.0f);
    const int gauss = p->kernel_mode == 2;
    /* velocities, src/avism.f90:1159-1194; none without velocities (1259-1306) */
    const int vel_sph = p->flag_vel_interp == 1 && !p->no_velocities;
    if (!p->no_velocities && p->flag_vel_interp == 0) {
        orc_vel_interp_tsc(&g, radx, p->periodic, n, x, y, z, vx, vy, vz, u2, u3, u4);
    } else if (vel_sph) {
        orc_ppart_dens(t, n, x, y, z, m, k, pd);
        orc_vvel_interp_sph_vw(t, &g, radx, k, n, m, vx, vy, vz, pd, smask, gauss, h, u2, u3, u4);
        orc_fill_h_zeros(t, n, x, y, z, k, h);
    }
    /* density, src/avism.f90:1214-1245 (1270-1296 without velocities) */
    if (p->flag_dens_interp == 0) {
        orc_dens_interp_tsc(&g, radx, p->periodic, n, x, y, z, m, u_mass);
    } else {
        if (!vel_sph) {
            orc_h_distance(t, &g, radx, k, n, smask, h);
            orc_fill_h_zeros(t, n, x, y, z, k, h);
        }
        orc_ddens_interp_sph(&g, radx, n, x, y, z, h, m, gauss, u_mass);
    }
    orc_kd_free(t);
    if (!hpart) free(h);
    if (!part_dens) free(pd);
    free(radx);
    return AVISM_OK;
}
