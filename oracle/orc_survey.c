/*
 * orc_survey.c -- oracle: survey mode (FLAG_SURVEY = 1), test infrastructure.
 *
 * Restates src/avism.f90:1420-1596: the tracers go to the grid as particles
 * (with the survey mask SMASK), the randoms with the same interpolation -- TSC
 * (DENS_INTERP_TSC), or SPH with their own kNN: H_DISTANCE and FILL_H_ZEROS
 * with KNEIGHBOURS2 = MIN(8*KNEIGHBOURS, 256), then DDENS_INTERP_SPH -- and
 * the density contrast becomes D/(alpha R): ALPHA = DSUM/RSUM over the
 * observed cells, the ratio floored at 1e-4 and clamped at 1000, then divided
 * by its mean over SMASK > 0.  MEANDENS is the background density.  Without
 * velocities the divergence is the linear-theory one (src/avism.f90:1647-1650).
 *
 * Order rule: DSUM, RSUM (an OpenMP reduction in the reference) and the
 * MEANRATIO sum (a serial SUM) are REAL*8 sums taken per x-row, the rows of a
 * plane summed in j order, the planes in k order -- the order the GPU's
 * row / plane / total kernels use.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

#define UM_F 9.1717E18f
#define UL_F 10.98f

/* REAL*8 sum of a[c] over the cells where take(c), rows then planes then total */
static double blocked_sum(int nx, const float *a, const int8_t *smask, int positive_only)
{
    double tot = 0.0;
    for (int k = 0; k < nx; k++) {
        double plane = 0.0;
        for (int j = 0; j < nx; j++) {
            double row = 0.0;
            for (int i = 0; i < nx; i++) {
                const int64_t c = (int64_t)i + (int64_t)nx * ((int64_t)j + (int64_t)nx * k);
                const int8_t s = smask[c];
                if (positive_only ? s > 0 : s != 0) row = row + (double)a[c];
            }
            plane = plane + row;
        }
        tot = tot + plane;
    }
    return tot;
}

int orc_survey_contrast(const avism_params *p, const avism_grid *g, const int8_t *smask, const float *u1rand,
                        float *u1, float *meandens)
{
    const int nx = g->nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    /* WEIGHTS D,R sum (src/avism.f90:1527-1540) */
    const double dsum = blocked_sum(nx, u1, smask, 0);
    const double rsum = blocked_sum(nx, u1rand, smask, 0);
    const double alpha = dsum / rsum;
    /* DENSITY RATIO (1543-1566): floor and clamp in REAL*8, stored as REAL*4 */
    const float ratiofloor = 1e-4f, ratiomax = 1000.0f;
    for (int64_t c = 0; c < nc; c++) {
        if (smask[c] == 0) continue;
        double bass8;
        if ((double)u1rand[c] > 0.0) bass8 = (double)u1[c] / (alpha * (double)u1rand[c]);
        else bass8 = (double)ratiofloor;
        bass8 = fmax((double)ratiofloor, bass8);
        bass8 = fmin((double)ratiomax, bass8);
        u1[c] = (float)bass8;
    }
    /* MEANRATIO over SMASK > 0, then U1CO / MEANRATIO there (1569-1573) */
    int64_t count = 0;
    for (int64_t c = 0; c < nc; c++) count += smask[c] > 0;
    const float meanratio = (float)(blocked_sum(nx, u1, smask, 1) / (double)count);
    for (int64_t c = 0; c < nc; c++)
        if (smask[c] > 0) u1[c] = u1[c] / meanratio;
    /* MEANDENS = ROTE * (UM / UL**3) (1578) */
    const float ul3 = (UL_F * UL_F) * UL_F;
    *meandens = g->rote * (UM_F / ul3);
    (void)p;
    return AVISM_OK;
}

int orc_survey_fields(const avism_params *p, int64_t n, const float *x, const float *y, const float *z,
                      const float *vx, const float *vy, const float *vz, const float *m, int64_t nrand,
                      const float *rx, const float *ry, const float *rz, const float *rw, const int8_t *smask,
                      float *u1co_ext, float *diverco_ext, float *meandens, float *u1rand_out)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    if (!smask || nrand < 1) return AVISM_ERR_ARG;
    const int nx = g.nx, ne = g.ne, low1 = g.low1;
    const int64_t nc = (int64_t)nx * nx * nx;
    float *um = (float *)malloc((size_t)nc * sizeof(float)), *u2 = (float *)malloc((size_t)nc * sizeof(float));
    float *u3 = (float *)malloc((size_t)nc * sizeof(float)), *u4 = (float *)malloc((size_t)nc * sizeof(float));
    float *ur = (float *)malloc((size_t)nc * sizeof(float)), *d = (float *)malloc((size_t)nc * sizeof(float));
    float *s2 = (float *)malloc((size_t)nc * sizeof(float)), *s3 = (float *)malloc((size_t)nc * sizeof(float));
    float *s4 = (float *)malloc((size_t)nc * sizeof(float));
    float *zr = (float *)calloc((size_t)nrand, sizeof(float));
    if (!um || !u2 || !u3 || !u4 || !ur || !d || !s2 || !s3 || !s4 || !zr) {
        free(um); free(u2); free(u3); free(u4); free(ur); free(d); free(s2); free(s3); free(s4); free(zr);
        return AVISM_ERR_OOM;
    }
    /* tracers to the grid, with the mask */
    st = orc_particles_to_grid(p, n, x, y, z, vx, vy, vz, m, smask, um, u2, u3, u4, NULL, NULL);
    /* randoms: no velocities; SPH with KNEIGHBOURS2 = MIN(8*KNEIGHBOURS, 256) (1516) */
    avism_params pr = *p;
    pr.no_velocities = 1;
    pr.kneighbours = 8 * p->kneighbours < 256 ? 8 * p->kneighbours : 256;
    if (!st) st = orc_particles_to_grid(&pr, nrand, rx, ry, rz, zr, zr, zr, rw, smask, ur, s2, s3, s4, NULL, NULL);
    if (!st) {
        const float dx = g.dx;
        const float vol = ((dx * dx) * dx) * ((g.rete * g.rete) * g.rete);
        float *u1 = s2;
        for (int64_t c = 0; c < nc; c++) {           /* U1CO = U1DMCO * ROTE (1249-1250, 1386) */
            float v = um[c] / vol;
            v = v / g.rote;
            u1[c] = v * g.rote;
        }
        orc_survey_contrast(p, &g, smask, ur, u1, meandens);
        if (p->no_velocities) {
            const float coef = (powf(p->omega0, 0.6f) * g.rete) * g.hte;
            for (int64_t c = 0; c < nc; c++) d[c] = -(coef * (u1[c] - 1.0f));
        } else {
            orc_diver_uniform(nx, dx, u2, u3, u4, p->periodic, d);
        }
        for (int kz = 0; kz < ne; kz++)
            for (int jy = 0; jy < ne; jy++)
                for (int ix = 0; ix < ne; ix++) {
                    int i = ix + low1, j = jy + low1, k = kz + low1;
                    if (i < 1) i += nx; else if (i > nx) i -= nx;
                    if (j < 1) j += nx; else if (j > nx) j -= nx;
                    if (k < 1) k += nx; else if (k > nx) k -= nx;
                    const int64_t e = (int64_t)ix + (int64_t)ne * ((int64_t)jy + (int64_t)ne * kz);
                    const int64_t c = (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1));
                    u1co_ext[e] = u1[c];
                    diverco_ext[e] = d[c];
                }
        if (u1rand_out) memcpy(u1rand_out, ur, (size_t)nc * sizeof(float));
    }
    free(um); free(u2); free(u3); free(u4); free(ur); free(d); free(s2); free(s3); free(s4); free(zr);
    return st;
}

/* The level's copies of grids given at NHY^3 (level 0): copied at level 0;
 * below it SMOOTH_2 (src/amr2uniform.f90:65-120): a serial scatter of U*WEI
 * into the coarse cell of every input cell, K, J, I order.  co[q] hold zeros. */
void orc_level_grids(const avism_params *p, int32_t nhy, int ngrids, const float *const *in, float *const *co)
{
    avism_grid g, g0;
    orc_grid_setup(p, &g, NULL);
    const int nx = g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    if (nx == nhy) {
        for (int q = 0; q < ngrids; q++) memcpy(co[q], in[q], (size_t)nc * sizeof(float));
        return;
    }
    float *radx = (float *)malloc((size_t)(g.rad_hi - g.rad_lo + 1) * sizeof(float));
    orc_grid_setup(p, &g, radx);
    avism_params p0 = *p;
    p0.nx = nhy;
    orc_grid_setup(&p0, &g0, NULL);
    float *rad0 = (float *)malloc((size_t)(g0.rad_hi - g0.rad_lo + 1) * sizeof(float));
    orc_grid_setup(&p0, &g0, rad0);
    const float dx = g.dx, dx0 = g0.dx, r1 = radx[1 - g.rad_lo];
    const float wei = ((dx0 * dx0) * dx0) / ((dx * dx) * dx);
    for (int kk = 1; kk <= nhy; kk++)
        for (int jj = 1; jj <= nhy; jj++)
            for (int ii = 1; ii <= nhy; ii++) {
                const int i = (int)(((rad0[ii - g0.rad_lo] - r1) / dx) + 0.5f) + 1;
                const int j = (int)(((rad0[jj - g0.rad_lo] - r1) / dx) + 0.5f) + 1;
                const int k = (int)(((rad0[kk - g0.rad_lo] - r1) / dx) + 0.5f) + 1;
                const int64_t c = (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1));
                const int64_t f = (int64_t)(ii - 1) + (int64_t)nhy * ((int64_t)(jj - 1) + (int64_t)nhy * (kk - 1));
                for (int q = 0; q < ngrids; q++) co[q][c] = co[q][c] + in[q][f] * wei;
            }
    free(rad0);
    free(radx);
}

/* Grid input (FLAG_DATA = 2, src/avism.f90:1316-1362): U1CO = U1GCO, MEANDENS =
 * ROTE*(UM/UL**3), DIVERCO = DIVER_UNIFORM of the velocities.  Levels below 0
 * take SMOOTH_2 (src/amr2uniform.f90:65-120) of the NHY^3 input grids: a serial
 * scatter of U*WEI into the coarse cell of every input cell, K, J, I order. */
int orc_grid_fields(const avism_params *p, int32_t nhy, const float *u1g, const float *u2g, const float *u3g,
                    const float *u4g, float *u1co_ext, float *diverco_ext, float *meandens)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    if (p->level > 0) return AVISM_ERR_UNSUPPORTED;          /* 'LEVEL > 0 FOR BIN_GRID NOT IMPLEMENTED YET' */
    if (((int64_t)p->nx << (-p->level)) != (int64_t)nhy) return AVISM_ERR_ARG;
    const int nx = g.nx, ne = g.ne, low1 = g.low1;
    const int64_t nc = (int64_t)nx * nx * nx;
    float *co[4];
    for (int q = 0; q < 4; q++) co[q] = (float *)calloc((size_t)nc, sizeof(float));
    float *d = (float *)malloc((size_t)nc * sizeof(float));
    const float *in[4] = {u1g, u2g, u3g, u4g};
    orc_level_grids(p, nhy, 4, in, co);
    orc_diver_uniform(nx, g.dx, co[1], co[2], co[3], p->periodic, d);
    for (int kz = 0; kz < ne; kz++)
        for (int jy = 0; jy < ne; jy++)
            for (int ix = 0; ix < ne; ix++) {
                int i = ix + low1, j = jy + low1, k = kz + low1;
                if (i < 1) i += nx; else if (i > nx) i -= nx;
                if (j < 1) j += nx; else if (j > nx) j -= nx;
                if (k < 1) k += nx; else if (k > nx) k -= nx;
                const int64_t e = (int64_t)ix + (int64_t)ne * ((int64_t)jy + (int64_t)ne * kz);
                const int64_t c = (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1));
                u1co_ext[e] = co[0][c];
                diverco_ext[e] = d[c];
            }
    const float ul3 = (UL_F * UL_F) * UL_F;
    *meandens = g.rote * (UM_F / ul3);
    for (int q = 0; q < 4; q++) free(co[q]);
    free(d);
    return AVISM_OK;
}
