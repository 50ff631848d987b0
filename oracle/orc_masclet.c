/*
 * orc_masclet.c -- oracle: MASCLET input (FLAG_DATA = 0) at levels <= 0, test
 * infrastructure.
 *
 * Restates the MASCLET branch of the level loop, src/avism.f90:980-1156:
 *  - the dark-matter particles go to the grid as in the particle path (SPH or
 *    TSC), when FLAG_DIV <= 1 or FLAG_DENS <= 1 (984); U1DMCO is then the mass
 *    over DXX*DYY*DZZ*RETE**3, over ROTE (1065-1066);
 *  - the gas grids: U1GCO = U1G, U2GCO.. = U2G.. at level 0 (1081-1087), and
 *    SMOOTH_2 below it (1071-1075);
 *  - DIVER_UNIFORM of the DM velocities and / or the gas velocities by FLAG_DIV
 *    (1129-1145);
 * then the choices of 1366-1405 and 1633-1650: U1CO = U1DMCO + U1GCO, U1DMCO or
 * U1GCO (FLAG_DENS 0, 1, 2), times ROTE, over its REAL*8 mean in K, J, I order;
 * DIVERCO = MIN(DIVERGCO, DIVERDMCO), DIVERDMCO or DIVERGCO (FLAG_DIV 0, 1, 2),
 * or -OMEGA0**0.6*RETE*HTE*(U1CO - 1) (FLAG_DIV = -1).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

#define UM_F 9.1717E18f
#define UL_F 10.98f

int orc_masclet_fields(const avism_params *p, int32_t nhy, const float *u1g, const float *u2g, const float *u3g,
                       const float *u4g, int64_t n, const float *x, const float *y, const float *z,
                       const float *vx, const float *vy, const float *vz, const float *m, float *u1co_ext,
                       float *diverco_ext, float *meandens)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    if (p->level > 0) return AVISM_ERR_UNSUPPORTED;              /* AMR patches: VMESH, DIVER_FINA_GAS */
    if (((int64_t)p->nx << (-p->level)) != (int64_t)nhy) return AVISM_ERR_ARG;
    if (p->flag_dens < 0 || p->flag_dens > 2 || p->flag_div < -1 || p->flag_div > 2) return AVISM_ERR_ARG;
    const int need_dm = p->flag_dens <= 1 || p->flag_div == 0 || p->flag_div == 1;
    const int need_gas_v = p->flag_div == 0 || p->flag_div == 2;
    const int nx = g.nx, ne = g.ne, low1 = g.low1;
    const int64_t nc = (int64_t)nx * nx * nx;
    float *um = (float *)calloc((size_t)nc, sizeof(float));
    float *d2 = (float *)calloc((size_t)nc, sizeof(float));
    float *d3 = (float *)calloc((size_t)nc, sizeof(float));
    float *d4 = (float *)calloc((size_t)nc, sizeof(float));
    float *co[4];
    for (int q = 0; q < 4; q++) co[q] = (float *)calloc((size_t)nc, sizeof(float));
    float *u1 = (float *)malloc((size_t)nc * sizeof(float));
    float *dg = (float *)calloc((size_t)nc, sizeof(float));
    float *dd = (float *)calloc((size_t)nc, sizeof(float));
    float *dv = (float *)calloc((size_t)nc, sizeof(float));
    if (need_dm) st = orc_particles_to_grid(p, n, x, y, z, vx, vy, vz, m, NULL, um, d2, d3, d4, NULL, NULL);
    if (!st) {
        const float *in[4] = {u1g, u2g, u3g, u4g};
        orc_level_grids(p, nhy, need_gas_v ? 4 : 1, in, co);
        const float dx = g.dx;
        const float vol = ((dx * dx) * dx) * ((g.rete * g.rete) * g.rete);
        for (int64_t c = 0; c < nc; c++) {
            float dm = 0.0f;
            if (p->flag_dens <= 1) {
                dm = um[c] / vol;
                dm = dm / g.rote;
            }
            const float u = p->flag_dens == 0 ? dm + co[0][c] : (p->flag_dens == 1 ? dm : co[0][c]);
            u1[c] = u * g.rote;
        }
        double mean8 = 0.0;
        for (int64_t c = 0; c < nc; c++) mean8 = mean8 + (double)u1[c];
        const float mean = (float)(mean8 / (double)nc);
        for (int64_t c = 0; c < nc; c++) u1[c] = u1[c] / mean;
        const float ul3 = (UL_F * UL_F) * UL_F;
        *meandens = mean * (UM_F / ul3);
        if (p->flag_div == -1) {
            const float coef = (powf(p->omega0, 0.6f) * g.rete) * g.hte;
            for (int64_t c = 0; c < nc; c++) dv[c] = -(coef * (u1[c] - 1.0f));
        } else {
            if (need_gas_v) orc_diver_uniform(nx, dx, co[1], co[2], co[3], p->periodic, dg);
            if (p->flag_div <= 1) orc_diver_uniform(nx, dx, d2, d3, d4, p->periodic, dd);
            for (int64_t c = 0; c < nc; c++)
                dv[c] = p->flag_div == 2 ? dg[c] : (p->flag_div == 1 ? dd[c] : (dd[c] < dg[c] ? dd[c] : dg[c]));
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
                    diverco_ext[e] = dv[c];
                }
    }
    free(um); free(d2); free(d3); free(d4);
    for (int q = 0; q < 4; q++) free(co[q]);
    free(u1); free(dg); free(dd); free(dv);
    return st;
}
