/*
 * orc_fields.c -- oracle: density normalisation, divergence, ghost fill
 * (test infrastructure).
 *
 * Restates src/avism.f90:1249-1250 and 1384-1411 (rho/rho_B, then rho/<rho>
 * with an FP64 mean), src/divergence.f90:2-50 (DIVER_UNIFORM) and
 * src/num.f90:89-133 (REAL_MAKE_PERIODIC: every ghost cell takes the value of
 * the inner cell at the wrapped coordinates).  The FP64 mean is summed in
 * K,J,I order (the reference uses an OpenMP reduction of unspecified order).
 * Without velocities the divergence is the linear-theory one of
 * src/avism.f90:1647-1650.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

#define UM_F 9.1717E18f
#define UL_F 10.98f

static inline int64_t in_id(int nx, int i, int j, int k)   /* 1-based */
{
    return (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (int64_t)(k - 1));
}

int orc_diver_uniform(int nx, float dx, const float *v2, const float *v3, const float *v4,
                      int periodic, float *diver)
{
    if (nx < 3) return AVISM_ERR_ARG;
    for (int k = 1; k <= nx; k++)
        for (int j = 1; j <= nx; j++)
            for (int i = 1; i <= nx; i++) {
                float ddx, ddy, ddz;
                /* d/dx of V2 along i, src/divergence.f90:23-45 */
                if (i > 1 && i < nx) ddx = (v2[in_id(nx, i + 1, j, k)] - v2[in_id(nx, i - 1, j, k)]) / 2.0f;
                else if (periodic) {
                    const int ip = i == nx ? 1 : i + 1, im = i == 1 ? nx : i - 1;
                    ddx = (v2[in_id(nx, ip, j, k)] - v2[in_id(nx, im, j, k)]) / 2.0f;
                } else if (i == 1) {
                    const float inner = (v2[in_id(nx, 3, j, k)] - v2[in_id(nx, 1, j, k)]) / 2.0f;
                    ddx = 2.0f * (v2[in_id(nx, 2, j, k)] - v2[in_id(nx, 1, j, k)]) - inner;
                } else {
                    const float inner = (v2[in_id(nx, nx, j, k)] - v2[in_id(nx, nx - 2, j, k)]) / 2.0f;
                    ddx = 2.0f * (v2[in_id(nx, nx, j, k)] - v2[in_id(nx, nx - 1, j, k)]) - inner;
                }
                if (j > 1 && j < nx) ddy = (v3[in_id(nx, i, j + 1, k)] - v3[in_id(nx, i, j - 1, k)]) / 2.0f;
                else if (periodic) {
                    const int jp = j == nx ? 1 : j + 1, jm = j == 1 ? nx : j - 1;
                    ddy = (v3[in_id(nx, i, jp, k)] - v3[in_id(nx, i, jm, k)]) / 2.0f;
                } else if (j == 1) {
                    const float inner = (v3[in_id(nx, i, 3, k)] - v3[in_id(nx, i, 1, k)]) / 2.0f;
                    ddy = 2.0f * (v3[in_id(nx, i, 2, k)] - v3[in_id(nx, i, 1, k)]) - inner;
                } else {
                    const float inner = (v3[in_id(nx, i, nx, k)] - v3[in_id(nx, i, nx - 2, k)]) / 2.0f;
                    ddy = 2.0f * (v3[in_id(nx, i, nx, k)] - v3[in_id(nx, i, nx - 1, k)]) - inner;
                }
                if (k > 1 && k < nx) ddz = (v4[in_id(nx, i, j, k + 1)] - v4[in_id(nx, i, j, k - 1)]) / 2.0f;
                else if (periodic) {
                    const int kp = k == nx ? 1 : k + 1, km = k == 1 ? nx : k - 1;
                    ddz = (v4[in_id(nx, i, j, kp)] - v4[in_id(nx, i, j, km)]) / 2.0f;
                } else if (k == 1) {
                    const float inner = (v4[in_id(nx, i, j, 3)] - v4[in_id(nx, i, j, 1)]) / 2.0f;
                    ddz = 2.0f * (v4[in_id(nx, i, j, 2)] - v4[in_id(nx, i, j, 1)]) - inner;
                } else {
                    const float inner = (v4[in_id(nx, i, j, nx)] - v4[in_id(nx, i, j, nx - 2)]) / 2.0f;
                    ddz = 2.0f * (v4[in_id(nx, i, j, nx)] - v4[in_id(nx, i, j, nx - 1)]) - inner;
                }
                diver[in_id(nx, i, j, k)] = (ddx / dx + ddy / dx) + ddz / dx;
            }
    return AVISM_OK;
}

int orc_fields(const avism_params *p, const float *u_mass, const float *u2, const float *u3,
               const float *u4, float *u1co_ext, float *diverco_ext, float *meandens)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    const int nx = g.nx, ne = g.ne, low1 = g.low1;
    const int64_t nc = (int64_t)nx * nx * nx;
    const float dx = g.dx;
    const float vol = ((dx * dx) * dx) * ((g.rete * g.rete) * g.rete);
    float *u1 = (float *)malloc((size_t)nc * sizeof(float));
    float *dv = (float *)malloc((size_t)nc * sizeof(float));
    if (!u1 || !dv) { free(u1); free(dv); return AVISM_ERR_OOM; }
    /* U1DMCO -> rho/rho_B (1249-1250), U1CO = U1DMCO*ROTE (1386) */
    for (int64_t c = 0; c < nc; c++) {
        float v = u_mass[c] / vol;
        v = v / g.rote;
        u1[c] = v * g.rote;
    }
    double mean8 = 0.0;
    for (int64_t c = 0; c < nc; c++) mean8 = mean8 + (double)u1[c];
    float mean = (float)(mean8 / (double)nc);
    for (int64_t c = 0; c < nc; c++) u1[c] = u1[c] / mean;
    const float ul3 = (UL_F * UL_F) * UL_F;
    *meandens = mean * (UM_F / ul3);
    if (p->no_velocities) {
        /* DIVERCO = - OMEGA0**(0.6)*RETE*HTE*(U1CO(:,:,:) - 1.0), src/avism.f90:1647-1650 */
        const float coef = (powf(p->omega0, 0.6f) * g.rete) * g.hte;
        for (int64_t c = 0; c < nc; c++) dv[c] = -(coef * (u1[c] - 1.0f));
    } else {
        orc_diver_uniform(nx, dx, u2, u3, u4, p->periodic, dv);
    }
    /* ext grids with the periodic ghost fill (src/num.f90:89-133) */
    for (int kz = 0; kz < ne; kz++)
        for (int jy = 0; jy < ne; jy++)
            for (int ix = 0; ix < ne; ix++) {
                int i = ix + low1, j = jy + low1, k = kz + low1;
                if (i < 1) i += nx; else if (i > nx) i -= nx;
                if (j < 1) j += nx; else if (j > nx) j -= nx;
                if (k < 1) k += nx; else if (k > nx) k -= nx;
                const int64_t e = (int64_t)ix + (int64_t)ne * ((int64_t)jy + (int64_t)ne * kz);
                u1co_ext[e] = u1[in_id(nx, i, j, k)];
                diverco_ext[e] = dv[in_id(nx, i, j, k)];
            }
    free(u1); free(dv);
    return AVISM_OK;
}
