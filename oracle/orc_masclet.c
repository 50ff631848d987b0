/*
 * orc_masclet.c -- oracle: MASCLET input (FLAG_DATA = 0) at levels <= 1, test
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
 *
 * Level 1 (1094-1124): the gas comes from the level-1 patches.  DIVER_FINA_GAS
 * (src/divergence.f90:55-340) takes DIVER0, the central-difference divergence
 * of the base grid with its faces copied from the planes inside, and each
 * patch's own central differences inside it (2..N-1), with the patch's 2-cell
 * rim from its parent base cells' differences (averaged with the patch's at
 * index 2 and N-1, taking their place at 1 and N).  VMESH
 * (src/amr2uniform.f90:127-248) adds the patch cells into the level grid in
 * patch order, divides by FLAGAMR (which starts at 1), and gives the children
 * of every base cell that no patch refines the base cell's U1G and DIVER0.
 * DIVERDMCO stays 0 at levels above 0 (only 1129-1145 compute it, for IR <= 0).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

#define UM_F 9.1717E18f
#define UL_F 10.98f

/* DIVER0 (src/divergence.f90:140-167): central differences inside, then the
 * six faces copied from the planes inside, x, then y, then z */
static void diver0(int nh, float dx0, const float *u2, const float *u3, const float *u4, float *d)
{
#define B(i, j, k) ((int64_t)((i) - 1) + (int64_t)nh * ((int64_t)((j) - 1) + (int64_t)nh * ((k) - 1)))
    for (int k = 2; k <= nh - 1; k++)
        for (int j = 2; j <= nh - 1; j++)
            for (int i = 2; i <= nh - 1; i++) {
                float b21 = u2[B(i + 1, j, k)] - u2[B(i - 1, j, k)];
                b21 = b21 / (2.0f * dx0);
                float b32 = u3[B(i, j + 1, k)] - u3[B(i, j - 1, k)];
                b32 = b32 / (2.0f * dx0);
                float b43 = u4[B(i, j, k + 1)] - u4[B(i, j, k - 1)];
                b43 = b43 / (2.0f * dx0);
                d[B(i, j, k)] = (b21 + b32) + b43;
            }
    for (int k = 1; k <= nh; k++)
        for (int j = 1; j <= nh; j++) { d[B(1, j, k)] = d[B(2, j, k)]; }
    for (int k = 1; k <= nh; k++)
        for (int j = 1; j <= nh; j++) { d[B(nh, j, k)] = d[B(nh - 1, j, k)]; }
    for (int k = 1; k <= nh; k++)
        for (int i = 1; i <= nh; i++) { d[B(i, 1, k)] = d[B(i, 2, k)]; }
    for (int k = 1; k <= nh; k++)
        for (int i = 1; i <= nh; i++) { d[B(i, nh, k)] = d[B(i, nh - 1, k)]; }
    for (int j = 1; j <= nh; j++)
        for (int i = 1; i <= nh; i++) { d[B(i, j, 1)] = d[B(i, j, 2)]; }
    for (int j = 1; j <= nh; j++)
        for (int i = 1; i <= nh; i++) { d[B(i, j, nh)] = d[B(i, j, nh - 1)]; }
#undef B
}

/* level 1: UGR and DIVR on the level grid (nx = 2 nhy) from the patches */
static int amr_level1(const avism_params *p, int nhy, const float *u1g, const float *u2g, const float *u3g,
                      const float *u4g, const avism_patches *a, float *ugr, float *divr)
{
    avism_grid g, g0;
    orc_grid_setup(p, &g, NULL);
    avism_params p0 = *p;
    p0.nx = nhy;
    orc_grid_setup(&p0, &g0, NULL);
    float *radx = (float *)malloc((size_t)(g.rad_hi - g.rad_lo + 1) * sizeof(float));
    orc_grid_setup(p, &g, radx);
    const float dx0 = g0.dx, dxr_div = dx0 / 2.0f, dxr = g.dx, rx1 = radx[1 - g.rad_lo];
    free(radx);
    const int nx = g.nx, nh = nhy;
    const int64_t nc = (int64_t)nx * nx * nx, n0 = (int64_t)nh * nh * nh;
    float *d0 = (float *)calloc((size_t)n0, sizeof(float));
    diver0(nh, dx0, u2g, u3g, u4g, d0);
    int32_t *flagamr = (int32_t *)malloc((size_t)nc * sizeof(int32_t));
    uint8_t *flagr = (uint8_t *)calloc((size_t)n0, 1);
    for (int64_t c = 0; c < nc; c++) { flagamr[c] = 1; ugr[c] = 0.0f; divr[c] = 0.0f; }
    int st = AVISM_OK;
    /* the corners' level-grid offsets must fit an int before the truncation */
    for (int ip = 0; ip < a->npatch && !st; ip++) {
        const float rc[3] = {a->rx[ip], a->ry[ip], a->rz[ip]};
        for (int ax = 0; ax < 3; ax++) {
            const float f = (((rc[ax] - 0.5f * dxr) - rx1) / dxr) + 0.5f;
            if (!isfinite(f) || fabsf(f) >= 1.0e9f) st = AVISM_ERR_ARG;
        }
    }
    for (int ip = 0; ip < a->npatch && !st; ip++) {
        const int n1 = a->nx[ip], n2 = a->ny[ip], n3 = a->nz[ip];
        const int l1 = a->ix[ip], l2 = a->iy[ip], l3 = a->iz[ip];
        const int64_t o = a->offset[ip];
#define P(i, j, k) (o + (int64_t)((i) - 1) + (int64_t)n1 * ((int64_t)((j) - 1) + (int64_t)n2 * ((k) - 1)))
#define B(i, j, k) ((int64_t)((i) - 1) + (int64_t)nh * ((int64_t)((j) - 1) + (int64_t)nh * ((k) - 1)))
        /* the patch's divergence: inside from its own cells, the rim from its base cells */
        const int64_t np = (int64_t)n1 * n2 * n3;
        float *dv = (float *)calloc((size_t)np, sizeof(float));
        for (int k = 2; k <= n3 - 1; k++)
            for (int j = 2; j <= n2 - 1; j++)
                for (int i = 2; i <= n1 - 1; i++) {
                    float b21 = a->u12g[P(i + 1, j, k)] - a->u12g[P(i - 1, j, k)];
                    b21 = b21 / (2.0f * dxr_div);
                    float b32 = a->u13g[P(i, j + 1, k)] - a->u13g[P(i, j - 1, k)];
                    b32 = b32 / (2.0f * dxr_div);
                    float b43 = a->u14g[P(i, j, k + 1)] - a->u14g[P(i, j, k - 1)];
                    b43 = b43 / (2.0f * dxr_div);
                    dv[P(i, j, k) - o] = (b21 + b32) + b43;
                }
        for (int k = 1; k <= n3; k++)
            for (int j = 1; j <= n2; j++)
                for (int i = 1; i <= n1; i++) {
                    float aux = 0.0f;
                    if (i < 3 || i > n1 - 2 || j < 3 || j > n2 - 2 || k < 3 || k > n3 - 2) {
                        const int c1 = (i + 1) / 2 + l1 - 1, c2 = (j + 1) / 2 + l2 - 1, c3 = (k + 1) / 2 + l3 - 1;
                        if (c1 < 2 || c1 > nh - 1 || c2 < 2 || c2 > nh - 1 || c3 < 2 || c3 > nh - 1) {
                            st = AVISM_ERR_ARG;       /* the reference reads outside U2G there */
                            continue;
                        }
                        float b21 = u2g[B(c1 + 1, c2, c3)] - u2g[B(c1 - 1, c2, c3)];
                        b21 = b21 / (2.0f * dx0);
                        float b32 = u3g[B(c1, c2 + 1, c3)] - u3g[B(c1, c2 - 1, c3)];
                        b32 = b32 / (2.0f * dx0);
                        float b43 = u4g[B(c1, c2, c3 + 1)] - u4g[B(c1, c2, c3 - 1)];
                        b43 = b43 / (2.0f * dx0);
                        aux = (b21 + b32) + b43;
                    }
                    float *v = &dv[P(i, j, k) - o];
                    if (i == 2 || i == n1 - 1 || j == 2 || j == n2 - 1 || k == 2 || k == n3 - 1)
                        *v = 0.5f * (aux + *v);
                    if (i == 1 || i == n1 || j == 1 || j == n2 || k == 1 || k == n3) *v = aux;
                }
        /* VMESH: the patch cells into the level grid */
        const int xr1 = (int)((((a->rx[ip] - 0.5f * dxr) - rx1) / dxr) + 0.5f);
        const int yr1 = (int)((((a->ry[ip] - 0.5f * dxr) - rx1) / dxr) + 0.5f);
        const int zr1 = (int)((((a->rz[ip] - 0.5f * dxr) - rx1) / dxr) + 0.5f);
        for (int k = 1; k <= n3 && !st; k++)
            for (int j = 1; j <= n2 && !st; j++)
                for (int i = 1; i <= n1; i++) {
                    const int xr = xr1 + i, yr = yr1 + j, zr = zr1 + k;
                    if (xr < 1 || xr > nx || yr < 1 || yr > nx || zr < 1 || zr > nx) {
                        st = AVISM_ERR_ARG;           /* the reference writes outside its grid there */
                        break;
                    }
                    const int64_t c = (int64_t)(xr - 1) + (int64_t)nx * ((int64_t)(yr - 1) + (int64_t)nx * (zr - 1));
                    flagamr[c] = flagamr[c] + 1;
                    ugr[c] = ugr[c] + a->u11g[P(i, j, k)];
                    divr[c] = divr[c] + dv[P(i, j, k) - o];
                    flagr[B((xr - 1) / 2 + 1, (yr - 1) / 2 + 1, (zr - 1) / 2 + 1)] = 1;
                }
        free(dv);
#undef P
    }
    if (!st) {
        for (int64_t c = 0; c < nc; c++) {
            ugr[c] = ugr[c] / (float)flagamr[c];
            divr[c] = divr[c] / (float)flagamr[c];
        }
        for (int k0 = 1; k0 <= nh; k0++)
            for (int j0 = 1; j0 <= nh; j0++)
                for (int i0 = 1; i0 <= nh; i0++) {
                    if (flagr[B(i0, j0, k0)]) continue;
                    for (int kr = 2 * k0 - 1; kr <= 2 * k0; kr++)
                        for (int jr = 2 * j0 - 1; jr <= 2 * j0; jr++)
                            for (int ir = 2 * i0 - 1; ir <= 2 * i0; ir++) {
                                const int64_t c = (int64_t)(ir - 1) + (int64_t)nx * ((int64_t)(jr - 1) + (int64_t)nx * (kr - 1));
                                ugr[c] = u1g[B(i0, j0, k0)];
                                divr[c] = d0[B(i0, j0, k0)];
                            }
                }
    }
#undef B
    free(d0); free(flagamr); free(flagr);
    return st;
}

int orc_masclet_fields(const avism_params *p, int32_t nhy, const float *u1g, const float *u2g, const float *u3g,
                       const float *u4g, const avism_patches *amr, int64_t n, const float *x, const float *y,
                       const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                       float *u1co_ext, float *diverco_ext, float *meandens)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    if (p->level > 1) return AVISM_ERR_UNSUPPORTED;              /* VMESH beyond level 1 */
    if (p->level == 1 ? (!amr || p->nx != 2 * nhy) : (((int64_t)p->nx << (-p->level)) != (int64_t)nhy))
        return AVISM_ERR_ARG;
    if (p->flag_dens < 0 || p->flag_dens > 2 || p->flag_div < -1 || p->flag_div > 2) return AVISM_ERR_ARG;
    if (p->level == 1) {
        if (amr->npatch < 0 || !amr->offset || amr->offset[0] < 0) return AVISM_ERR_ARG;
        for (int q = 0; q < amr->npatch; q++)
            if (amr->nx[q] < 1 || amr->ny[q] < 1 || amr->nz[q] < 1 || amr->nx[q] > (1 << 20) ||
                amr->ny[q] > (1 << 20) || amr->nz[q] > (1 << 20) ||
                amr->offset[q + 1] - amr->offset[q] != (int64_t)amr->nx[q] * amr->ny[q] * amr->nz[q])
                return AVISM_ERR_ARG;
    }
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
    if (!st && p->level == 1) st = amr_level1(p, nhy, u1g, u2g, u3g, u4g, amr, co[0], dg);
    if (!st) {
        const float *in[4] = {u1g, u2g, u3g, u4g};
        if (p->level <= 0) orc_level_grids(p, nhy, need_gas_v ? 4 : 1, in, co);
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
            /* level 1: DIVERGCO = DIVR (already in dg), DIVERDMCO = 0 */
            if (need_gas_v && p->level <= 0) orc_diver_uniform(nx, dx, co[1], co[2], co[3], p->periodic, dg);
            if (p->flag_div <= 1 && p->level <= 0) orc_diver_uniform(nx, dx, d2, d3, d4, p->periodic, dd);
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
