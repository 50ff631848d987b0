/*
 * orc_grid.c -- oracle: level grid geometry and cosmology (test infrastructure).
 *
 * Follows src/grid.f90:3-76 (MALLA), the PBC block src/avism.f90:780-865 and
 * the cosmology of src/avism.f90:476-488, 607-616.  Every expression keeps the
 * reference's REAL*4 / REAL*8 types; the file is compiled with -ffp-contract=off.
 */
#include <math.h>
#include <string.h>
#include "avism_oracle.h"

int orc_grid_setup(const avism_params *p, avism_grid *g, float *radx)
{
    if (!p || !g || p->nx < 4 || !(p->lado0 > 0.0f)) return AVISM_ERR_ARG;
    const int nx = p->nx;
    const float lado0 = p->lado0;
    memset(g, 0, sizeof(*g));

    /* src/avism.f90:780-812: ghost-shell width and the extended box */
    int nplus = 0, low1 = 1, low2 = nx;
    float lado0plus = lado0;
    if (p->periodic) {
        float sizing = 50.0f;
        const float dx0 = lado0 / (float)nx;            /* DX = LADO0/NXX        */
        sizing = fminf(sizing, lado0 / 2.0f);           /* MIN(SIZING,LADO0/2.)  */
        const int t = (int)(sizing / dx0);              /* INT() truncates        */
        nplus = nx / 8 > t ? nx / 8 : t;                /* MAX(NXX/8, ...)       */
        low1 = -nplus + 1;
        low2 = nx + nplus;
        lado0plus = lado0 + (2.0f * (float)nplus) * dx0;
    }

    /* src/grid.f90:23-55 with LADO = LADO0-(LADO0/NXX) (src/avism.f90:816) */
    const float lado = lado0 - (lado0 / (float)nx);
    const float a = -lado / 2.0f, b = lado / 2.0f;
    const float c = (b - a) / (float)(nx - 1);
    const int rad_lo = low1 < 0 ? low1 : 0;
    const int rad_hi = low2 > nx + 1 ? low2 : nx + 1;
    const float r1 = a;
    const float r2 = r1 + (float)(2 - 1) * c;
    const float dx = r2 - r1;                            /* DXX=RADXX(2)-RADXX(1) */
    const float rnx = r1 + (float)(nx - 1) * c;

    if (radx) {
        for (int i = rad_lo; i <= rad_hi; i++) {
            float v;
            if (i >= 1 && i <= nx) v = r1 + (float)(i - 1) * c;
            else if (!p->periodic) v = (i == 0) ? r1 - c : rnx + c;   /* fictitious cells */
            else if (i < 1) v = r1 - (float)(1 - i) * dx;             /* avism.f90:840-845 */
            else v = rnx + (float)(i - nx) * dx;
            radx[i - rad_lo] = v;
        }
    }

    /* cosmology, src/avism.f90:476-488 and 607-616 (REAL*4 variables) */
    const float ache = p->ache, omega0 = p->omega0;
    const float ache0 = (float)((double)ache * 3.66e-3);
    const float rodo = (float)((double)omega0 * 3.0 * (double)(ache0 * ache0));
    const float re0 = 1.0f / 10.98f;
    float zeta = p->zeta;
    if (zeta < 0.0f) zeta = 0.0f;
    const float t1 = 1.0f + zeta;
    const float rote = rodo * ((t1 * t1) * t1);
    const float rete = re0 / (1.0f + zeta);
    const float rr = re0 / rete;
    float hte = omega0 * (((rr * rr) * rr) - 1.0f) + 1.0f;
    hte = ache * sqrtf(hte);

    g->nx = nx; g->nplus = nplus; g->low1 = low1; g->low2 = low2;
    g->ne = low2 - low1 + 1;
    g->rad_lo = rad_lo; g->rad_hi = rad_hi;
    g->dx = dx; g->rx1 = r1; g->lado = lado; g->lado0plus = lado0plus;
    g->rete = rete; g->rote = rote; g->hte = hte;
    return AVISM_OK;
}
