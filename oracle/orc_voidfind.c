/*
 * orc_voidfind.c -- oracle: MARK_ALL, VOIDFIND and INDEXX (test infrastructure).
 *
 * Restates src/voidfinding.f90:13-55 (MARK_ALL), 59-713 (VOIDFIND) and
 * src/num.f90:2-84 (INDEXX, the Numerical Recipes index quicksort).
 *
 * Cube growth (src/voidfinding.f90:449-704) is restated in closed form.  The
 * reference grows all six faces together, one shell per pass, while every face
 * passes; reaching the NSEC=1 border sets the boundary flags, after which one
 * more pass only decides FLAG2: it is set when, along some axis, exactly one
 * side sits at the border (the pass evaluates that axis' faces only if not both
 * of its flags are set).  A cube that touches the border on all six sides stops
 * with FLAG2 unchanged.  Single-cell cubes are rejected.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

/* ---- INDEXX (src/num.f90:2-84), arrays 1-based through offset pointers --- */
int orc_indexx(int32_t n, const float *arr_in, int32_t *indx_out)
{
    enum { M = 7, NSTACK = 50 };
    if (n < 0) return AVISM_ERR_ARG;
    const float *arr = arr_in - 1;
    int32_t *indx = indx_out - 1;
    int32_t istack[NSTACK + 1];
    for (int32_t j = 1; j <= n; j++) indx[j] = j;
    int32_t jstack = 0, l = 1, ir = n;
    for (;;) {
        if (ir - l < M) {
            /* straight insertion on indx(l..ir); the scan may run below l */
            for (int32_t j = l + 1; j <= ir; j++) {
                const int32_t indxt = indx[j];
                const float a = arr[indxt];
                int32_t i;
                for (i = j - 1; i >= 1; i--) {
                    if (arr[indx[i]] <= a) break;
                    indx[i + 1] = indx[i];
                }
                indx[i + 1] = indxt;
            }
            if (jstack == 0) return AVISM_OK;
            ir = istack[jstack];
            l = istack[jstack - 1];
            jstack -= 2;
        } else {
            int32_t t;
            const int32_t k = (l + ir) / 2;
            t = indx[k]; indx[k] = indx[l + 1]; indx[l + 1] = t;
            if (arr[indx[l + 1]] > arr[indx[ir]]) { t = indx[l + 1]; indx[l + 1] = indx[ir]; indx[ir] = t; }
            if (arr[indx[l]] > arr[indx[ir]]) { t = indx[l]; indx[l] = indx[ir]; indx[ir] = t; }
            if (arr[indx[l + 1]] > arr[indx[l]]) { t = indx[l + 1]; indx[l + 1] = indx[l]; indx[l] = t; }
            int32_t i = l + 1, j = ir;
            const int32_t indxt = indx[l];
            const float a = arr[indxt];
            for (;;) {
                do i++; while (arr[indx[i]] < a);
                do j--; while (arr[indx[j]] > a);
                if (j < i) break;
                t = indx[i]; indx[i] = indx[j]; indx[j] = t;
            }
            indx[l] = indx[j];
            indx[j] = indxt;
            jstack += 2;
            if (jstack > NSTACK) return AVISM_ERR_INTERNAL;   /* 'NSTACK too small in indexx' */
            if (ir - i + 1 >= j - l) {
                istack[jstack] = ir; istack[jstack - 1] = i; ir = j - 1;
            } else {
                istack[jstack] = j - 1; istack[jstack - 1] = l; l = i;
            }
        }
    }
}

/* ---- MARK_ALL + the six directional flag grids --------------------------- */
typedef struct {
    int low1, low2, ne;
    const float *u1, *dv;
    const int8_t *smask;
    const int32_t *marcap;
    uint8_t *fl;
} vf_grid;

static inline int64_t eid(const vf_grid *G, int i, int j, int k)
{
    return (int64_t)(i - G->low1) + (int64_t)G->ne * ((int64_t)(j - G->low1) + (int64_t)G->ne * (int64_t)(k - G->low1));
}
static inline int sm(const vf_grid *G, int64_t e) { return G->smask ? G->smask[e] != 0 : 1; }
static inline int32_t mp(const vf_grid *G, int64_t e) { return G->marcap ? G->marcap[e] : -1; }

/* gradient test value f32((a-b)/(2.D0*DX)) as in src/voidfinding.f90:290 */
static inline float grad32(float a, float b, float dx)
{
    return (float)((double)(a - b) / (2.0 * (double)dx));
}

/* One direction's face flag of cell c; returns -1 if the masked-neighbour CYCLE
 * of the reference stops the remaining directions. axis 0..2, sgn +1/-1. */
static int dir_flag(const vf_grid *G, const avism_params *p, float dx, int c[3], int axis, int sgn)
{
    const int low1 = G->low1, low2 = G->low2;
    const int pos = c[axis];
    if (sgn > 0 ? pos >= low2 - 1 : pos <= low1 + 1) return 1;
    int nb[3] = {c[0], c[1], c[2]};
    const int ii = pos + sgn;
    nb[axis] = ii;
    const int64_t en = eid(G, nb[0], nb[1], nb[2]);
    if (!sm(G, en)) return -1;
    int f = 0;
    if (ii == (sgn > 0 ? low2 : low1)) {
        if (G->dv[en] < p->div_thre) f = 1;
        if (G->u1[en] >= p->dens_thre2 + 1.0f) f = 1;
        return f;
    }
    int a[3] = {nb[0], nb[1], nb[2]}, b[3] = {nb[0], nb[1], nb[2]};
    a[axis] = ii + sgn; b[axis] = ii - sgn;
    const float dd = grad32(G->u1[eid(G, a[0], a[1], a[2])], G->u1[eid(G, b[0], b[1], b[2])], dx);
    if (dd >= p->grad_thre) f = 1;
    /* FLAG_NEXT_GRAD = 1: the next cell's gradient must agree */
    if (f == 1 && (sgn > 0 ? ii < low2 - 1 : ii > low1 + 1)) {
        int a2[3] = {nb[0], nb[1], nb[2]};
        a2[axis] = ii + 2 * sgn;
        const float dd2 = grad32(G->u1[eid(G, a2[0], a2[1], a2[2])], G->u1[en], dx);
        if (dd2 < p->grad_thre) f = 0;
    }
    /* FLAG_DIV_EDGE = 1 */
    if (G->dv[en] < p->div_thre) f = 1;
    if (G->u1[en] >= p->dens_thre2 + 1.0f) f = 1;
    return f;
}

static void make_flags(const vf_grid *G, const avism_params *p, float dx)
{
    const int low1 = G->low1, low2 = G->low2;
    #pragma omp parallel for collapse(2)
    for (int k = low1; k <= low2; k++)
        for (int j = low1; j <= low2; j++)
            for (int i = low1; i <= low2; i++) {
                const int64_t e = eid(G, i, j, k);
                uint8_t f = 0;
                if (sm(G, e) && mp(G, e) != 0) {
                    f |= 0x80;                                         /* FLAG_SUB */
                    if (G->u1[e] < p->dens_thre + 1.0f && G->dv[e] > 0.0f) f |= 0x01;   /* FLAGV */
                }
                int c[3] = {i, j, k};
                /* order +X, -X, +Y, -Y, +Z, -Z; bits X1=1, X2=2, Y1=3, Y2=4, Z1=5, Z2=6 */
                static const int ax[6] = {0, 0, 1, 1, 2, 2};
                static const int sg[6] = {+1, -1, +1, -1, +1, -1};
                static const int bit[6] = {2, 1, 4, 3, 6, 5};
                for (int d = 0; d < 6; d++) {
                    const int r = dir_flag(G, p, dx, c, ax[d], sg[d]);
                    if (r < 0) break;
                    if (r) f |= (uint8_t)(1u << bit[d]);
                }
                G->fl[e] = f;
            }
}

/* all six faces of the cube of half-width w around c pass the growth test of
 * src/voidfinding.f90:500-619 */
static int faces_pass(const vf_grid *G, const int c[3], int w, int32_t indv)
{
    static const int bitm[3] = {1, 3, 5};   /* minus-side bit, plus = +1 */
    for (int axis = 0; axis < 3; axis++) {
        const int u = (axis + 1) % 3, v = (axis + 2) % 3;
        for (int s = -1; s <= 1; s += 2) {
            const int face = c[axis] + s * w;
            const uint8_t fb = (uint8_t)(1u << (s > 0 ? bitm[axis] + 1 : bitm[axis]));
            for (int b = c[v] - w; b <= c[v] + w; b++)
                for (int a = c[u] - w; a <= c[u] + w; a++) {
                    int cell[3], nb[3];
                    cell[axis] = face; cell[u] = a; cell[v] = b;
                    nb[axis] = face + s; nb[u] = a; nb[v] = b;
                    const int64_t en = eid(G, nb[0], nb[1], nb[2]);
                    if (!(G->fl[en] & 0x80)) return 0;
                    if (mp(G, en) != indv) return 0;
                    if (G->fl[eid(G, cell[0], cell[1], cell[2])] & fb) return 0;
                }
        }
    }
    return 1;
}

int orc_voidfind(const avism_params *p, const float *u1co_ext, const float *diverco_ext,
                 const int8_t *smask_ext, const int32_t *marcap_ext, const float *reqp,
                 avism_cubes *cubes, int32_t *nvoid_out, uint8_t *flags_ext,
                 int32_t *ncand_out, int32_t *cand_order)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    const int low1 = g.low1, low2 = g.low2, ne = g.ne;
    const int64_t next = (int64_t)ne * ne * ne;
    const float dx = g.dx, rx1 = g.rx1;
    vf_grid G = {low1, low2, ne, u1co_ext, diverco_ext, smask_ext, marcap_ext, NULL};
    G.fl = flags_ext ? flags_ext : (uint8_t *)malloc((size_t)next);
    if (!G.fl) return AVISM_ERR_OOM;
    make_flags(&G, p, dx);

    /* candidates in K,J,I order (src/voidfinding.f90:161-176) */
    int64_t ncand = 0;
    for (int64_t e = 0; e < next; e++) if (G.fl[e] & 0x01) ncand++;
    if (ncand > INT32_MAX) { if (!flags_ext) free(G.fl); return AVISM_ERR_ARG; }
    float *ddd = (float *)malloc((size_t)(ncand ? ncand : 1) * sizeof(float));
    int64_t *pos = (int64_t *)malloc((size_t)(ncand ? ncand : 1) * sizeof(int64_t));
    int32_t *ord = (int32_t *)malloc((size_t)(ncand ? ncand : 1) * sizeof(int32_t));
    int64_t ii = 0;
    for (int64_t e = 0; e < next; e++)
        if (G.fl[e] & 0x01) { ddd[ii] = diverco_ext[e]; pos[ii] = e; ii++; }
    st = orc_indexx((int32_t)ncand, ddd, ord);
    if (ncand_out) *ncand_out = (int32_t)ncand;

    int32_t *marca_aux = (int32_t *)calloc((size_t)next, sizeof(int32_t));
    int32_t nvoid = 0;
    for (int64_t l1 = 0; l1 < ncand && st == AVISM_OK; l1++) {
        const int64_t e = pos[ord[ncand - 1 - l1] - 1];   /* descending divergence */
        if (cand_order) cand_order[l1] = (int32_t)e;
        const int c[3] = {(int)(e % ne) + low1, (int)((e / ne) % ne) + low1, (int)(e / ((int64_t)ne * ne)) + low1};
        if (marca_aux[e] > 0) continue;
        if (c[0] <= low1 + 1 || c[1] <= low1 + 1 || c[2] <= low1 + 1 ||
            c[0] >= low2 - 1 || c[1] >= low2 - 1 || c[2] >= low2 - 1) continue;
        if (nvoid + 1 > p->nvoid_max) { st = AVISM_ERR_NVOID_MAX; break; }
        const int32_t indv = mp(&G, e);
        int flag1 = 0;
        if (indv > 0 && reqp && reqp[indv - 1] < p->rmin_sub) flag1 = 1;
        /* growth, closed form of src/voidfinding.f90:496-679 */
        int w = 0, f2 = 0;
        if (!flag1) {
            for (;;) {
                if (!faces_pass(&G, c, w, indv)) break;
                w++;
                int blo[3], bhi[3], any = 0, all = 1;
                for (int a = 0; a < 3; a++) {
                    blo[a] = c[a] - w <= low1 + 1;
                    bhi[a] = c[a] + w >= low2 - 1;
                    any |= blo[a] | bhi[a];
                    all &= blo[a] & bhi[a];
                }
                if (any) {
                    if (!all)
                        for (int a = 0; a < 3; a++)
                            if ((blo[a] || bhi[a]) && !(blo[a] && bhi[a])) f2 = 1;
                    break;
                }
            }
        }
        if (w == 0) f2 = 1;
        /* edge test of src/voidfinding.f90:674-679 (never true with NSEC=1, kept) */
        for (int a = 0; a < 3; a++) if (c[a] - w == low1 || c[a] + w == low2) f2 = 1;
        if (f2) continue;
        const int32_t id = nvoid++;
        const int x0 = c[0] - w, x1 = c[0] + w, y0 = c[1] - w, y1 = c[1] + w, z0 = c[2] - w, z1 = c[2] + w;
        cubes->inicio_x[id] = x0; cubes->final_x[id] = x1;
        cubes->inicio_y[id] = y0; cubes->final_y[id] = y1;
        cubes->inicio_z[id] = z0; cubes->final_z[id] = z1;
        cubes->icx[id] = c[0]; cubes->icy[id] = c[1]; cubes->icz[id] = c[2];
        cubes->father[id] = indv;
        const float A = (float)(x1 - x0 + 1) * dx, B = (float)(y1 - y0 + 1) * dx, C = (float)(z1 - z0 + 1) * dx;
        cubes->vol[id] = (A * B) * C;
        cubes->rini_x[id] = (rx1 + (float)(x0 - 1) * dx) - 0.5f * dx;
        cubes->rfin_x[id] = (rx1 + (float)(x1 - 1) * dx) + 0.5f * dx;
        cubes->rini_y[id] = (rx1 + (float)(y0 - 1) * dx) - 0.5f * dx;
        cubes->rfin_y[id] = (rx1 + (float)(y1 - 1) * dx) + 0.5f * dx;
        cubes->rini_z[id] = (rx1 + (float)(z0 - 1) * dx) - 0.5f * dx;
        cubes->rfin_z[id] = (rx1 + (float)(z1 - 1) * dx) + 0.5f * dx;
        for (int k = z0; k <= z1; k++)
            for (int j = y0; j <= y1; j++)
                for (int i = x0; i <= x1; i++) marca_aux[eid(&G, i, j, k)] = nvoid;
    }
    *nvoid_out = nvoid;
    free(marca_aux); free(ddd); free(pos); free(ord);
    if (!flags_ext) free(G.fl);
    return st;
}
