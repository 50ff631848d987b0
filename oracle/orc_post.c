/*
 * orc_post.c -- oracle: volume ordering, MERGE_VOID and post-processing
 * (test infrastructure).
 *
 * Restates src/avism.f90:1738-1745 (INDEXX on VOL, reversed), MERGE_VOID
 * (src/voidfinding.f90:718-999), the post-processing of src/avism.f90:1797-1973,
 * VOID_SHAPE/JACOBI/SORT (src/shape.f90), SIMPLE_CONNECTION_FAST
 * (src/voidfinding.f90:1007-1162) and VOID_PERIODIC (1367-1569).
 *
 * The per-void whole-grid WHERE rewrites of the reference are replaced by
 * label bookkeeping with the same results (each removal only touches cells
 * and owners equal to the removed id, so the decisions are independent).
 * Ball-search results in MERGE_VOID are visited in (squared distance, cube id)
 * order.  VOID_PERIODIC's candidate list records each kept void twice
 * (src/voidfinding.f90:1395-1420); the second visit is a no-op, so each kept
 * void is visited once here (and no list overflows).
 */
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

typedef struct {
    int low1, low2, ne, nx;
    int32_t *marca;
} pgrid;

static inline int64_t pid(const pgrid *G, int i, int j, int k)
{
    return (int64_t)(i - G->low1) + (int64_t)G->ne * ((int64_t)(j - G->low1) + (int64_t)G->ne * (int64_t)(k - G->low1));
}

static void paint(pgrid *G, const avism_cubes *cb, int32_t cube, int32_t val)
{
    const int c = cube - 1;
    for (int k = cb->inicio_z[c]; k <= cb->final_z[c]; k++)
        for (int j = cb->inicio_y[c]; j <= cb->final_y[c]; j++)
            for (int i = cb->inicio_x[c]; i <= cb->final_x[c]; i++) {
                const int64_t e = pid(G, i, j, k);
                if (G->marca[e] == 0) G->marca[e] = val;
            }
}

/* GC(IND0) <- volume-weighted centre, src/voidfinding.f90:867-872 */
static void absorb_centre(float *gxc, float *gyc, float *gzc, float *vol, int32_t i0, int32_t i1)
{
    const float v0 = vol[i0 - 1], v1 = vol[i1 - 1];
    gxc[i0 - 1] = (gxc[i0 - 1] * v0 + gxc[i1 - 1] * v1) / (v0 + v1);
    gyc[i0 - 1] = (gyc[i0 - 1] * v0 + gyc[i1 - 1] * v1) / (v0 + v1);
    gzc[i0 - 1] = (gzc[i0 - 1] * v0 + gzc[i1 - 1] * v1) / (v0 + v1);
    vol[i0 - 1] = v0 + v1;
}

/* ---- JACOBI (src/shape.f90:46-134), REAL*4 with the REAL*8 literals' promotions */
static void jacobi3(float a[3][3], float d[3])
{
    const int n = 3;
    float b[3], z[3];
    for (int ip = 0; ip < n; ip++) { b[ip] = a[ip][ip]; d[ip] = b[ip]; z[ip] = 0.0f; }
    for (int i = 1; i <= 50; i++) {
        float sm = 0.0f;
        for (int ip = 0; ip < n - 1; ip++)
            for (int iq = ip + 1; iq < n; iq++) sm = sm + fabsf(a[ip][iq]);
        if (sm == 0.0f) return;
        float tresh;
        if (i < 4) tresh = (float)(0.2 * (double)(sm * sm));
        else tresh = 0.0f;
        for (int ip = 0; ip < n - 1; ip++)
            for (int iq = ip + 1; iq < n; iq++) {
                float g = (float)(100.0 * (double)fabsf(a[ip][iq]));
                if (i > 4 && fabsf(d[ip]) + g == fabsf(d[ip]) && fabsf(d[iq]) + g == fabsf(d[iq])) {
                    a[ip][iq] = 0.0f;
                } else if (fabsf(a[ip][iq]) > tresh) {
                    float h = d[iq] - d[ip];
                    float t;
                    if (fabsf(h) + g == fabsf(h)) {
                        t = a[ip][iq] / h;
                    } else {
                        const float theta = (float)(0.5 * (double)h / (double)a[ip][iq]);
                        t = (float)(1.0 / ((double)fabsf(theta) + sqrt(1.0 + (double)(theta * theta))));
                        if (theta < 0.0f) t = -t;
                    }
                    const float c = (float)(1.0 / sqrt(1.0 + (double)(t * t)));
                    const float s = t * c;
                    const float tau = (float)((double)s / (1.0 + (double)c));
                    h = t * a[ip][iq];
                    z[ip] = z[ip] - h;
                    z[iq] = z[iq] + h;
                    d[ip] = d[ip] - h;
                    d[iq] = d[iq] + h;
                    a[ip][iq] = 0.0f;
                    for (int j = 0; j < ip; j++) {
                        const float gg = a[j][ip], hh = a[j][iq];
                        a[j][ip] = gg - s * (hh + gg * tau);
                        a[j][iq] = hh + s * (gg - hh * tau);
                    }
                    for (int j = ip + 1; j < iq; j++) {
                        const float gg = a[ip][j], hh = a[j][iq];
                        a[ip][j] = gg - s * (hh + gg * tau);
                        a[j][iq] = hh + s * (gg - hh * tau);
                    }
                    for (int j = iq + 1; j < n; j++) {
                        const float gg = a[ip][j], hh = a[iq][j];
                        a[ip][j] = gg - s * (hh + gg * tau);
                        a[iq][j] = hh + s * (gg - hh * tau);
                    }
                }
            }
        for (int ip = 0; ip < n; ip++) { b[ip] = b[ip] + z[ip]; d[ip] = b[ip]; z[ip] = 0.0f; }
    }
}

/* SORT (src/shape.f90:2-29): descending selection sort keeping the last maximum */
static void sort_desc3(float d[3])
{
    const int n = 3;
    for (int i = 0; i < n - 1; i++) {
        int k = i;
        float p = d[i];
        for (int j = i + 1; j < n; j++)
            if (d[j] >= p) { k = j; p = d[j]; }
        if (k != i) { d[k] = d[i]; d[i] = p; }
    }
}

typedef struct { int64_t *c; int64_t n, cap; } cell_vec;

static void cv_push(cell_vec *v, int64_t e)
{
    if (v->n == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 16;
        v->c = (int64_t *)realloc(v->c, (size_t)v->cap * sizeof(int64_t));
    }
    v->c[v->n++] = e;
}

int orc_merge_post(const avism_params *p, int32_t nvoid, const avism_cubes *cb,
                   const float *u1co_ext, float meandens, avism_voids *out)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    if (nvoid < 0) return AVISM_ERR_ARG;
    float *radx = (float *)malloc((size_t)(g.rad_hi - g.rad_lo + 1) * sizeof(float));
    orc_grid_setup(p, &g, radx);
#define RAD(i) radx[(i) - g.rad_lo]
    const int low1 = g.low1, low2 = g.low2, ne = g.ne, nx = g.nx;
    const int64_t next = (int64_t)ne * ne * ne;
    const float dx = g.dx;
    const double pi = acos(-1.0);
    pgrid G = {low1, low2, ne, nx, NULL};
    G.marca = out->marca ? out->marca : (int32_t *)malloc((size_t)next * sizeof(int32_t));
    int32_t *marca = G.marca;

    const int32_t nv = nvoid;
    int32_t *indice = out->indice, *uvoid = out->uvoid, *ncellv = out->ncellv;
    float *volnew = out->volnew, *gxc = out->gxc, *gyc = out->gyc, *gzc = out->gzc;
    const int32_t *father = cb->father;

    /* INDEXX(VOL) lowest->highest, reversed: largest first (avism.f90:1738-1745) */
    int32_t *ind2 = (int32_t *)malloc((size_t)(nv ? nv : 1) * sizeof(int32_t));
    orc_indexx(nv, cb->vol, ind2);
    for (int32_t i = 0; i < nv; i++) indice[i] = ind2[nv - 1 - i];
    free(ind2);

    /* ---- MERGE_VOID ------------------------------------------------------ */
    for (int32_t i = 0; i < nv; i++) {
        gxc[i] = RAD(1) + (float)(cb->icx[i] - 1) * dx;
        gyc[i] = RAD(1) + (float)(cb->icy[i] - 1) * dx;
        gzc[i] = RAD(1) + (float)(cb->icz[i] - 1) * dx;
        volnew[i] = ((cb->rfin_x[i] - cb->rini_x[i]) * (cb->rfin_y[i] - cb->rini_y[i])) *
                    (cb->rfin_z[i] - cb->rini_z[i]);
    }
    orc_kdtree *tree = orc_kd_build(nv, gxc, gyc, gzc, p->periodic ? g.lado0plus : 0.0f);
    char *major = (char *)calloc((size_t)(nv ? nv : 1), 1);
    for (int32_t i = 0; i < nv; i++) uvoid[i] = -1;
    memset(marca, 0, (size_t)next * sizeof(int32_t));
    int32_t nvoid2 = nv;
    int64_t *bidx = NULL; float *bd2 = NULL; int64_t bcap = 0;
    const int nbuff = 1;
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind1 = indice[I];
        const int c1 = ind1 - 1;
        int32_t ind0, indp;
        if (uvoid[c1] > 0) {
            ind0 = uvoid[c1];
            indp = father[ind0 - 1];
        } else {
            ind0 = ind1;
            indp = father[ind0 - 1];
            int ix1 = cb->inicio_x[c1] - 1, ix2 = cb->final_x[c1] + 1;
            int jy1 = cb->inicio_y[c1] - 1, jy2 = cb->final_y[c1] + 1;
            int kz1 = cb->inicio_z[c1] - 1, kz2 = cb->final_z[c1] + 1;
            if (ix1 < low1) ix1 = low1; if (ix2 > low2) ix2 = low2;
            if (jy1 < low1) jy1 = low1; if (jy2 > low2) jy2 = low2;
            if (kz1 < low1) kz1 = low1; if (kz2 > low2) kz2 = low2;
            int dist = INT_MAX;
            for (int kz = kz1; kz <= kz2; kz++)
                for (int jy = jy1; jy <= jy2; jy++)
                    for (int ix = ix1; ix <= ix2; ix++) {
                        const int32_t mv = marca[pid(&G, ix, jy, kz)];
                        if (mv > 0) {
                            if (father[mv - 1] != indp) continue;
                            const int ddx = cb->icx[c1] - ix, ddy = cb->icy[c1] - jy, ddz = cb->icz[c1] - kz;
                            const int d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            if (d2 < dist) { ind0 = mv; dist = d2; }
                        }
                    }
            if (ind0 != ind1) {
                uvoid[c1] = ind0;
                absorb_centre(gxc, gyc, gzc, volnew, ind0, ind1);
                paint(&G, cb, ind1, ind0);
                nvoid2--;
            } else {
                paint(&G, cb, ind0, ind0);
                major[ind0 - 1] = 1;
            }
        }
        /* absorb overlapping cubes found by a ball search on cube centres */
        const int ix1 = cb->inicio_x[c1] - nbuff, ix2 = cb->final_x[c1] + nbuff;
        const int jy1 = cb->inicio_y[c1] - nbuff, jy2 = cb->final_y[c1] + nbuff;
        const int kz1 = cb->inicio_z[c1] - nbuff, kz2 = cb->final_z[c1] + nbuff;
        const float tx = gxc[c1], ty = gyc[c1], tz = gzc[c1];
        const float rthis = (sqrtf(3.0f) / 2.0f) * powf(volnew[c1], 1.0f / 3.0f);
        const float rr = 2.0f * rthis + ((2.1f * sqrtf(3.0f)) * dx) * (float)nbuff;
        const int64_t cnt = orc_kd_ball(tree, tx, ty, tz, rr, &bidx, &bd2, &bcap);
        for (int64_t q = 0; q < cnt; q++) {
            const int32_t ind2c = (int32_t)bidx[q];          /* 0-based */
            const int32_t i2 = ind2c + 1;
            if (i2 == ind1) continue;
            if (major[ind2c]) continue;
            if (uvoid[ind2c] >= 0) continue;
            if (indp != father[ind2c]) continue;
            const int ix3 = cb->inicio_x[ind2c] - nbuff, ix4 = cb->final_x[ind2c] + nbuff;
            const int jy3 = cb->inicio_y[ind2c] - nbuff, jy4 = cb->final_y[ind2c] + nbuff;
            const int kz3 = cb->inicio_z[ind2c] - nbuff, kz4 = cb->final_z[ind2c] + nbuff;
            if (ix1 <= ix4 && ix3 <= ix2 && jy1 <= jy4 && jy3 <= jy2 && kz1 <= kz4 && kz3 <= kz2) {
                uvoid[ind2c] = ind0;
                absorb_centre(gxc, gyc, gzc, volnew, ind0, i2);
                paint(&G, cb, i2, ind0);
                nvoid2--;
            }
        }
    }
    free(bidx); free(bd2); free(major);
    orc_kd_free(tree);
    out->nvoid2 = nvoid2;

    /* ---- post-processing ------------------------------------------------ */
    char *rm = (char *)calloc((size_t)(nv ? nv : 1) + 1, 1);   /* rm[id], 1-based */
    for (int32_t i = 0; i < nv; i++) ncellv[i] = 0;
    for (int64_t e = 0; e < next; e++) {
        const int32_t m = marca[e];
        if (m > 0 && uvoid[m - 1] == -1) ncellv[m - 1]++;
    }
    /* removal of main voids, the WHERE rewrites of avism.f90:1816-1826 */
#define APPLY_REMOVALS()                                                              \
    do {                                                                              \
        for (int64_t e = 0; e < next; e++) if (marca[e] > 0 && rm[marca[e]]) marca[e] = 0; \
        for (int32_t i = 0; i < nv; i++) if (uvoid[i] > 0 && rm[uvoid[i]]) uvoid[i] = 0;  \
        for (int32_t i = 1; i <= nv; i++) if (rm[i]) { uvoid[i - 1] = 0; volnew[i - 1] = 0.0f; ncellv[i - 1] = 0; rm[i] = 0; } \
    } while (0)
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        if (ncellv[ind - 1] < 10) rm[ind] = 1;                       /* NCELL_MIN */
    }
    APPLY_REMOVALS();

    /* VOID_SHAPE (src/shape.f90:140-225): inertia in K,J,I order, REAL*4 */
    float *inert = (float *)calloc((size_t)(nv ? nv : 1) * 9, sizeof(float));
    for (int k = low1; k <= low2; k++)
        for (int j = low1; j <= low2; j++)
            for (int i = low1; i <= low2; i++) {
                const int32_t m = marca[pid(&G, i, j, k)];
                if (m <= 0) continue;
                float rk[3];
                rk[0] = RAD(i) - gxc[m - 1];
                rk[1] = RAD(j) - gyc[m - 1];
                rk[2] = RAD(k) - gzc[m - 1];
                const float rr = sqrtf((rk[0] * rk[0] + rk[1] * rk[1]) + rk[2] * rk[2]);
                float *I3 = inert + (size_t)(m - 1) * 9;
                for (int i2 = 0; i2 < 3; i2++)
                    for (int i1 = 0; i1 < 3; i1++) {
                        const float delta = (i1 == i2) ? 1.0f : 0.0f;
                        /* INERTIA + DELTA*RR*RR - RK(I1)*RK(I2), left to right */
                        I3[i1 + 3 * i2] = (I3[i1 + 3 * i2] + (delta * rr) * rr) - rk[i1] * rk[i2];
                    }
            }
    for (int32_t i = 0; i < nv; i++) { out->eps[i] = 0.0f; out->ip[i] = 0.0f; }
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] != -1) continue;
        float a[3][3], ev[3] = {0.0f, 0.0f, 0.0f}, axis[3];
        const float *I3 = inert + (size_t)(ind - 1) * 9;
        for (int i2 = 0; i2 < 3; i2++)
            for (int i1 = 0; i1 < 3; i1++) a[i1][i2] = I3[i1 + 3 * i2] / (float)ncellv[ind - 1];
        jacobi3(a, ev);
        axis[0] = sqrtf(2.5f * fabsf((ev[1] + ev[2]) - ev[0]));
        axis[1] = sqrtf(2.5f * fabsf((ev[2] + ev[0]) - ev[1]));
        axis[2] = sqrtf(2.5f * fabsf((ev[0] + ev[1]) - ev[2]));
        sort_desc3(axis);
        const float aa = axis[0], bb = axis[1], cc = axis[2];
        float eps = 1.0f - cc / aa;
        const float volm = (((float)ncellv[ind - 1] * dx) * dx) * dx;
        const float vell = (float)(((((double)(4.0f / 3.0f) * pi) * (double)aa) * (double)bb) * (double)cc);
        float ip = volm / vell;
        if (ip > 1.0f) { ip = -99.0f; eps = -99.0f; }
        out->eps[ind - 1] = eps;
        out->ip[ind - 1] = ip;
    }
    free(inert);

    const float cellv = (dx * dx) * dx;
    const double vmin = ((double)(4.0f / 3.0f) * pi) * (double)((p->rmin * p->rmin) * p->rmin);
    for (int32_t i = 0; i < nv; i++) volnew[i] = 0.0f;
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        volnew[ind - 1] = (float)((double)ncellv[ind - 1] * (double)cellv);
    }
    for (int32_t I = 0; I < nv; I++) {                                 /* RMIN */
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        if ((double)volnew[ind - 1] < vmin) rm[ind] = 1;
    }
    APPLY_REMOVALS();
    for (int32_t i = 0; i < nv; i++) { out->xc[i] = 0.0f; out->yc[i] = 0.0f; out->zc[i] = 0.0f; }
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        out->xc[ind - 1] = RAD(1) + (float)(cb->icx[ind - 1] - 1) * dx;
        out->yc[ind - 1] = RAD(1) + (float)(cb->icy[ind - 1] - 1) * dx;
        out->zc[ind - 1] = RAD(1) + (float)(cb->icz[ind - 1] - 1) * dx;
    }

    /* SIMPLE_CONNECTION_FAST: BFS of non-void cells from the LOW1 corner */
    {
        uint8_t *aux = (uint8_t *)malloc((size_t)next);
        int64_t *queue = (int64_t *)malloc((size_t)next * sizeof(int64_t));
        for (int64_t e = 0; e < next; e++) aux[e] = marca[e] > 0 ? 1 : 0;
        int64_t head = 0, tail = 0;
        queue[tail++] = 0;
        aux[0] = 2;
        const int64_t sy = ne, sz = (int64_t)ne * ne;
        while (head < tail) {
            const int64_t e = queue[head++];
            const int ix = (int)(e % ne), jy = (int)((e / ne) % ne), kz = (int)(e / sz);
            const int64_t nb[6] = {e - 1, e + 1, e - sy, e + sy, e - sz, e + sz};
            const int ok[6] = {ix > 0, ix < ne - 1, jy > 0, jy < ne - 1, kz > 0, kz < ne - 1};
            for (int d = 0; d < 6; d++)
                if (ok[d] && aux[nb[d]] == 0) { aux[nb[d]] = 2; queue[tail++] = nb[d]; }
        }
        for (int64_t e = 0; e < next; e++) {
            if (aux[e] > 0) continue;
            int64_t f = e;
            const int64_t rowend = e - (e % ne) + ne;
            while (f < rowend && aux[f] == 0) f++;
            marca[e] = f < rowend ? marca[f] : 0;   /* a hole never reaches LOW2 */
        }
        free(aux); free(queue);
    }

    /* VOID_PERIODIC */
    if (p->periodic) {
        char *inner = (char *)calloc((size_t)nv + 1, 1);
        for (int k = 1; k <= nx; k++)
            for (int j = 1; j <= nx; j++)
                for (int i = 1; i <= nx; i++) {
                    const int32_t m = marca[pid(&G, i, j, k)];
                    if (m > 0) inner[m] = 1;
                }
        int32_t *kept = (int32_t *)malloc((size_t)(nv ? nv : 1) * sizeof(int32_t));
        int32_t nkept = 0;
        for (int32_t I = 0; I < nv; I++) {
            const int32_t ind = indice[I];
            if (uvoid[ind - 1] >= 0) continue;
            if (!inner[ind]) rm[ind] = 1; else kept[nkept++] = ind;
        }
        APPLY_REMOVALS();
        free(inner);
        cell_vec *cells = (cell_vec *)calloc((size_t)nv + 1, sizeof(cell_vec));
        for (int64_t e = 0; e < next; e++) if (marca[e] > 0) cv_push(&cells[marca[e]], e);
        const float half = p->lado0 / 2.0f;
        for (int32_t J = 0; J < nkept; J++) {
            const int32_t ind = kept[J];
            const float xc1 = gxc[ind - 1], yc1 = gyc[ind - 1], zc1 = gzc[ind - 1];
            int sx = 0, sy = 0, sz = 0;
            if (xc1 < -half) sx = +1; if (xc1 > half) sx = -1;
            if (yc1 < -half) sy = +1; if (yc1 > half) sy = -1;
            if (zc1 < -half) sz = +1; if (zc1 > half) sz = -1;
            if (sx == 0 && sy == 0 && sz == 0) continue;
            const int igx = (int)((gxc[ind - 1] - RAD(1)) / dx) + 1;
            const int igy = (int)((gyc[ind - 1] - RAD(1)) / dx) + 1;
            const int igz = (int)((gzc[ind - 1] - RAD(1)) / dx) + 1;
            const int cx = igx + sx * nx, cy = igy + sy * nx, cz = igz + sz * nx;
            if (cx < low1 || cx > low2 || cy < low1 || cy > low2 || cz < low1 || cz > low2) continue;
            const int32_t ind2 = marca[pid(&G, cx, cy, cz)];
            if (ind2 == 0) continue;
            int64_t counter = 0, counter2 = 0;
            const cell_vec *cv = &cells[ind];
            for (int64_t q = 0; q < cv->n; q++) {
                const int64_t e = cv->c[q];
                const int ix = (int)(e % ne) + low1 + sx * nx;
                const int jy = (int)((e / ne) % ne) + low1 + sy * nx;
                const int kz = (int)(e / ((int64_t)ne * ne)) + low1 + sz * nx;
                if (ix >= low1 && ix <= low2 && jy >= low1 && jy <= low2 && kz >= low1 && kz <= low2) {
                    counter2++;
                    if (marca[pid(&G, ix, jy, kz)] == ind2) counter++;
                }
            }
            const float intersec = counter2 == 0 ? 0.0f : (float)counter / (float)counter2;
            if (intersec > 0.4f) {                                   /* CHANGE_BELONG */
                uvoid[ind - 1] = ind2;
                for (int32_t i = 0; i < nv; i++) if (uvoid[i] == ind) uvoid[i] = ind2;
                if (ind2 != ind) {
                    cell_vec *src = &cells[ind], *dst = &cells[ind2];
                    for (int64_t q = 0; q < src->n; q++) { marca[src->c[q]] = ind2; cv_push(dst, src->c[q]); }
                    src->n = 0;
                }
                volnew[ind - 1] = 0.0f;
            }
        }
        for (int32_t i = 0; i <= nv; i++) free(cells[i].c);
        free(cells); free(kept);
    }

    /* global properties on inner cells (avism.f90:1917-1970) */
    float *umean = out->umean, *mtot = out->mtot;
    for (int32_t i = 0; i < nv; i++) { ncellv[i] = 0; umean[i] = 0.0f; mtot[i] = 0.0f; }
    double volt = 0.0;
    const float rete3 = (g.rete * g.rete) * g.rete;
    for (int k = 1; k <= nx; k++)
        for (int j = 1; j <= nx; j++)
            for (int i = 1; i <= nx; i++) {
                const int64_t e = pid(&G, i, j, k);
                const int32_t m = marca[e];
                if (m <= 0 || uvoid[m - 1] != -1) continue;
                const float u = u1co_ext[e];
                ncellv[m - 1]++;
                umean[m - 1] = umean[m - 1] + u;
                mtot[m - 1] = mtot[m - 1] + ((((u * meandens) * dx) * dx) * dx) * rete3;
                volt = volt + (double)cellv;
            }
    for (int32_t i = 0; i < nv; i++) if (ncellv[i] > 0) umean[i] = umean[i] / (float)ncellv[i];
    for (int32_t i = 0; i < nv; i++) volnew[i] = 0.0f;
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        volnew[ind - 1] = (float)((double)ncellv[ind - 1] * (double)cellv);
    }
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        if ((double)volnew[ind - 1] < vmin) rm[ind] = 1;
    }
    APPLY_REMOVALS();
    int32_t nvoidt = 0;
    for (int32_t i = 0; i < nv; i++) {
        out->req[i] = 0.0f;
        if (uvoid[i] == -1) {
            nvoidt++;
            /* ((3.*VOLM)/(4.*PI))**(1./3.), src/avism.f90:2071: VOLM is REAL*8
               (src/avism.f90:73), so 3.*VOLM is a REAL*8 product */
            out->req[i] = (float)pow((3.0 * (double)volnew[i]) / (4.0 * pi), (double)(1.0f / 3.0f));
        }
    }
    out->nvoidt = nvoidt;
    out->volt_clean = volt;
    free(rm);
    if (!out->marca) free(G.marca);
    free(radx);
#undef RAD
    return AVISM_OK;
}

int orc_run_level(const avism_params *p, int64_t n, const float *x, const float *y,
                  const float *z, const float *vx, const float *vy, const float *vz,
                  const float *m, avism_cubes *cubes, int32_t *nvoid, avism_voids *voids,
                  float *meandens, float *u1co_ext, float *diverco_ext)
{
    avism_grid g;
    int st = orc_grid_setup(p, &g, NULL);
    if (st) return st;
    const int64_t nc = (int64_t)g.nx * g.nx * g.nx;
    float *um = (float *)malloc((size_t)nc * sizeof(float) * 4);
    if (!um) return AVISM_ERR_OOM;
    st = orc_particles_to_grid(p, n, x, y, z, vx, vy, vz, m, NULL, um, um + nc, um + 2 * nc,
                               um + 3 * nc, NULL, NULL);
    if (!st) st = orc_fields(p, um, um + nc, um + 2 * nc, um + 3 * nc, u1co_ext, diverco_ext, meandens);
    free(um);
    if (!st) st = orc_voidfind(p, u1co_ext, diverco_ext, NULL, NULL, NULL, cubes, nvoid, NULL, NULL, NULL);
    if (!st) st = orc_merge_post(p, *nvoid, cubes, u1co_ext, *meandens, voids);
    return st;
}
