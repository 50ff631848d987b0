/*
 * orc_kdtree.c -- oracle: k-d tree kNN and ball search (test infrastructure).
 *
 * Restates the search semantics of src/kdtree.f90 (module cosmokdtree):
 *   - squared distance as in distance() src/kdtree.f90:1441-1465: per axis
 *     dx = p - q, periodic dx = min(|dx|, L-|dx|), d2 = ((0+dx^2)+dy^2)+dz^2;
 *   - knn_search (504-540) returns the k smallest squared distances, ascending,
 *     then sqrt; ball_search (1015-1070) returns all points with d2 <= r*r;
 *   - ties: the reference orders equal distances by its traversal and an
 *     unstable quicksort (1553-1643); the oracle orders by (d2, point index).
 * The tree itself (median split on the widest axis, leaves of <= 16 points) is
 * only an accelerator: results are defined by the rule above.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "avism_oracle.h"

typedef struct {
    float lo[3], hi[3];
    int64_t start, end;
    int32_t left, right;
} kd_node;

struct orc_kdtree {
    int64_t n;
    float box_l;
    int periodic;
    float *p[3];      /* points in tree order */
    int64_t *pidx;    /* original index of each tree-order point */
    kd_node *nodes;
    int32_t nnodes, cap;
};

static inline float orc_d2(float px, float py, float pz, float qx, float qy, float qz,
                           float L, int periodic)
{
    float dx = px - qx, dy = py - qy, dz = pz - qz;
    if (periodic) {
        float a = fabsf(dx); dx = fminf(a, L - a);
        a = fabsf(dy); dy = fminf(a, L - a);
        a = fabsf(dz); dz = fminf(a, L - a);
    }
    float d = dx * dx;
    d = d + dy * dy;
    d = d + dz * dz;
    return d;
}

/* lower bound of the distance from q to [lo,hi] on one axis (minimum image) */
static inline float axis_gap(float q, float lo, float hi, float L, int periodic)
{
    float d = 0.0f;
    if (q < lo) d = lo - q; else if (q > hi) d = q - hi;
    if (periodic && d > 0.0f) {
        float q2 = q + L, d2 = 0.0f;
        if (q2 < lo) d2 = lo - q2; else if (q2 > hi) d2 = q2 - hi;
        if (d2 < d) d = d2;
        q2 = q - L; d2 = 0.0f;
        if (q2 < lo) d2 = lo - q2; else if (q2 > hi) d2 = q2 - hi;
        if (d2 < d) d = d2;
    }
    return d;
}

static float box_d2(const kd_node *nd, float qx, float qy, float qz, float L, int periodic)
{
    const float gx = axis_gap(qx, nd->lo[0], nd->hi[0], L, periodic);
    const float gy = axis_gap(qy, nd->lo[1], nd->hi[1], L, periodic);
    const float gz = axis_gap(qz, nd->lo[2], nd->hi[2], L, periodic);
    /* shrink slightly: the bound must never exceed a true point distance */
    return ((gx * gx + gy * gy) + gz * gz) * (1.0f - 1e-5f);
}

static void swap_pt(orc_kdtree *t, int64_t a, int64_t b)
{
    for (int d = 0; d < 3; d++) { float v = t->p[d][a]; t->p[d][a] = t->p[d][b]; t->p[d][b] = v; }
    int64_t v = t->pidx[a]; t->pidx[a] = t->pidx[b]; t->pidx[b] = v;
}

/* quickselect: place the k-th smallest (by axis value, then index) at position k */
static void select_kth(orc_kdtree *t, int axis, int64_t lo, int64_t hi, int64_t k)
{
    float *v = t->p[axis];
    while (hi > lo) {
        const int64_t mid = lo + (hi - lo) / 2;
        swap_pt(t, mid, hi);
        const float pv = v[hi];
        const int64_t pi = t->pidx[hi];
        int64_t s = lo;
        for (int64_t i = lo; i < hi; i++) {
            if (v[i] < pv || (v[i] == pv && t->pidx[i] < pi)) { swap_pt(t, i, s); s++; }
        }
        swap_pt(t, s, hi);
        if (s == k) return;
        if (s < k) lo = s + 1; else hi = s - 1;
    }
}

static int32_t build_rec(orc_kdtree *t, int64_t start, int64_t end)
{
    if (t->nnodes == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->nodes = (kd_node *)realloc(t->nodes, (size_t)t->cap * sizeof(kd_node));
    }
    const int32_t id = t->nnodes++;
    kd_node nd;
    nd.start = start; nd.end = end; nd.left = nd.right = -1;
    for (int d = 0; d < 3; d++) { nd.lo[d] = INFINITY; nd.hi[d] = -INFINITY; }
    for (int64_t i = start; i < end; i++)
        for (int d = 0; d < 3; d++) {
            const float v = t->p[d][i];
            if (v < nd.lo[d]) nd.lo[d] = v;
            if (v > nd.hi[d]) nd.hi[d] = v;
        }
    if (end - start > 16) {
        int axis = 0;
        float ext = nd.hi[0] - nd.lo[0];
        for (int d = 1; d < 3; d++) if (nd.hi[d] - nd.lo[d] > ext) { ext = nd.hi[d] - nd.lo[d]; axis = d; }
        const int64_t mid = start + (end - start) / 2;
        select_kth(t, axis, start, end - 1, mid);
        const int32_t l = build_rec(t, start, mid);
        const int32_t r = build_rec(t, mid, end);
        nd.left = l; nd.right = r;
    }
    t->nodes[id] = nd;
    return id;
}

orc_kdtree *orc_kd_build(int64_t n, const float *x, const float *y, const float *z, float box_l)
{
    orc_kdtree *t = (orc_kdtree *)calloc(1, sizeof(orc_kdtree));
    t->n = n; t->box_l = box_l; t->periodic = box_l > 0.0f;
    for (int d = 0; d < 3; d++) t->p[d] = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    t->pidx = (int64_t *)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
    memcpy(t->p[0], x, (size_t)n * sizeof(float));
    memcpy(t->p[1], y, (size_t)n * sizeof(float));
    memcpy(t->p[2], z, (size_t)n * sizeof(float));
    for (int64_t i = 0; i < n; i++) t->pidx[i] = i;
    if (n > 0) build_rec(t, 0, n);
    return t;
}

void orc_kd_free(orc_kdtree *t)
{
    if (!t) return;
    for (int d = 0; d < 3; d++) free(t->p[d]);
    free(t->pidx); free(t->nodes); free(t);
}

/* ---- kNN with a bounded max-heap keyed by (d2, idx) ---------------------- */
typedef struct { float d2; int64_t idx; } kd_item;

static inline int item_less(kd_item a, kd_item b)
{
    return a.d2 < b.d2 || (a.d2 == b.d2 && a.idx < b.idx);
}

static void heap_push(kd_item *h, int *cnt, int k, kd_item it)
{
    if (*cnt < k) {
        int i = (*cnt)++;
        h[i] = it;
        while (i > 0) {
            int pa = (i - 1) / 2;
            if (item_less(h[pa], h[i])) { kd_item tmp = h[pa]; h[pa] = h[i]; h[i] = tmp; i = pa; }
            else break;
        }
    } else if (item_less(it, h[0])) {
        h[0] = it;
        int i = 0;
        for (;;) {
            int l = 2 * i + 1, r = l + 1, m = i;
            if (l < k && item_less(h[m], h[l])) m = l;
            if (r < k && item_less(h[m], h[r])) m = r;
            if (m == i) break;
            kd_item tmp = h[m]; h[m] = h[i]; h[i] = tmp; i = m;
        }
    }
}

static void knn_rec(const orc_kdtree *t, int32_t id, float qx, float qy, float qz, int k,
                    kd_item *h, int *cnt)
{
    const kd_node *nd = &t->nodes[id];
    if (*cnt == k && box_d2(nd, qx, qy, qz, t->box_l, t->periodic) > h[0].d2) return;
    if (nd->left < 0) {
        for (int64_t i = nd->start; i < nd->end; i++) {
            kd_item it;
            it.d2 = orc_d2(t->p[0][i], t->p[1][i], t->p[2][i], qx, qy, qz, t->box_l, t->periodic);
            it.idx = t->pidx[i];
            heap_push(h, cnt, k, it);
        }
        return;
    }
    const float dl = box_d2(&t->nodes[nd->left], qx, qy, qz, t->box_l, t->periodic);
    const float dr = box_d2(&t->nodes[nd->right], qx, qy, qz, t->box_l, t->periodic);
    if (dl <= dr) {
        knn_rec(t, nd->left, qx, qy, qz, k, h, cnt);
        knn_rec(t, nd->right, qx, qy, qz, k, h, cnt);
    } else {
        knn_rec(t, nd->right, qx, qy, qz, k, h, cnt);
        knn_rec(t, nd->left, qx, qy, qz, k, h, cnt);
    }
}

static int cmp_item(const void *a, const void *b)
{
    const kd_item *x = (const kd_item *)a, *y = (const kd_item *)b;
    if (item_less(*x, *y)) return -1;
    if (item_less(*y, *x)) return 1;
    return 0;
}

void orc_kd_knn(const orc_kdtree *t, float qx, float qy, float qz, int k, int64_t *idx, float *d2)
{
    kd_item stackbuf[256];
    kd_item *h = k <= 256 ? stackbuf : (kd_item *)malloc((size_t)k * sizeof(kd_item));
    int cnt = 0;
    if (t->n > 0) knn_rec(t, 0, qx, qy, qz, k, h, &cnt);
    qsort(h, (size_t)cnt, sizeof(kd_item), cmp_item);
    for (int i = 0; i < k; i++) {
        if (i < cnt) { idx[i] = h[i].idx; d2[i] = h[i].d2; }
        else { idx[i] = -1; d2[i] = HUGE_VALF; }   /* dist = HUGE(0.0), idx = -1 */
    }
    if (h != stackbuf) free(h);
}

/* ---- ball search -------------------------------------------------------- */
typedef struct { kd_item *it; int64_t n, cap; } item_vec;

static void ball_rec(const orc_kdtree *t, int32_t id, float qx, float qy, float qz, float r2,
                     item_vec *v)
{
    const kd_node *nd = &t->nodes[id];
    if (box_d2(nd, qx, qy, qz, t->box_l, t->periodic) > r2) return;
    if (nd->left < 0) {
        for (int64_t i = nd->start; i < nd->end; i++) {
            const float d = orc_d2(t->p[0][i], t->p[1][i], t->p[2][i], qx, qy, qz, t->box_l, t->periodic);
            if (d <= r2) {
                if (v->n == v->cap) {
                    v->cap = v->cap ? 2 * v->cap : 128;
                    v->it = (kd_item *)realloc(v->it, (size_t)v->cap * sizeof(kd_item));
                }
                v->it[v->n].d2 = d; v->it[v->n].idx = t->pidx[i]; v->n++;
            }
        }
        return;
    }
    ball_rec(t, nd->left, qx, qy, qz, r2, v);
    ball_rec(t, nd->right, qx, qy, qz, r2, v);
}

int64_t orc_kd_ball(const orc_kdtree *t, float qx, float qy, float qz, float r,
                    int64_t **idx, float **d2, int64_t *cap)
{
    item_vec v = {0, 0, 0};
    const float r2 = r * r;                          /* radius**2 in REAL*4 */
    if (t->n > 0) ball_rec(t, 0, qx, qy, qz, r2, &v);
    qsort(v.it, (size_t)v.n, sizeof(kd_item), cmp_item);
    if (v.n > *cap) {
        *cap = v.n + 64;
        *idx = (int64_t *)realloc(*idx, (size_t)*cap * sizeof(int64_t));
        *d2 = (float *)realloc(*d2, (size_t)*cap * sizeof(float));
    }
    for (int64_t i = 0; i < v.n; i++) { (*idx)[i] = v.it[i].idx; (*d2)[i] = v.it[i].d2; }
    free(v.it);
    return v.n;
}

int orc_knn(int64_t n, const float *x, const float *y, const float *z, float box_l,
            int64_t nq, const float *qx, const float *qy, const float *qz, int k,
            int64_t *idx, float *dist)
{
    if (k <= 0 || n < 0 || nq < 0) return AVISM_ERR_ARG;
    orc_kdtree *t = orc_kd_build(n, x, y, z, box_l);
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t q = 0; q < nq; q++) {
        float d2[1024];
        int64_t *ix = idx + q * k;
        orc_kd_knn(t, qx[q], qy[q], qz[q], k, ix, d2);
        for (int i = 0; i < k; i++) {
            dist[q * k + i] = sqrtf(d2[i]);
            ix[i] = ix[i] >= 0 ? ix[i] + 1 : -1;
        }
    }
    orc_kd_free(t);
    return AVISM_OK;
}
