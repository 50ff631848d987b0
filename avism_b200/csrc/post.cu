// post.cu -- volume ordering, MERGE_VOID painting and the post-processing of
// src/avism.f90:1738-1973 on the device.
//
//  * INDEXX on VOL (exact permutation), MERGE_VOID on cube records (merge.cpp);
//  * MARCA painting: every cell takes the owner of the earliest-painted cube
//    containing it (atomicMin of the paint time), which is the reference's
//    first-writer-wins "IF(MARCA.EQ.0) MARCA=IND0";
//  * NCELLV, the NCELL_MIN / RMIN removals (decided per void on the host,
//    applied by one relabel pass instead of a WHERE per void);
//  * VOID_SHAPE inertia sums in the reference's serial REAL*4 order per void,
//    JACOBI / SORT per main void on the device (src/shape.f90);
//  * SIMPLE_CONNECTION_FAST as union-find connected components of the non-void
//    cells (shared-memory tiles, then the tile faces): everything not connected
//    to the LOW1 corner is a hole, filled with the id of the first void cell in +x;
//  * VOID_PERIODIC: overlap counts of every outer-centred void computed in one
//    pass, then validated in catalogue order on the host; a void whose inputs
//    an earlier merge could have changed is recounted on the device;
//  * global properties UMEAN and MTOT on the inner cells, REAL*4 sums in the
//    reference's serial order per void.
#include <cub/cub.cuh>
#include <algorithm>
#include <array>
#include <climits>
#include <functional>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "merge.h"

namespace avism {

struct PostGrid {
    int low1, low2, ne, nx;
};

__device__ __forceinline__ int64_t pidx(const PostGrid &G, int i, int j, int k) {
    return (int64_t)(i - G.low1) + (int64_t)G.ne * ((int64_t)(j - G.low1) + (int64_t)G.ne * (k - G.low1));
}

// cube boxes: 6 int arrays of cap entries (x0,x1,y0,y1,z0,z1)
__global__ void k_paint_time(PostGrid G, const int32_t *box, int32_t cap, const int32_t *ptime, int32_t nv,
                             int32_t *tgrid) {
    const int lane = threadIdx.x & 31;
    const int64_t wi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wi >= nv) return;
    const int32_t x0 = box[0 * cap + wi], x1 = box[1 * cap + wi], y0 = box[2 * cap + wi];
    const int32_t y1 = box[3 * cap + wi], z0 = box[4 * cap + wi], z1 = box[5 * cap + wi];
    const int sx = x1 - x0 + 1, sy = y1 - y0 + 1, sz = z1 - z0 + 1;
    const int64_t vol = (int64_t)sx * sy * sz;
    const int32_t t = ptime[wi];
    for (int64_t q = lane; q < vol; q += 32) {
        const int a = (int)(q % sx), b = (int)((q / sx) % sy), d = (int)(q / ((int64_t)sx * sy));
        atomicMin(&tgrid[pidx(G, x0 + a, y0 + b, z0 + d)], t);
    }
}

__global__ void k_fill_i32(int64_t n, int32_t *a, int32_t v) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] = v;
}

__global__ void k_time_to_label(int64_t ne3, const int32_t *tgrid, const int32_t *owner_by_time, int32_t *marca) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne3) return;
    const int32_t t = tgrid[e];
    marca[e] = t == INT_MAX ? 0 : owner_by_time[t];
}

// MARCA = map[MARCA] for the void cells, four cells per thread (16-byte loads:
// MARCA is the context's own B_MARCA buffer, 256-byte aligned by cudaMalloc),
// stores only where a label changes
__global__ void k_relabel(int64_t ne3, int32_t *marca, const int32_t *map) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t e = q * 4;
    if (e >= ne3) return;
    if (e + 4 <= ne3) {
        int4 v = *reinterpret_cast<const int4 *>(marca + e);
        const int4 o = v;
        if (v.x > 0) v.x = map[v.x];
        if (v.y > 0) v.y = map[v.y];
        if (v.z > 0) v.z = map[v.z];
        if (v.w > 0) v.w = map[v.w];
        if (v.x != o.x || v.y != o.y || v.z != o.z || v.w != o.w) *reinterpret_cast<int4 *>(marca + e) = v;
        return;
    }
    for (int64_t f = e; f < ne3; f++) {
        const int32_t m = marca[f];
        if (m > 0 && map[m] != m) marca[f] = map[m];
    }
}

// warp-aggregated count per main-void label (uvoid == -1) over the ext grid
__global__ void k_ncellv(int64_t ne3, const int32_t *marca, const int32_t *uvoid, int32_t *ncell) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int32_t m = 0;
    if (e < ne3) {
        m = marca[e];
        if (m > 0 && uvoid[m - 1] != -1) m = 0;
    }
    const unsigned grp = __match_any_sync(0xffffffffu, m);
    const int lane = threadIdx.x & 31;
    if (m > 0 && lane == __ffs(grp) - 1) atomicAdd(&ncell[m - 1], __popc(grp));
}

// ---- per-void REAL*4 sums in the reference's serial K, J, I order -------------
// VOID_SHAPE's inertia (src/shape.f90:158-182) and the global properties UMEAN and
// MTOT (src/avism.f90:1917-1936) are REAL*4 accumulations over a void's cells in
// the order of the reference's serial triple loop, so their bits depend on that
// order.  The cells of every void are listed in increasing linear index (the
// K, J, I order: a stable sort by label of the void cells taken in grid order),
// then one warp per void walks its list 32 cells at a time: all lanes compute
// the cells' terms into shared memory, then one lane per accumulator adds them
// in order.  The chains stay serial, as the reference's; voids run in parallel.

// void cells of the ext grid (VOID_SHAPE: every cell LOW1..LOW2 with MARCA > 0)
struct ExtVoidCell {
    const int32_t *marca;
    __host__ __device__ bool operator()(int32_t e) const { return marca[e] > 0; }
};
// inner cells of main voids (the global properties' loop, 1..NX)
struct InnerMainCell {
    PostGrid G;
    const int32_t *marca, *uvoid;
    __device__ bool operator()(int32_t c) const {
        const int nx = G.nx;
        const int i = c % nx + 1, j = (c / nx) % nx + 1, k = c / (nx * nx) + 1;
        const int32_t m = marca[pidx(G, i, j, k)];
        return m > 0 && uvoid[m - 1] == -1;
    }
};

__global__ void k_cell_labels(int32_t n, const int32_t *__restrict__ cell, const int32_t *__restrict__ marca,
                              PostGrid G, int inner, int32_t *__restrict__ key, int32_t *__restrict__ cnt) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int32_t c = cell[t];
    int32_t m;
    if (inner) {
        const int nx = G.nx;
        m = marca[pidx(G, c % nx + 1, (c / nx) % nx + 1, c / (nx * nx) + 1)];
    } else {
        m = marca[c];
    }
    key[t] = m;
    atomicAdd(&cnt[m - 1], 1);
}

constexpr int SEQ_WARPS = 4;

// VOID_SHAPE: INERTIA(I1,I2) = INERTIA(I1,I2) + DELTA*RR*RR - RK(I1)*RK(I2), evaluated
// left to right, per cell in order; off-diagonal DELTA*RR*RR is +0, and adding +0
// leaves the (never -0) sum unchanged, so those chains subtract only.  Output:
// 6 sums per label (I11, I22, I33, I12, I13, I23).
__global__ void __launch_bounds__(SEQ_WARPS * 32)
k_inertia_seq(int32_t nv, const int64_t *__restrict__ off, const int32_t *__restrict__ cell, PostGrid G,
              const float *__restrict__ rad, int rad_lo, const float *__restrict__ gxc, const float *__restrict__ gyc,
              const float *__restrict__ gzc, float *__restrict__ inert) {
    __shared__ float term[SEQ_WARPS][7][33];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t v = blockIdx.x * SEQ_WARPS + w;
    if (v >= nv) return;
    const int64_t a = off[v], b = off[v + 1];
    const float cx = gxc[v], cy = gyc[v], cz = gzc[v];
    float acc = 0.0f;                                   // lane q < 6 owns accumulator q
    float (*T)[33] = term[w];
    for (int64_t base = a; base < b; base += 32) {
        const int n = (int)(b - base < 32 ? b - base : 32);
        if (lane < n) {
            const int32_t e = cell[base + lane];
            const int i = e % G.ne + G.low1, j = (e / G.ne) % G.ne + G.low1, k = e / (G.ne * G.ne) + G.low1;
            const float r0 = __fsub_rn(rad[i - rad_lo], cx);
            const float r1 = __fsub_rn(rad[j - rad_lo], cy);
            const float r2 = __fsub_rn(rad[k - rad_lo], cz);
            const float rr = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(r0, r0), __fmul_rn(r1, r1)), __fmul_rn(r2, r2)));
            T[0][lane] = __fmul_rn(__fmul_rn(1.0f, rr), rr);
            T[1][lane] = __fmul_rn(r0, r0);
            T[2][lane] = __fmul_rn(r1, r1);
            T[3][lane] = __fmul_rn(r2, r2);
            T[4][lane] = __fmul_rn(r0, r1);
            T[5][lane] = __fmul_rn(r0, r2);
            T[6][lane] = __fmul_rn(r1, r2);
        }
        __syncwarp();
        if (lane < 3) {
            for (int t = 0; t < n; t++) acc = __fsub_rn(__fadd_rn(acc, T[0][t]), T[1 + lane][t]);
        } else if (lane < 6) {
            for (int t = 0; t < n; t++) acc = __fsub_rn(acc, T[1 + lane][t]);
        }
        __syncwarp();
    }
    if (lane < 6) inert[(size_t)v * 6 + lane] = acc;
}

// global properties: UMEAN(IND) = UMEAN(IND) + U1CO and MTOT(IND) = MTOT(IND) +
// U1CO*MEANDENS*DXX*DYY*DZZ*RETE**3 per inner cell in order; 2 sums per label
__global__ void __launch_bounds__(SEQ_WARPS * 32)
k_props_seq(int32_t nv, const int64_t *__restrict__ off, const int32_t *__restrict__ cell,
            const float *__restrict__ u1co, float meandens, float dx, float rete3, float *__restrict__ sums) {
    __shared__ float term[SEQ_WARPS][2][33];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t v = blockIdx.x * SEQ_WARPS + w;
    if (v >= nv) return;
    const int64_t a = off[v], b = off[v + 1];
    float acc = 0.0f;
    float (*T)[33] = term[w];
    for (int64_t base = a; base < b; base += 32) {
        const int n = (int)(b - base < 32 ? b - base : 32);
        if (lane < n) {
            const float u = u1co[cell[base + lane]];
            T[0][lane] = u;
            T[1][lane] = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(u, meandens), dx), dx), dx), rete3);
        }
        __syncwarp();
        if (lane < 2)
            for (int t = 0; t < n; t++) acc = __fadd_rn(acc, T[lane][t]);
        __syncwarp();
    }
    if (lane < 2) sums[(size_t)v * 2 + lane] = acc;
}

// the cells passing `pick` among 0..ncells-1, grouped by their label (1..nv)
// in increasing cell index; off[v]..off[v+1] are label v+1's
template <class Pick>
static void void_cell_lists(Ctx &c, int32_t ncells, Pick pick, const int32_t *marca, PostGrid G, int inner,
                            int32_t nv, const int32_t **cell_out, const int64_t **off_out, int32_t *cnt_host) {
    const int32_t nvs = std::max(nv, 1);
    int32_t *cell = c.get_t<int32_t>(B_LL_CELL, (size_t)std::max(ncells, 1));
    int32_t *nsel_d = c.get_t<int32_t>(B_SCAL, 4);
    cub::CountingInputIterator<int32_t> it(0);
    size_t tmp = 0;
    AV_CUDA(cub::DeviceSelect::If(nullptr, tmp, it, cell, nsel_d, ncells, pick, c.stream));
    AV_CUDA(cub::DeviceSelect::If(c.get(B_CUB_TMP, tmp), tmp, it, cell, nsel_d, ncells, pick, c.stream));
    int32_t nsel = 0;
    AV_CUDA(cudaMemcpyAsync(&nsel, nsel_d, sizeof nsel, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const int32_t m1 = std::max(nsel, 1);
    int32_t *key = c.get_t<int32_t>(B_LL_KEY, (size_t)m1);
    int32_t *key2 = c.get_t<int32_t>(B_LL_KEY2, (size_t)m1);
    int32_t *cell2 = c.get_t<int32_t>(B_LL_CELL2, (size_t)m1);
    int32_t *cnt = c.get_t<int32_t>(B_LL_CNT, (size_t)nvs + 1);
    int64_t *off = c.get_t<int64_t>(B_LL_OFF, (size_t)nvs + 1);
    AV_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)nvs + 1), c.stream));
    if (nsel > 0)
        ++c.launches, k_cell_labels<<<grid_for(nsel, 256), 256, 0, c.stream>>>(nsel, cell, marca, G, inner, key, cnt);
    AV_CUDA(cudaGetLastError());
    cub::DoubleBuffer<int32_t> dk(key, key2), dv(cell, cell2);
    int bits = 1;
    while ((1LL << bits) <= (int64_t)nv) bits++;
    tmp = 0;
    AV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, nsel, 0, bits, c.stream));
    AV_CUDA(cub::DeviceRadixSort::SortPairs(c.get(B_CUB_TMP, tmp), tmp, dk, dv, nsel, 0, bits, c.stream));
    tmp = 0;
    AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, off, nv + 1, c.stream));
    AV_CUDA(cub::DeviceScan::ExclusiveSum(c.get(B_CUB_TMP, tmp), tmp, cnt, off, nv + 1, c.stream));
    if (cnt_host) AV_CUDA(cudaMemcpyAsync(cnt_host, cnt, sizeof(int32_t) * (size_t)nv, cudaMemcpyDeviceToHost, c.stream));
    *cell_out = dv.Current();
    *off_out = off;
}

// ---- VOID_SHAPE axes: one thread per main void (src/shape.f90:198-232) -----
// JACOBI (src/shape.f90:46-134, Numerical Recipes) and SORT (src/shape.f90:2-29)
// in REAL*4 with the REAL*8 promotions of their literals.  The library is built
// with --fmad=false and IEEE division and square roots, so every operation
// rounds as the Fortran's does.
__device__ void jacobi3(float a[3][3], float d[3]) {
    const int n = 3;
    float b[3], z[3];
    for (int ip = 0; ip < n; ip++) { b[ip] = a[ip][ip]; d[ip] = b[ip]; z[ip] = 0.0f; }
    for (int it = 1; it <= 50; it++) {
        float sm = 0.0f;
        for (int ip = 0; ip < n - 1; ip++)
            for (int iq = ip + 1; iq < n; iq++) sm = sm + fabsf(a[ip][iq]);
        if (sm == 0.0f) return;
        const float tresh = it < 4 ? (float)(0.2 * (double)(sm * sm)) : 0.0f;
        for (int ip = 0; ip < n - 1; ip++)
            for (int iq = ip + 1; iq < n; iq++) {
                const float g = (float)(100.0 * (double)fabsf(a[ip][iq]));
                if (it > 4 && fabsf(d[ip]) + g == fabsf(d[ip]) && fabsf(d[iq]) + g == fabsf(d[iq])) {
                    a[ip][iq] = 0.0f;
                    continue;
                }
                if (!(fabsf(a[ip][iq]) > tresh)) continue;
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
        for (int ip = 0; ip < n; ip++) { b[ip] = b[ip] + z[ip]; d[ip] = b[ip]; z[ip] = 0.0f; }
    }
}

__device__ __forceinline__ void sort_desc3(float d[3]) {
    for (int i = 0; i < 2; i++) {
        int k = i;
        float p = d[i];
        for (int j = i + 1; j < 3; j++)
            if (d[j] >= p) { k = j; p = d[j]; }
        if (k != i) { d[k] = d[i]; d[i] = p; }
    }
}


__global__ void k_void_axes(int32_t nv, const int32_t *__restrict__ uvoid, const int32_t *__restrict__ ncellv,
                            const float *__restrict__ inert, float dx, double pi, float *__restrict__ eps,
                            float *__restrict__ ipv) {
    const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    float e = 0.0f, ip = 0.0f;
    if (uvoid[v] == -1) {
        const float *s = &inert[(size_t)v * 6];
        const float n = (float)ncellv[v];
        float a[3][3];
        a[0][0] = s[0] / n; a[1][1] = s[1] / n; a[2][2] = s[2] / n;
        a[0][1] = a[1][0] = s[3] / n;
        a[0][2] = a[2][0] = s[4] / n;
        a[1][2] = a[2][1] = s[5] / n;
        float ev[3] = {0.0f, 0.0f, 0.0f}, ax[3];
        jacobi3(a, ev);
        ax[0] = sqrtf(2.5f * fabsf((ev[1] + ev[2]) - ev[0]));
        ax[1] = sqrtf(2.5f * fabsf((ev[2] + ev[0]) - ev[1]));
        ax[2] = sqrtf(2.5f * fabsf((ev[0] + ev[1]) - ev[2]));
        sort_desc3(ax);
        e = 1.0f - ax[2] / ax[0];
        const float volm = (((float)ncellv[v] * dx) * dx) * dx;
        const float vell = (float)(((((double)(4.0f / 3.0f) * pi) * (double)ax[0]) * (double)ax[1]) * (double)ax[2]);
        ip = volm / vell;
        if (ip > 1.0f) { ip = -99.0f; e = -99.0f; }
    }
    eps[v] = e;
    ipv[v] = ip;
}

// ---- SIMPLE_CONNECTION_FAST: union-find of non-void cells --------------------
__device__ __forceinline__ int32_t uf_find(int32_t *P, int32_t x) {
    while (true) {
        const int32_t px = P[x];
        if (px == x) return x;
        const int32_t ppx = P[px];
        if (ppx != px) P[x] = ppx;
        x = px;
    }
}
__device__ __forceinline__ void uf_union(int32_t *P, int32_t a, int32_t b) {
    while (true) {
        a = uf_find(P, a);
        b = uf_find(P, b);
        if (a == b) return;
        if (a < b) { const int32_t t = a; a = b; b = t; }
        const int32_t old = atomicCAS(&P[a], a, b);
        if (old == a) return;
        a = old;
    }
}
// Union-find in shared memory over one CL_TX x CL_TY x CL_TZ tile of the
// non-void cells (MARCA <= 0), then every such cell points at its tile
// component's smallest cell (global index); k_ccl_faces joins components
// across the tiles' low faces.  Local and global indices are both (z, y,
// x)-lexicographic, so the local minimum is the global minimum and parents
// keep pointing to smaller indices.  A warp takes whole x-rows of 32 cells: the
// x-runs come from one ballot, and a cell joins the row below (y - 1, z - 1)
// only where its left neighbour's pair is not already joined, so a run
// overlapping another costs one union, not one per cell.
constexpr int CL_TX = 32, CL_TY = 8, CL_TZ = 8, CL_N = CL_TX * CL_TY * CL_TZ, CL_THREADS = 256;
constexpr int CL_ROWS = CL_TY * CL_TZ, CL_WARPS = CL_THREADS / 32;

__device__ __forceinline__ int32_t luf_find(int32_t *L, int32_t x) {
    volatile int32_t *V = L;
    while (true) {                                  // path halving, as uf_find
        const int32_t px = V[x];
        if (px == x) return x;
        const int32_t ppx = V[px];
        if (ppx != px) V[x] = ppx;
        x = px;
    }
}
__device__ __forceinline__ void luf_union(int32_t *L, int32_t a, int32_t b) {
    while (true) {
        a = luf_find(L, a);
        b = luf_find(L, b);
        if (a == b) return;
        if (a < b) { const int32_t t = a; a = b; b = t; }
        const int32_t old = atomicCAS(&L[a], a, b);
        if (old == a) return;
        a = old;
    }
}

__global__ void __launch_bounds__(CL_THREADS) k_ccl_local(PostGrid G, const int32_t *__restrict__ marca,
                                                          int32_t *__restrict__ P) {
    __shared__ int32_t L[CL_N];
    const int ne = G.ne;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntx = (ne + CL_TX - 1) / CL_TX, nty = (ne + CL_TY - 1) / CL_TY;
    const int bx = (int)(blockIdx.x % ntx), by = (int)((blockIdx.x / ntx) % nty), bz = (int)(blockIdx.x / (ntx * nty));
    const int x = bx * CL_TX + lane, Y0 = by * CL_TY, Z0 = bz * CL_TZ;
    const uint32_t below = (1u << lane) - 1u;
    for (int r = warp; r < CL_ROWS; r += CL_WARPS) {
        const int y = Y0 + r % CL_TY, z = Z0 + r / CL_TY;
        const bool in = x < ne && y < ne && z < ne;
        const bool nv = in && marca[(int64_t)x + (int64_t)ne * (y + (int64_t)ne * z)] <= 0;
        const uint32_t gaps = ~__ballot_sync(0xffffffffu, nv) & below;      // void lanes to the left
        const int start = gaps ? 32 - __clz(gaps) : 0;                        // first lane of this run
        L[r * CL_TX + lane] = nv ? r * CL_TX + start : -1;
    }
    __syncthreads();
    for (int r = warp; r < CL_ROWS; r += CL_WARPS) {
        const int li = r * CL_TX + lane;
        if (L[li] < 0) continue;
        const bool left = lane > 0 && L[li - 1] >= 0;
        if (r % CL_TY > 0 && L[li - CL_TX] >= 0 && !(left && L[li - CL_TX - 1] >= 0)) luf_union(L, li, li - CL_TX);
        if (r >= CL_TY && L[li - CL_TX * CL_TY] >= 0 && !(left && L[li - CL_TX * CL_TY - 1] >= 0))
            luf_union(L, li, li - CL_TX * CL_TY);
    }
    __syncthreads();
    for (int r = warp; r < CL_ROWS; r += CL_WARPS) {
        const int y = Y0 + r % CL_TY, z = Z0 + r / CL_TY;
        if (x >= ne || y >= ne || z >= ne) continue;
        const int li = r * CL_TX + lane;
        int32_t q = L[li];
        if (q >= 0)
            while (L[q] != q) q = L[q];
        const int32_t gq = q < 0 ? -1
                                 : (int32_t)((int64_t)(bx * CL_TX + q % CL_TX) +
                                             (int64_t)ne * ((Y0 + (q / CL_TX) % CL_TY) + (int64_t)ne * (Z0 + q / (CL_TX * CL_TY))));
        P[(int64_t)x + (int64_t)ne * (y + (int64_t)ne * z)] = gq;
    }
}

// the unions across the tiles' low faces: axis 0 over the planes x = 32a,
// axis 1 over y = 8a, axis 2 over z = 8a (a >= 1), x fastest in every launch;
// on the y and z faces a cell skips the union its left neighbour's pair
// already made (inside one x-tile)
__global__ void k_ccl_faces(PostGrid G, int axis, int32_t *P) {
    const int ne = G.ne;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nf = (ne - 1) / (axis == 0 ? CL_TX : axis == 1 ? CL_TY : CL_TZ);   // faces at a = 1..nf
    const int64_t plane = (int64_t)ne * ne;
    if (t >= (int64_t)nf * plane) return;
    const int a = (int)(t / plane) + 1;
    const int u = (int)(t % ne), v = (int)((t / ne) % ne);
    int x, y, z;
    int64_t step;
    if (axis == 0) { x = a * CL_TX; y = u; z = v; step = 1; }
    else if (axis == 1) { x = u; y = a * CL_TY; z = v; step = ne; }
    else { x = u; y = v; z = a * CL_TZ; step = plane; }
    const int64_t e = (int64_t)x + (int64_t)ne * (y + (int64_t)ne * z);
    if (P[e] < 0 || P[e - step] < 0) return;
    if (axis != 0 && x % CL_TX > 0 && P[e - 1] >= 0 && P[e - step - 1] >= 0) return;
    uf_union(P, (int32_t)e, (int32_t)(e - step));
}

// root of x without path compression (read-only: the unions are done)
__device__ __forceinline__ int32_t uf_root(const int32_t *P, int32_t x) {
    while (true) {
        const int32_t px = P[x];
        if (px == x) return x;
        x = px;
    }
}
// A hole is a non-void cell outside the component of the first cell; it takes
// the id of the first non-hole cell in +x (src/voidfinding.f90:1142-1158).
// In place: only holes are written and only non-holes are read.  Parents point
// to smaller indices, so cell 0, when non-void, is its component's root.
__global__ void k_fill_holes(PostGrid G, const int32_t *__restrict__ P, int32_t *marca) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = G.ne;
    const int64_t ne3 = (int64_t)ne * ne * ne;
    if (e >= ne3) return;
    const int32_t root0 = P[0] >= 0 ? 0 : -1;
    auto hole = [&](int64_t f) { return P[f] >= 0 && uf_root(P, (int32_t)f) != root0; };
    if (!hole(e)) return;
    const int64_t rowend = e - (e % ne) + ne;
    int64_t f = e + 1;
    while (f < rowend && hole(f)) f++;
    marca[e] = f < rowend ? marca[f] : 0;
}

// ---- VOID_PERIODIC helpers ----------------------------------------------------
__global__ void k_inner_presence(PostGrid G, const int32_t *marca, int32_t *has) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = G.nx;
    if (c >= (int64_t)nx * nx * nx) return;
    const int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    const int32_t m = marca[pidx(G, i, j, k)];
    if (m > 0) has[m - 1] = 1;
}
__global__ void k_bbox(PostGrid G, const int32_t *marca, int32_t *bb /* 6 per label: min xyz, max xyz */) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = G.ne;
    if (e >= (int64_t)ne * ne * ne) return;
    const int32_t m = marca[e];
    if (m <= 0) return;
    const int c[3] = {(int)(e % ne) + G.low1, (int)((e / ne) % ne) + G.low1, (int)(e / ((int64_t)ne * ne)) + G.low1};
    for (int a = 0; a < 3; a++) {
        atomicMin(&bb[(size_t)(m - 1) * 6 + a], c[a]);
        atomicMax(&bb[(size_t)(m - 1) * 6 + 3 + a], c[a]);
    }
}
// shifted-cell overlap counts of every outer-centred void against its IND2;
// labmap maps stored labels to the current ones (identity for the first pass);
// only_label > 0 restricts the pass to one (current) label
// (box: when bdim[0] > 0 only the cells of the box starting at ext offsets
// blo are visited -- the bounding box of the one label being recounted)
__global__ void k_periodic_counts(PostGrid G, const int32_t *marca, const int32_t *labmap, const int8_t *shift,
                                  const int32_t *ind2, int32_t only_label, int32_t *cnt /* 2 per label */,
                                  int3 blo = make_int3(0, 0, 0), int3 bdim = make_int3(0, 0, 0),
                                  int32_t only_ind2 = 0) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = G.ne;
    if (bdim.x > 0) {
        if (e >= (int64_t)bdim.x * bdim.y * bdim.z) return;
        const int bx = (int)(e % bdim.x), by = (int)((e / bdim.x) % bdim.y), bz = (int)(e / ((int64_t)bdim.x * bdim.y));
        e = (int64_t)(blo.x + bx) + (int64_t)ne * ((blo.y + by) + (int64_t)ne * (blo.z + bz));
    } else if (e >= (int64_t)ne * ne * ne) {
        return;
    }
    int32_t m = marca[e];
    if (m <= 0) return;
    m = labmap[m];
    if (only_label > 0 && m != only_label) return;
    const int8_t *s = shift + (size_t)(m - 1) * 3;
    if (s[0] == 0 && s[1] == 0 && s[2] == 0) return;
    const int i = (int)(e % ne) + G.low1 + s[0] * G.nx;
    const int j = (int)((e / ne) % ne) + G.low1 + s[1] * G.nx;
    const int k = (int)(e / ((int64_t)ne * ne)) + G.low1 + s[2] * G.nx;
    if (i < G.low1 || i > G.low2 || j < G.low1 || j > G.low2 || k < G.low1 || k > G.low2) return;
    atomicAdd(&cnt[(size_t)(m - 1) * 2 + 1], 1);
    int32_t lab = marca[pidx(G, i, j, k)];
    if (lab > 0) lab = labmap[lab];
    if (lab == (only_label > 0 ? only_ind2 : ind2[m - 1])) atomicAdd(&cnt[(size_t)(m - 1) * 2], 1);
}
// out[i] = src[idx[i]]
__global__ void k_gather_i32(int32_t n, const int64_t *__restrict__ idx, const int32_t *__restrict__ src,
                             int32_t *__restrict__ out) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[idx[i]];
}
// dst[pairs[2i]] = pairs[2i + 1]
__global__ void k_scatter_pairs(int32_t n, const int32_t *__restrict__ pairs, int32_t *__restrict__ dst) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[pairs[2 * i]] = pairs[2 * i + 1];
}

// ---- neighbour lists of MERGE_VOID: cubes of the same father whose 1-cell
//      halo boxes overlap; d2 is distance() of src/kdtree.f90:1441-1465 on the
//      initial centres, inball tests it against the cube's ball radius ----------
struct NbrArgs {
    int32_t nv, cap, nbk, low1, bs;
    const int32_t *box;          // x0,x1,y0,y1,z0,z1 arrays of cap entries
    const int32_t *father;
    const float *cx, *cy, *cz, *r2;
    const int32_t *bstart, *bitems;
    float L;
    int periodic;
};
__device__ __forceinline__ int nbr_bucket(const NbrArgs &A, int v) {
    const int b = (v - A.low1) / A.bs;
    return b < 0 ? 0 : (b >= A.nbk ? A.nbk - 1 : b);
}
__global__ void k_cube_bucket_count(NbrArgs A, int32_t *cnt) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nv) return;
    const int bx = nbr_bucket(A, (A.box[0 * A.cap + i] + A.box[1 * A.cap + i]) / 2);
    const int by = nbr_bucket(A, (A.box[2 * A.cap + i] + A.box[3 * A.cap + i]) / 2);
    const int bz = nbr_bucket(A, (A.box[4 * A.cap + i] + A.box[5 * A.cap + i]) / 2);
    atomicAdd(&cnt[bx + A.nbk * (by + A.nbk * bz)], 1);
}
__global__ void k_cube_bucket_fill(NbrArgs A, int32_t *cursor, int32_t *items) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nv) return;
    const int bx = nbr_bucket(A, (A.box[0 * A.cap + i] + A.box[1 * A.cap + i]) / 2);
    const int by = nbr_bucket(A, (A.box[2 * A.cap + i] + A.box[3 * A.cap + i]) / 2);
    const int bz = nbr_bucket(A, (A.box[4 * A.cap + i] + A.box[5 * A.cap + i]) / 2);
    items[atomicAdd(&cursor[bx + A.nbk * (by + A.nbk * bz)], 1)] = i;
}
template <bool FILL>
__global__ void k_cube_nbrs(NbrArgs A, int32_t *count, const int32_t *start, int32_t *nbr, float *d2out,
                            uint8_t *inball) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nv) return;
    int lo[3], hi[3], bc[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = A.box[(2 * a) * A.cap + i];
        hi[a] = A.box[(2 * a + 1) * A.cap + i];
        bc[a] = nbr_bucket(A, (lo[a] + hi[a]) / 2);
    }
    const int32_t f = A.father[i];
    int32_t n = 0;
    const int32_t base = FILL ? start[i] : 0;
    for (int bz = max(bc[2] - 1, 0); bz <= min(bc[2] + 1, A.nbk - 1); bz++)
        for (int by = max(bc[1] - 1, 0); by <= min(bc[1] + 1, A.nbk - 1); by++)
            for (int bx = max(bc[0] - 1, 0); bx <= min(bc[0] + 1, A.nbk - 1); bx++) {
                const int b = bx + A.nbk * (by + A.nbk * bz);
                for (int32_t t = A.bstart[b]; t < A.bstart[b + 1]; t++) {
                    const int32_t j = A.bitems[t];
                    if (j == i || A.father[j] != f) continue;
                    bool ov = true;
                    for (int a = 0; a < 3; a++)
                        if (lo[a] - 1 > A.box[(2 * a + 1) * A.cap + j] + 1 || A.box[(2 * a) * A.cap + j] - 1 > hi[a] + 1) ov = false;
                    if (!ov) continue;
                    if (FILL) {
                        float dx = __fsub_rn(A.cx[j], A.cx[i]), dy = __fsub_rn(A.cy[j], A.cy[i]), dz = __fsub_rn(A.cz[j], A.cz[i]);
                        if (A.periodic) {
                            float q = fabsf(dx); dx = fminf(q, __fsub_rn(A.L, q));
                            q = fabsf(dy); dy = fminf(q, __fsub_rn(A.L, q));
                            q = fabsf(dz); dz = fminf(q, __fsub_rn(A.L, q));
                        }
                        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
                        nbr[base + n] = j;
                        d2out[base + n] = d2;
                        inball[base + n] = d2 <= A.r2[i] ? 1 : 0;
                    }
                    n++;
                }
            }
    if (!FILL) count[i] = n;
}

template <class T>
static T *dev_upload(Ctx &c, BufId id, const T *h, size_t n) {
    T *d = c.get_t<T>(id, std::max<size_t>(n, 1));
    if (n) AV_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return d;
}
template <class T>
static void dev_download(Ctx &c, T *h, const T *d, size_t n) {
    if (n) AV_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
}

void merge_post(Ctx &c, const avism_params *p, const Level &L, int32_t nv, const avism_cubes *cb,
                const float *u1co_inner, float meandens, avism_voids *out, int32_t *marca_ext_out) {
    const avism_grid &g = L.g;
    const int ne = g.ne, nx = g.nx;
    const int64_t ne3 = (int64_t)ne * ne * ne;
    const float dx = g.dx;
    const double pi = 3.141592653589793;
    PostGrid PG{g.low1, g.low2, ne, nx};
    const int32_t nvs = std::max(nv, 1);

    // ---- INDEXX on VOL, reversed (avism.f90:1738-1745)
    std::vector<int32_t> indice(nvs);
    {
        float *vol_d = dev_upload<float>(c, B_RED2, cb->vol, nv);
        int32_t *ind_d = c.get_t<int32_t>(B_QUERY, nvs);
        indexx_device(c, nv, vol_d, ind_d);
        std::vector<int32_t> asc(nvs);
        dev_download(c, asc.data(), ind_d, nv);
        for (int32_t i = 0; i < nv; i++) indice[i] = asc[nv - 1 - i];
    }
    c.mark("indexx_vol");
    // ---- neighbour lists for MERGE_VOID, built on the device
    std::vector<int32_t> nbr_start(nvs + 1, 0), nbr;
    std::vector<float> nbr_d2;
    std::vector<uint8_t> nbr_inball;
    int32_t *box_d = nullptr;
    {
        std::vector<int32_t> boxes((size_t)nvs * 6);
        const int32_t *src[6] = {cb->inicio_x, cb->final_x, cb->inicio_y, cb->final_y, cb->inicio_z, cb->final_z};
        int ext_max = 1;
        for (int a = 0; a < 6; a++) std::memcpy(&boxes[(size_t)a * nvs], src[a], sizeof(int32_t) * (size_t)nv);
        for (int32_t i = 0; i < nv; i++)
            for (int a = 0; a < 3; a++) ext_max = std::max(ext_max, src[2 * a + 1][i] - src[2 * a][i] + 1);
        box_d = dev_upload<int32_t>(c, B_RED0, boxes.data(), boxes.size());
        std::vector<float> cen((size_t)nvs * 4);
        for (int32_t i = 0; i < nv; i++) {
            cen[i] = L.rad_at(1) + (float)(cb->icx[i] - 1) * dx;
            cen[(size_t)nvs + i] = L.rad_at(1) + (float)(cb->icy[i] - 1) * dx;
            cen[(size_t)2 * nvs + i] = L.rad_at(1) + (float)(cb->icz[i] - 1) * dx;
            const float v = ((cb->rfin_x[i] - cb->rini_x[i]) * (cb->rfin_y[i] - cb->rini_y[i])) * (cb->rfin_z[i] - cb->rini_z[i]);
            cen[(size_t)3 * nvs + i] = merge_ball_r2(v, dx);
        }
        float *cen_d = dev_upload<float>(c, B_RED1, cen.data(), cen.size());
        int32_t *fa_d = dev_upload<int32_t>(c, B_LABMAP, cb->father, nv);
        NbrArgs A;
        A.nv = nv; A.cap = nvs; A.low1 = g.low1; A.bs = ext_max + 2;
        A.nbk = std::max(1, (ne + A.bs - 1) / A.bs);
        A.box = box_d; A.father = fa_d; A.cx = cen_d; A.cy = cen_d + nvs; A.cz = cen_d + 2 * (size_t)nvs;
        A.r2 = cen_d + 3 * (size_t)nvs; A.L = p->periodic ? g.lado0plus : 0.0f; A.periodic = p->periodic;
        const int64_t nb3 = (int64_t)A.nbk * A.nbk * A.nbk;
        int32_t *bcnt = c.get_t<int32_t>(B_SCAN_A, nb3 + 1);
        int32_t *bstart = c.get_t<int32_t>(B_SCAN_B, nb3 + 1);
        int32_t *items = c.get_t<int32_t>(B_LIST_A, nvs);
        AV_CUDA(cudaMemsetAsync(bcnt, 0, sizeof(int32_t) * (size_t)(nb3 + 1), c.stream));
        if (nv > 0) ++c.launches, k_cube_bucket_count<<<grid_for(nv, 256), 256, 0, c.stream>>>(A, bcnt);
        size_t tmp = 0;
        AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, bcnt, bstart, (int)(nb3 + 1), c.stream));
        void *t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, bcnt, bstart, (int)(nb3 + 1), c.stream));
        AV_CUDA(cudaMemcpyAsync(bcnt, bstart, sizeof(int32_t) * (size_t)(nb3 + 1), cudaMemcpyDeviceToDevice, c.stream));
        if (nv > 0) ++c.launches, k_cube_bucket_fill<<<grid_for(nv, 256), 256, 0, c.stream>>>(A, bcnt, items);
        A.bstart = bstart; A.bitems = items;
        int32_t *ncount = c.get_t<int32_t>(B_LIST_B, nvs + 1);
        int32_t *nstart = c.get_t<int32_t>(B_GE, nvs + 1);
        AV_CUDA(cudaMemsetAsync(ncount, 0, sizeof(int32_t) * (size_t)(nvs + 1), c.stream));
        if (nv > 0) ++c.launches, k_cube_nbrs<false><<<grid_for(nv, 128), 128, 0, c.stream>>>(A, ncount, nullptr, nullptr, nullptr, nullptr);
        AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, ncount, nstart, nv + 1, c.stream));
        t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, ncount, nstart, nv + 1, c.stream));
        dev_download(c, nbr_start.data(), nstart, (size_t)nv + 1);
        const int32_t tot = nbr_start[nv];
        int32_t *nbr_d = c.get_t<int32_t>(B_CAND_POS, std::max(tot, 1));
        float *d2_d = c.get_t<float>(B_CAND_KEY, std::max(tot, 1));
        uint8_t *ib_d = c.get_t<uint8_t>(B_COVER, std::max(tot, 1));
        if (nv > 0) ++c.launches, k_cube_nbrs<true><<<grid_for(nv, 128), 128, 0, c.stream>>>(A, nullptr, nstart, nbr_d, d2_d, ib_d);
        AV_CUDA(cudaGetLastError());
        nbr.resize(std::max(tot, 1));
        nbr_d2.resize(std::max(tot, 1));
        nbr_inball.resize(std::max(tot, 1));
        AV_CUDA(cudaMemcpyAsync(nbr.data(), nbr_d, sizeof(int32_t) * (size_t)tot, cudaMemcpyDeviceToHost, c.stream));
        AV_CUDA(cudaMemcpyAsync(nbr_d2.data(), d2_d, sizeof(float) * (size_t)tot, cudaMemcpyDeviceToHost, c.stream));
        dev_download(c, nbr_inball.data(), ib_d, (size_t)tot);
    }
    c.mark("merge_lists");
    // ---- MERGE_VOID
    MergeIn mi;
    mi.nvoid = nv; mi.low1 = g.low1; mi.low2 = g.low2; mi.periodic = p->periodic;
    mi.dx = dx; mi.rx1 = L.rad_at(1); mi.lado0plus = g.lado0plus;
    mi.x0 = cb->inicio_x; mi.x1 = cb->final_x; mi.y0 = cb->inicio_y; mi.y1 = cb->final_y;
    mi.z0 = cb->inicio_z; mi.z1 = cb->final_z; mi.icx = cb->icx; mi.icy = cb->icy; mi.icz = cb->icz;
    mi.father = cb->father; mi.rix = cb->rini_x; mi.rfx = cb->rfin_x; mi.riy = cb->rini_y;
    mi.rfy = cb->rfin_y; mi.riz = cb->rini_z; mi.rfz = cb->rfin_z; mi.indice = indice.data();
    mi.nbr_start = nbr_start.data(); mi.nbr = nbr.data(); mi.nbr_d2 = nbr_d2.data(); mi.nbr_inball = nbr_inball.data();
    MergeOut mo;
    merge_cubes_host(mi, mo);
    c.mark("merge_host");
    std::vector<int32_t> &uvoid = mo.uvoid;
    std::vector<float> &volnew = mo.volnew;

    // ---- paint MARCA
    int32_t *marca = c.get_t<int32_t>(B_MARCA, ne3);
    {
        int32_t *pt_d = dev_upload<int32_t>(c, B_RED1, mo.paint_time.data(), nv);
        std::vector<int32_t> owner_by_time(nvs, 0);
        for (int32_t i = 0; i < nv; i++) {
            AV_CHECK(mo.paint_time[i] >= 0 && mo.paint_time[i] < nv, AVISM_ERR_INTERNAL, "merge: cube never painted");
            owner_by_time[mo.paint_time[i]] = mo.paint_owner[i];
        }
        int32_t *obt_d = dev_upload<int32_t>(c, B_LABMAP, owner_by_time.data(), nv);
        int32_t *tgrid = c.get_t<int32_t>(B_CCL, ne3);
        ++c.launches, k_fill_i32<<<grid_for(ne3, 256), 256, 0, c.stream>>>(ne3, tgrid, INT_MAX);
        if (nv > 0) ++c.launches, k_paint_time<<<grid_for((int64_t)nv * 32, 256), 256, 0, c.stream>>>(PG, box_d, nvs, pt_d, nv, tgrid);
        ++c.launches, k_time_to_label<<<grid_for(ne3, 256), 256, 0, c.stream>>>(ne3, tgrid, obt_d, marca);
        AV_CUDA(cudaGetLastError());
    }
    c.mark("paint_marca");
    std::vector<char> rm(nvs + 1, 0);
    std::vector<int32_t> ncellv(nvs, 0);
    int32_t *map_d = c.get_t<int32_t>(B_LABEL_AUX, nvs + 1);
    int32_t *uv_d = c.get_t<int32_t>(B_RED1, nvs);
    auto push_uvoid = [&]() { AV_CUDA(cudaMemcpyAsync(uv_d, uvoid.data(), sizeof(int32_t) * (size_t)nv, cudaMemcpyHostToDevice, c.stream)); };
    // removal of main voids: cells to 0, owners of absorbed cubes to 0
    auto apply_removals = [&]() {
        bool any = false;
        for (int32_t i = 1; i <= nv; i++) any |= rm[i] != 0;
        if (!any) return;
        std::vector<int32_t> map(nvs + 1);
        for (int32_t i = 0; i <= nv; i++) map[i] = rm[i] ? 0 : i;
        AV_CUDA(cudaMemcpyAsync(map_d, map.data(), sizeof(int32_t) * (size_t)(nv + 1), cudaMemcpyHostToDevice, c.stream));
        ++c.launches, k_relabel<<<grid_for((ne3 + 3) / 4, 256), 256, 0, c.stream>>>(ne3, marca, map_d);
        for (int32_t i = 0; i < nv; i++)
            if (uvoid[i] > 0 && rm[uvoid[i]]) uvoid[i] = 0;
        for (int32_t i = 1; i <= nv; i++)
            if (rm[i]) { uvoid[i - 1] = 0; volnew[i - 1] = 0.0f; ncellv[i - 1] = 0; rm[i] = 0; }
        c.sync();
    };
    auto count_cells = [&]() {
        int32_t *nc_d = c.get_t<int32_t>(B_RED2, nvs);
        AV_CUDA(cudaMemsetAsync(nc_d, 0, sizeof(int32_t) * (size_t)nvs, c.stream));
        push_uvoid();
        ++c.launches, k_ncellv<<<grid_for(ne3, 256), 256, 0, c.stream>>>(ne3, marca, uv_d, nc_d);
        dev_download(c, ncellv.data(), nc_d, nv);
    };
    count_cells();
    for (int32_t I = 0; I < nv; I++) {                        // NCELL_MIN = 10
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        if (ncellv[ind - 1] < 10) rm[ind] = 1;
    }
    apply_removals();
    c.mark("ncell_min");

    // ---- VOID_SHAPE
    std::vector<float> eps(nvs, 0.0f), ipv(nvs, 0.0f);
    {
        float *rad_d = dev_upload<float>(c, B_RAD, L.rad.data(), L.rad.size());
        float *gc_d = c.get_t<float>(B_RED0, (size_t)nvs * 3);
        AV_CUDA(cudaMemcpyAsync(gc_d, mo.gxc.data(), sizeof(float) * nv, cudaMemcpyHostToDevice, c.stream));
        AV_CUDA(cudaMemcpyAsync(gc_d + nvs, mo.gyc.data(), sizeof(float) * nv, cudaMemcpyHostToDevice, c.stream));
        AV_CUDA(cudaMemcpyAsync(gc_d + 2 * nvs, mo.gzc.data(), sizeof(float) * nv, cudaMemcpyHostToDevice, c.stream));
        float *in_d = c.get_t<float>(B_LL_SUM, (size_t)nvs * 6);
        c.mark("shape_setup");
        const int32_t *vcell;
        const int64_t *voff;
        AV_CHECK(ne3 < (int64_t)INT32_MAX, AVISM_ERR_UNSUPPORTED, "VOID_SHAPE: ext grid above 2^31 cells");
        void_cell_lists(c, (int32_t)ne3, ExtVoidCell{marca}, marca, PG, 0, nv, &vcell, &voff, nullptr);
        c.mark("shape_lists");
        if (nv > 0)
            ++c.launches, k_inertia_seq<<<grid_for(nv, SEQ_WARPS), SEQ_WARPS * 32, 0, c.stream>>>(
                nv, voff, vcell, PG, rad_d, g.rad_lo, gc_d, gc_d + nvs, gc_d + 2 * nvs, in_d);
        AV_CUDA(cudaGetLastError());
        c.mark("shape_inertia");
        int32_t *nc_d = dev_upload<int32_t>(c, B_RED2, ncellv.data(), (size_t)nv);
        push_uvoid();
        float *ax_d = gc_d;                          // the centres are consumed by k_inertia_seq
        ++c.launches, k_void_axes<<<grid_for(nv, 128), 128, 0, c.stream>>>(nv, uv_d, nc_d, in_d, dx, pi, ax_d, ax_d + nvs);
        dev_download(c, eps.data(), ax_d, nv);
        dev_download(c, ipv.data(), ax_d + nvs, nv);
        c.mark("shape_axes");
    }
    const float cellv = (dx * dx) * dx;
    const double vmin = ((double)(4.0f / 3.0f) * pi) * (double)((p->rmin * p->rmin) * p->rmin);
    auto redefine_volnew = [&]() {
        for (int32_t i = 0; i < nv; i++) volnew[i] = 0.0f;
        for (int32_t I = 0; I < nv; I++) {
            const int32_t ind = indice[I];
            if (uvoid[ind - 1] >= 0) continue;
            volnew[ind - 1] = (float)((double)ncellv[ind - 1] * (double)cellv);
        }
    };
    auto rmin_filter = [&]() {
        for (int32_t I = 0; I < nv; I++) {
            const int32_t ind = indice[I];
            if (uvoid[ind - 1] >= 0) continue;
            if ((double)volnew[ind - 1] < vmin) rm[ind] = 1;
        }
        apply_removals();
    };
    c.mark("void_shape");
    redefine_volnew();
    rmin_filter();
    std::vector<float> xc(nvs, 0.0f), yc(nvs, 0.0f), zc(nvs, 0.0f);
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind = indice[I];
        if (uvoid[ind - 1] >= 0) continue;
        xc[ind - 1] = L.rad_at(1) + (float)(cb->icx[ind - 1] - 1) * dx;
        yc[ind - 1] = L.rad_at(1) + (float)(cb->icy[ind - 1] - 1) * dx;
        zc[ind - 1] = L.rad_at(1) + (float)(cb->icz[ind - 1] - 1) * dx;
    }

    // ---- SIMPLE_CONNECTION_FAST
    {
        int32_t *P = c.get_t<int32_t>(B_CCL, ne3);
        const int64_t ntl = (int64_t)((ne + CL_TX - 1) / CL_TX) * ((ne + CL_TY - 1) / CL_TY) * ((ne + CL_TZ - 1) / CL_TZ);
        ++c.launches, k_ccl_local<<<(unsigned)ntl, CL_THREADS, 0, c.stream>>>(PG, marca, P);
        for (int axis = 0; axis < 3; axis++) {
            const int64_t nface = (int64_t)((ne - 1) / (axis == 0 ? CL_TX : axis == 1 ? CL_TY : CL_TZ)) * ne * ne;
            if (nface > 0) ++c.launches, k_ccl_faces<<<grid_for(nface, 256), 256, 0, c.stream>>>(PG, axis, P);
        }
        ++c.launches, k_fill_holes<<<grid_for(ne3, 256), 256, 0, c.stream>>>(PG, P, marca);
        AV_CUDA(cudaGetLastError());
    }
    c.mark("simple_connection");

    // ---- VOID_PERIODIC
    if (p->periodic) {
        std::vector<int32_t> has(nvs, 0);
        {
            int32_t *has_d = c.get_t<int32_t>(B_RED2, nvs);
            AV_CUDA(cudaMemsetAsync(has_d, 0, sizeof(int32_t) * (size_t)nvs, c.stream));
            ++c.launches, k_inner_presence<<<grid_for((int64_t)nx * nx * nx, 256), 256, 0, c.stream>>>(PG, marca, has_d);
            dev_download(c, has.data(), has_d, nv);
        }
        std::vector<int32_t> kept;
        for (int32_t I = 0; I < nv; I++) {
            const int32_t ind = indice[I];
            if (uvoid[ind - 1] >= 0) continue;
            if (!has[ind - 1]) rm[ind] = 1; else kept.push_back(ind);
        }
        apply_removals();
        const float half = p->lado0 / 2.0f;
        std::vector<int8_t> shift((size_t)nvs * 3, 0);
        std::vector<int32_t> ind2spec(nvs, 0);
        std::vector<int32_t> outer;
        std::vector<int64_t> centre_cell(nvs, -1);
        for (int32_t ind : kept) {
            const float x = mo.gxc[ind - 1], y = mo.gyc[ind - 1], z = mo.gzc[ind - 1];
            int s[3] = {0, 0, 0};
            if (x < -half) s[0] = 1; if (x > half) s[0] = -1;
            if (y < -half) s[1] = 1; if (y > half) s[1] = -1;
            if (z < -half) s[2] = 1; if (z > half) s[2] = -1;
            if (!s[0] && !s[1] && !s[2]) continue;
            const int ig[3] = {(int)((x - L.rad_at(1)) / dx) + 1, (int)((y - L.rad_at(1)) / dx) + 1,
                               (int)((z - L.rad_at(1)) / dx) + 1};
            int cc[3];
            bool ok = true;
            for (int a = 0; a < 3; a++) {
                cc[a] = ig[a] + s[a] * nx;
                if (cc[a] < g.low1 || cc[a] > g.low2) ok = false;
            }
            if (!ok) continue;
            for (int a = 0; a < 3; a++) shift[(size_t)(ind - 1) * 3 + a] = (int8_t)s[a];
            centre_cell[ind - 1] = (int64_t)(cc[0] - g.low1) + (int64_t)ne * ((int64_t)(cc[1] - g.low1) + (int64_t)ne * (cc[2] - g.low1));
            outer.push_back(ind);
        }
        if (!outer.empty()) {
            // labels at the shifted centres, initial state (one gather)
            const int32_t nout = (int32_t)outer.size();
            std::vector<int32_t> m0(nout);
            {
                std::vector<int64_t> cells(nout);
                for (int32_t q = 0; q < nout; q++) cells[q] = centre_cell[outer[q] - 1];
                const int64_t *cells_d = dev_upload<int64_t>(c, B_PER_CELL, cells.data(), nout);
                int32_t *m0_d = c.get_t<int32_t>(B_PER_LAB, nout);
                ++c.launches, k_gather_i32<<<grid_for(nout, 256), 256, 0, c.stream>>>(nout, cells_d, marca, m0_d);
                dev_download(c, m0.data(), m0_d, nout);
            }
            for (int32_t q = 0; q < nout; q++) ind2spec[outer[q] - 1] = m0[q];
            std::vector<int32_t> labmap(nvs + 1);
            for (int32_t i = 0; i <= nv; i++) labmap[i] = i;
            int32_t *lm_d = dev_upload<int32_t>(c, B_LABMAP, labmap.data(), nv + 1);
            int8_t *sh_d = dev_upload<int8_t>(c, B_RED0, shift.data(), (size_t)nvs * 3);
            int32_t *i2_d = dev_upload<int32_t>(c, B_RED1, ind2spec.data(), nvs);
            int32_t *cnt_d = c.get_t<int32_t>(B_RED2, (size_t)nvs * 2);
            AV_CUDA(cudaMemsetAsync(cnt_d, 0, sizeof(int32_t) * 2 * (size_t)nvs, c.stream));
            ++c.launches, k_periodic_counts<<<grid_for(ne3, 256), 256, 0, c.stream>>>(PG, marca, lm_d, sh_d, i2_d, 0, cnt_d);
            std::vector<int32_t> cnt((size_t)nvs * 2);
            dev_download(c, cnt.data(), cnt_d, (size_t)nv * 2);
            std::vector<int32_t> bb((size_t)nvs * 6);
            {
                int32_t *bb_d = c.get_t<int32_t>(B_SCAN_B, (size_t)nvs * 6);
                std::vector<int32_t> init((size_t)nvs * 6);
                for (int32_t i = 0; i < nvs; i++)
                    for (int a = 0; a < 3; a++) { init[(size_t)i * 6 + a] = INT_MAX; init[(size_t)i * 6 + 3 + a] = INT_MIN; }
                AV_CUDA(cudaMemcpyAsync(bb_d, init.data(), sizeof(int32_t) * init.size(), cudaMemcpyHostToDevice, c.stream));
                ++c.launches, k_bbox<<<grid_for(ne3, 256), 256, 0, c.stream>>>(PG, marca, bb_d);
                dev_download(c, bb.data(), bb_d, (size_t)nv * 6);
            }
            // union-find over labels for CHANGE_BELONG
            std::vector<int32_t> parent(nvs + 1);
            for (int32_t i = 0; i <= nv; i++) parent[i] = i;
            std::function<int32_t(int32_t)> find = [&](int32_t x) {
                while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
                return x;
            };
            std::vector<std::vector<int32_t>> members(nvs + 1);
            std::vector<std::array<int32_t, 6>> curbb(nvs + 1);
            for (int32_t i = 1; i <= nv; i++) {
                for (int a = 0; a < 6; a++) curbb[i][a] = bb[(size_t)(i - 1) * 6 + a];
            }
            std::vector<std::array<int32_t, 6>> changed_bb;
            // (label, new root) pairs not yet applied to the device label map
            std::vector<int32_t> lm_pend;
            // voids by the main void they belong to (uvoid > 0): linked lists, so
            // CHANGE_BELONG moves a void's members without scanning all voids
            std::vector<int32_t> lhead(nvs + 1, -1), ltail(nvs + 1, -1), lnext(nvs, -1);
            auto lpush = [&](int32_t v, int32_t i) {
                lnext[i] = -1;
                if (ltail[v] < 0) lhead[v] = i; else lnext[ltail[v]] = i;
                ltail[v] = i;
            };
            for (int32_t i = 0; i < nv; i++)
                if (uvoid[i] > 0) lpush(uvoid[i], i);
            for (int32_t ind : outer) {
                const int8_t *s = &shift[(size_t)(ind - 1) * 3];
                int32_t i2 = ind2spec[ind - 1];
                if (i2 > 0) i2 = find(i2);
                if (i2 == 0) continue;
                // could an earlier CHANGE_BELONG have touched this void's counts?
                bool affected = !members[ind].empty() || i2 != ind2spec[ind - 1];
                const auto &b = curbb[ind];
                if (!affected && b[0] <= b[3]) {
                    for (const auto &cbx : changed_bb) {
                        bool inter = true;
                        for (int a = 0; a < 3; a++) {
                            const int lo = b[a] + s[a] * nx, hi = b[3 + a] + s[a] * nx;
                            if (hi < cbx[a] || lo > cbx[3 + a]) inter = false;
                        }
                        if (inter) { affected = true; break; }
                    }
                }
                int64_t counter = cnt[(size_t)(ind - 1) * 2], counter2 = cnt[(size_t)(ind - 1) * 2 + 1];
                if (affected) {
                    if (!lm_pend.empty()) {
                        const int32_t np = (int32_t)(lm_pend.size() / 2);
                        const int32_t *pr_d = dev_upload<int32_t>(c, B_PER_PAIRS, lm_pend.data(), lm_pend.size());
                        ++c.launches, k_scatter_pairs<<<grid_for(np, 256), 256, 0, c.stream>>>(np, pr_d, lm_d);
                        lm_pend.clear();
                    }
                    int32_t *one = c.get_t<int32_t>(B_RED2, (size_t)nvs * 2);
                    AV_CUDA(cudaMemsetAsync(one + (size_t)(ind - 1) * 2, 0, 8, c.stream));
                    // the label's cells lie in its bounding box (merges extend it)
                    const auto &bx = curbb[ind];
                    if (bx[0] <= bx[3]) {
                        const int3 blo = make_int3(bx[0] - g.low1, bx[1] - g.low1, bx[2] - g.low1);
                        const int3 bd = make_int3(bx[3] - bx[0] + 1, bx[4] - bx[1] + 1, bx[5] - bx[2] + 1);
                        const int64_t nbox = (int64_t)bd.x * bd.y * bd.z;
                        ++c.launches, k_periodic_counts<<<grid_for(nbox, 256), 256, 0, c.stream>>>(
                            PG, marca, lm_d, sh_d, i2_d, ind, one, blo, bd, i2);
                    }
                    int32_t r2[2];
                    dev_download(c, r2, one + (size_t)(ind - 1) * 2, 2);
                    counter = r2[0];
                    counter2 = r2[1];
                }
                const float inter = counter2 == 0 ? 0.0f : (float)counter / (float)counter2;
                if (inter > 0.4f) {                                  // CHANGE_BELONG(IND2, IND)
                    // UVOID(IND) = IND2, then every void with UVOID == IND follows
                    uvoid[ind - 1] = i2;
                    if (i2 != ind) {
                        for (int32_t i = lhead[ind]; i >= 0; i = lnext[i]) uvoid[i] = i2;
                        if (lhead[ind] >= 0) {
                            if (ltail[i2] < 0) lhead[i2] = lhead[ind]; else lnext[ltail[i2]] = lhead[ind];
                            ltail[i2] = ltail[ind];
                            lhead[ind] = ltail[ind] = -1;
                        }
                    }
                    lpush(i2, ind - 1);
                    if (i2 != ind) {
                        // IND's set (IND and what it absorbed) now resolves to IND2
                        lm_pend.push_back(ind);
                        lm_pend.push_back(i2);
                        for (int32_t mm : members[ind]) {
                            lm_pend.push_back(mm);
                            lm_pend.push_back(i2);
                        }
                        parent[ind] = i2;
                        members[i2].push_back(ind);
                        for (int32_t mm : members[ind]) members[i2].push_back(mm);
                        auto &tb = curbb[i2];
                        for (int a = 0; a < 3; a++) {
                            tb[a] = std::min(tb[a], b[a]);
                            tb[3 + a] = std::max(tb[3 + a], b[3 + a]);
                        }
                        changed_bb.push_back(b);
                    }
                    volnew[ind - 1] = 0.0f;
                }
            }
            // apply the label changes to MARCA
            std::vector<int32_t> flat(nvs + 1);
            for (int32_t i = 0; i <= nv; i++) flat[i] = i == 0 ? 0 : find(i);
            AV_CUDA(cudaMemcpyAsync(map_d, flat.data(), sizeof(int32_t) * (size_t)(nv + 1), cudaMemcpyHostToDevice, c.stream));
            ++c.launches, k_relabel<<<grid_for((ne3 + 3) / 4, 256), 256, 0, c.stream>>>(ne3, marca, map_d);
            c.sync();
        }
    }

    c.mark("void_periodic");
    // ---- global properties (inner cells), VOLNEW, RMIN, NVOIDT
    std::vector<float> umean(nvs, 0.0f), mtot(nvs, 0.0f);
    double volt = 0.0;
    {
        push_uvoid();
        const float rete3 = (g.rete * g.rete) * g.rete;
        const int32_t *pcell;
        const int64_t *poff;
        const int64_t nc3 = (int64_t)nx * nx * nx;
        AV_CHECK(nc3 < (int64_t)INT32_MAX, AVISM_ERR_UNSUPPORTED, "global properties: grid above 2^31 cells");
        void_cell_lists(c, (int32_t)nc3, InnerMainCell{PG, marca, uv_d}, marca, PG, 1, nv, &pcell, &poff,
                        ncellv.data());
        float *sum_d = c.get_t<float>(B_LL_SUM, (size_t)nvs * 2);
        if (nv > 0)
            ++c.launches, k_props_seq<<<grid_for(nv, SEQ_WARPS), SEQ_WARPS * 32, 0, c.stream>>>(
                nv, poff, pcell, u1co_inner, meandens, dx, rete3, sum_d);
        AV_CUDA(cudaGetLastError());
        std::vector<float> sums((size_t)nvs * 2);
        dev_download(c, sums.data(), sum_d, (size_t)nv * 2);
        int64_t ncount = 0;
        for (int32_t i = 0; i < nv; i++) {
            umean[i] = sums[(size_t)i * 2];
            mtot[i] = sums[(size_t)i * 2 + 1];
            ncount += ncellv[i];
            if (ncellv[i] > 0) umean[i] = umean[i] / (float)ncellv[i];
        }
        volt = (double)ncount * (double)cellv;
    }
    redefine_volnew();
    rmin_filter();
    int32_t nvoidt = 0;
    std::vector<float> req(nvs, 0.0f);
    for (int32_t i = 0; i < nv; i++) {
        if (uvoid[i] != -1) continue;
        nvoidt++;
        // ((3.*VOLM)/(4.*PI))**(1./3.) (src/avism.f90:2071): VOLM is REAL*8
        // (src/avism.f90:73), so 3.*VOLM, 4.*PI and the quotient are REAL*8
        // products; 1./3. is a REAL*4 quotient widened for the power
        req[i] = (float)std::pow((3.0 * (double)volnew[i]) / (4.0 * pi), (double)(1.0f / 3.0f));
    }

    // ---- outputs
    // host columns: a plain copy into host arrays, an upload into device ones
    auto put = [&](void *dst, const void *src, size_t bytes) {
        if (!dst || bytes == 0) return;
        if (is_device_ptr(dst)) AV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
        else std::memcpy(dst, src, bytes);
    };
    auto put_i = [&](int32_t *dst, const std::vector<int32_t> &v) { put(dst, v.data(), sizeof(int32_t) * (size_t)nv); };
    auto put_f = [&](float *dst, const std::vector<float> &v) { put(dst, v.data(), sizeof(float) * (size_t)nv); };
    put_i(out->indice, indice);
    put_i(out->uvoid, uvoid);
    put_i(out->ncellv, ncellv);
    put_f(out->volnew, volnew);
    put_f(out->req, req);
    put_f(out->xc, xc); put_f(out->yc, yc); put_f(out->zc, zc);
    put_f(out->gxc, mo.gxc); put_f(out->gyc, mo.gyc); put_f(out->gzc, mo.gzc);
    put_f(out->eps, eps); put_f(out->ip, ipv);
    put_f(out->umean, umean); put_f(out->mtot, mtot);
    out->nvoid2 = mo.nvoid2;
    out->nvoidt = nvoidt;
    out->volt_clean = volt;
    if (marca_ext_out) from_device(c, marca_ext_out, marca, (size_t)ne3 * 4);
    c.sync();
}

}  // namespace avism
