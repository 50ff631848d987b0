// bin_kernels.cuh -- kernels of the particle binning and the batch kNN that
// several translation units launch (knn.cu, sph.cu, proposal.cu, noalloc.cu).
// Non-template kernels are static: each unit that includes this file compiles
// its own copy, so the library builds as separate units in parallel.
#pragma once

#include <cfloat>

#include "common.cuh"
#include "knn_core.cuh"
#include "knn_warp.cuh"

namespace avism {

// ---- binning -----------------------------------------------------------------
static __global__ void k_bin_keys(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                           const float *__restrict__ z, float origin, float inv_bw, int nb,
                           uint32_t *__restrict__ keys, int32_t *__restrict__ vals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int bx = bin_coord(x[i], origin, inv_bw, nb);
    const int by = bin_coord(y[i], origin, inv_bw, nb);
    const int bz = bin_coord(z[i], origin, inv_bw, nb);
    keys[i] = (uint32_t)bx + (uint32_t)nb * ((uint32_t)by + (uint32_t)nb * (uint32_t)bz);
    vals[i] = (int32_t)i;
}

// keys of quarter-bin x cells: fine x + 4 nb (y + nb z); key / 4 is the bin
static __global__ void k_bin_keys_fine(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                const float *__restrict__ z, float origin, float inv_bw, int nb,
                                uint32_t *__restrict__ keys, int32_t *__restrict__ vals) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int fx = fine_coord(x[i], origin, inv_bw, nb);
    const int by = bin_coord(y[i], origin, inv_bw, nb);
    const int bz = bin_coord(z[i], origin, inv_bw, nb);
    keys[i] = (uint32_t)fx + (uint32_t)(KNN_XF * nb) * ((uint32_t)by + (uint32_t)nb * (uint32_t)bz);
    vals[i] = (int32_t)i;
}

// offsets of the key cells [prev + 1, cur] start at i; the last particle closes the rest
template <class T>
__device__ __forceinline__ void fill_starts(T *start, int64_t i, int64_t n, int64_t prev, int64_t cur,
                                            int64_t ncells) {
    for (int64_t b = prev + 1; b <= cur; b++) start[b] = (T)i;
    if (i == n - 1)
        for (int64_t b = cur + 1; b <= ncells; b++) start[b] = (T)n;
}

// binned records (x, y, z, original index) and the bin offsets
static __global__ void k_bin_gather(int64_t n, const uint32_t *__restrict__ keys, const int32_t *__restrict__ vals,
                             const float *__restrict__ x, const float *__restrict__ y,
                             const float *__restrict__ z, float4 *__restrict__ sp,
                             int64_t *__restrict__ start, int64_t nbins) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t v = vals[i];
    sp[i] = make_float4(x[v], y[v], z[v], __int_as_float(v));
    const int64_t cur = keys[i];
    const int64_t prev = i == 0 ? -1 : (int64_t)keys[i - 1];
    for (int64_t b = prev + 1; b <= cur; b++) start[b] = i;
    if (i == n - 1)
        for (int64_t b = cur + 1; b <= nbins; b++) start[b] = n;
}

// (x, y, z, m) and (vx, vy, vz, 0) side by side as one 32-byte record per
// particle in input order: the binned gather then fetches one DRAM sector per
// particle instead of seven scattered 4-byte words
static __global__ void k_pack_particles(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                 const float *__restrict__ z, const float *__restrict__ m,
                                 const float *__restrict__ vx, const float *__restrict__ vy,
                                 const float *__restrict__ vz, float4 *__restrict__ pab) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pab[2 * i] = make_float4(x[i], y[i], z[i], m[i]);
    pab[2 * i + 1] = make_float4(vx[i], vy[i], vz[i], 0.0f);
}

// positions and masses only, for the split form (velocities still in flight)
static __global__ void k_pack_pos_mass(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                       const float *__restrict__ z, const float *__restrict__ m,
                                       float4 *__restrict__ pa) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pa[i] = make_float4(x[i], y[i], z[i], m[i]);
}
// the velocities packed in input order, then gathered into the binned records'
// (vx, vy, vz) next to the masses already there
static __global__ void k_pack_vel(int64_t n, const float *__restrict__ vx, const float *__restrict__ vy,
                                  const float *__restrict__ vz, float4 *__restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pb[i] = make_float4(vx[i], vy[i], vz[i], 0.0f);
}
static __global__ void k_gather_vel(int64_t n, const float4 *__restrict__ sp, const float4 *__restrict__ pb,
                                    float4 *__restrict__ sv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 b = pb[__float_as_int(sp[i].w)];
    sv[i] = make_float4(b.x, b.y, b.z, sv[i].w);
}

// k_bin_gather with the attributes from the packed records (pa non-null: with
// velocities, 32-byte records (pa[2v], pa[2v + 1]); without, 16-byte (x, y, z,
// m) records and the velocities left 0) and, for FINE keys, the quarter-bin
// offsets as well
template <bool FINE>
static __global__ void k_bin_gather2(int64_t n, const uint32_t *__restrict__ keys, const int32_t *__restrict__ vals,
                              const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                              const float4 *__restrict__ pa, bool with_v, float4 *__restrict__ sp,
                              float4 *__restrict__ sv, int64_t *__restrict__ start, int64_t nbins,
                              int32_t *__restrict__ fstart) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t v = vals[i];
    if (pa) {
        const float4 a = with_v ? pa[2 * (int64_t)v] : pa[v];
        const float4 b = with_v ? pa[2 * (int64_t)v + 1] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        sp[i] = make_float4(a.x, a.y, a.z, __int_as_float(v));
        sv[i] = make_float4(b.x, b.y, b.z, a.w);
    } else {
        sp[i] = make_float4(x[v], y[v], z[v], __int_as_float(v));
    }
    const int64_t cur = keys[i];
    const int64_t prev = i == 0 ? -1 : (int64_t)keys[i - 1];
    if (FINE) {
        fill_starts(fstart, i, n, prev, cur, (int64_t)KNN_XF * nbins);
        fill_starts(start, i, n, prev < 0 ? -1 : prev / KNN_XF, cur / KNN_XF, nbins);
    } else {
        fill_starts(start, i, n, prev, cur, nbins);
    }
}

static __global__ void k_empty_start(int64_t *start, int64_t nbins) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nbins) start[i] = 0;
}

// per-particle attributes in binned order: (vx, vy, vz, m)
static __global__ void k_sorted_attrs(int64_t n, const float4 *__restrict__ sp, const float *__restrict__ vx,
                               const float *__restrict__ vy, const float *__restrict__ vz,
                               const float *__restrict__ m, float4 *__restrict__ sv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = __float_as_int(sp[i].w);
    sv[i] = make_float4(vx[o], vy[o], vz[o], m[o]);
}

// ---- batch kNN (the C-ABI's avism_gpu_knn) ----------------------------------
template <int KCAP>
static __global__ void __launch_bounds__(KNN_THREADS(KCAP))
k_knn_batch(KnnGrid G, int64_t nq, const float *__restrict__ qx, const float *__restrict__ qy,
            const float *__restrict__ qz, int K, int64_t *__restrict__ idx_out,
            float *__restrict__ dist_out) {
    extern __shared__ unsigned long long knn_smem[];
    const int S = blockDim.x;
    unsigned long long *col = knn_smem + threadIdx.x;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int cnt = knn_query<KCAP>(G, qx[q], qy[q], qz[q], K, col, S);
    for (int i = 0; i < K; i++) {
        if (i < cnt) {
            const unsigned long long key = col[(size_t)i * S];
            idx_out[q * K + i] = (int64_t)key_orig(G.sp, key) + 1;
            dist_out[q * K + i] = sqrtf(__uint_as_float((uint32_t)(key >> 32)));
        } else {
            idx_out[q * K + i] = -1;
            dist_out[q * K + i] = sqrtf(FLT_MAX);     // knn_search initialises dist = HUGE(0.0)
        }
    }
}

}  // namespace avism
