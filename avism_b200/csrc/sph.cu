// sph.cu -- SPH particle-to-grid interpolation on the exact kNN engine.
//
// Replaces src/particles.f90: PPART_DENS (742-801), VVEL_INTERP_SPH_VW
// (806-929) with KERNEL_FUNC (935-963), H_DISTANCE (276-350), FILL_H_ZEROS
// (398-430) and DDENS_INTERP_SPH (434-617).  Every REAL*4 expression is
// evaluated in the reference's order (the library is built with --fmad=false);
// the reference's REAL*8 accumulators stay REAL*8.  DDENS's FP64 atomic
// scatter becomes an exact integer scatter (add_exact), order independent, so
// the grid does not depend on thread timing.
#include <cub/cub.cuh>
#include <cfloat>
#include <climits>

#include "common.cuh"
#include "knn_core.cuh"
#include "knn_warp.cuh"
#include "bin_kernels.cuh"

namespace avism {

__device__ __forceinline__ float kernel_m4(float h, float dist) {
    // KERNEL_FUNC, M4 branch: Q = DIST/(H/2)
    // H/2 as h * 0.5: both are the correctly rounded h/2, so the bits agree
    const float q = __fdiv_rn(dist, __fmul_rn(h, 0.5f));
    if (q <= 1.0f) return __fsub_rn(1.0f, __fmul_rn(__fmul_rn(1.5f, __fmul_rn(q, q)), __fsub_rn(1.0f, __fmul_rn(0.5f, q))));
    if (q <= 2.0f) {
        const float t = __fsub_rn(2.0f, q);
        return __fmul_rn(0.25f, __fmul_rn(__fmul_rn(t, t), t));
    }
    return 0.0f;
}

// KERNEL_FUNC with KERNEL_MODE = 2 (src/particles.f90:955-956): Q = DIST/(H/2),
// EXP(-Q**2).  expf is CUDA's (within 2 ulp); the Gaussian fields agree with a
// host libm to the interpolation tolerance, not bit for bit.
__device__ __forceinline__ float kernel_w(bool gauss, float h, float dist) {
    if (gauss) {
        const float q = __fdiv_rn(dist, __fmul_rn(h, 0.5f));
        return expf(-__fmul_rn(q, q));
    }
    return kernel_m4(h, dist);
}

// HPART(j) = MAX(HPART(j), d): non-negative floats order as their int bits
__device__ __forceinline__ void atomic_max_pos(float *a, float v) {
    atomicMax((int *)a, __float_as_int(v));
}

// cell (ix, jy, kz), 1-based, of thread t in a tiled traversal of the NX^3 grid
__device__ __forceinline__ bool tile_cell(int nx, int tx, int ty, int tz, int &ix, int &jy, int &kz) {
    const int ntx = (nx + tx - 1) / tx, nty = (nx + ty - 1) / ty;
    const int64_t b = blockIdx.x;
    const int bx = (int)(b % ntx), by = (int)((b / ntx) % nty), bz = (int)(b / ((int64_t)ntx * nty));
    const int t = threadIdx.x;
    ix = bx * tx + (t % tx) + 1;
    jy = by * ty + ((t / tx) % ty) + 1;
    kz = bz * tz + t / (tx * ty) + 1;
    return ix <= nx && jy <= nx && kz <= nx;
}

template <int T> struct TileDims;
template <> struct TileDims<256> { static constexpr int x = 8, y = 8, z = 4; };
template <> struct TileDims<128> { static constexpr int x = 8, y = 4, z = 4; };
template <> struct TileDims<64> { static constexpr int x = 4, y = 4, z = 4; };
template <> struct TileDims<32> { static constexpr int x = 4, y = 4, z = 2; };

// ---- PPART_DENS: rho_p = sum_k m / ((4/3) pi h_k^3) ------------------------------
template <int KCAP>
__global__ void __launch_bounds__(KNN_THREADS(KCAP))
k_ppart_dens(KnnGrid G, int64_t n, int K, const float4 *__restrict__ sv, float *__restrict__ pd_s,
             float *__restrict__ part_dens) {
    extern __shared__ unsigned long long knn_smem[];
    const int S = blockDim.x;
    unsigned long long *col = knn_smem + threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = G.sp[i];
    const int cnt = knn_any<KCAP>(G, p.x, p.y, p.z, K, col, S);
    double bas8 = 0.0;
    for (int j = 0; j < cnt; j++) bas8 = bas8 + (double)sv[key_pos(col[(size_t)j * S])].w;
    const float hk = sqrtf(key_d2(col[(size_t)(K - 1) * S]));
    const double pi = 3.141592653589793;     // DACOS(-1.D0)
    const float rho = (float)(bas8 / ((4.0 / 3.0) * pi * (double)__fmul_rn(__fmul_rn(hk, hk), hk)));
    pd_s[i] = rho;
    if (part_dens) part_dens[__float_as_int(p.w)] = rho;
}

// ---- FILL_H_ZEROS: h = k-th neighbour distance where h is still 0 -----------
template <int KCAP>
__global__ void __launch_bounds__(KNN_THREADS(KCAP))
k_fill_h(KnnGrid G, int64_t n, int K, float *__restrict__ hp_s) {
    extern __shared__ unsigned long long knn_smem[];
    const int S = blockDim.x;
    unsigned long long *col = knn_smem + threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (hp_s[i] > 0.0f) return;
    const float4 p = G.sp[i];
    knn_any<KCAP>(G, p.x, p.y, p.z, K, col, S);
    hp_s[i] = sqrtf(key_d2(col[(size_t)(K - 1) * S]));
}

// particles whose h is still 0 (FILL_H_ZEROS will search for them)
__global__ void k_count_zero(int64_t n, const float *__restrict__ h, unsigned long long *cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool z = i < n && h[i] == 0.0f;
    const unsigned b = __ballot_sync(0xffffffffu, z);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(cnt, (unsigned long long)__popc(b));
}

// binned order -> input order
__global__ void k_unbin_f32(int64_t n, const float4 *__restrict__ sp, const float *__restrict__ src,
                            float *__restrict__ dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[__float_as_int(sp[i].w)] = src[i];
}

struct CellArgs {
    int nx, rad_lo, K;
    float dx;
    const float *rad;
    const int8_t *smask;
    const float4 *sv;                 // (vx, vy, vz, m) in binned order
    const float *pd_s;                // particle density in binned order
    const float4 *svw;                // (vx, vy, vz, m / pd) in binned order (k_cells_knn_w)
    float *hp_s, *u2, *u3, *u4;       // h in binned order
    int do_vel;
    int gauss;                        // KERNEL_MODE = 2
    int32_t *ball_list;
    int32_t *ball_count;
};

// ---- VVEL_INTERP_SPH_VW / H_DISTANCE for cells whose k-th distance > DX ------
template <int KCAP>
__global__ void __launch_bounds__(KNN_THREADS(KCAP))
k_cells_knn(KnnGrid G, CellArgs A) {
    extern __shared__ unsigned long long knn_smem[];
    constexpr int T = KNN_THREADS(KCAP);
    const int S = blockDim.x;
    unsigned long long *col = knn_smem + threadIdx.x;
    int ix, jy, kz;
    if (!tile_cell(A.nx, TileDims<T>::x, TileDims<T>::y, TileDims<T>::z, ix, jy, kz)) return;
    const int64_t c = (int64_t)(ix - 1) + (int64_t)A.nx * ((int64_t)(jy - 1) + (int64_t)A.nx * (kz - 1));
    if (A.smask && A.smask[c] == 0) return;
    const float qx = A.rad[ix - A.rad_lo], qy = A.rad[jy - A.rad_lo], qz = A.rad[kz - A.rad_lo];
    const int K = A.K;
    const int cnt = knn_any<KCAP>(G, qx, qy, qz, K, col, S);
    const float hk = sqrtf(key_d2(col[(size_t)(cnt - 1) * S]));
    if (!(hk > A.dx)) {                       // ball_search(TREE, TAR, DX) branch
        const int slot = atomicAdd(A.ball_count, 1);
        A.ball_list[slot] = (int32_t)c;
        return;
    }
    for (int i = 0; i < cnt; i++) {
        const unsigned long long key = col[(size_t)i * S];
        atomic_max_pos(&A.hp_s[key_pos(key)], sqrtf(key_d2(key)));
    }
    if (!A.do_vel) return;
    double b = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
    for (int i = 0; i < cnt; i++) {
        const unsigned long long key = col[(size_t)i * S];
        const uint32_t j = key_pos(key);
        const float4 a = A.sv[j];
        float w = kernel_w(A.gauss, hk, sqrtf(key_d2(key)));
        w = __fmul_rn(w, __fdiv_rn(a.w, A.pd_s[j]));
        const double w8 = (double)w;
        b = b + w8;
        bx = bx + w8 * (double)a.x;
        by = by + w8 * (double)a.y;
        bz = bz + w8 * (double)a.z;
    }
    A.u2[c] = (float)(bx / b);
    A.u3[c] = (float)(by / b);
    A.u4[c] = (float)(bz / b);
}

// ---- cells in the ball branch: all particles within DX (src/particles.f90:868-878)
// ball_search returns the ball sorted by distance (src/kdtree.f90:1015-1212), and
// the velocity sums run over it in that order.  Here the members of every ball
// cell are listed with 64-bit keys (squared-distance bits above the particle
// index, the tie rule), sorted per cell, and summed in that order:
//   k_ball_scan (count, h = max distance, K-th distance) -> scan of the counts
//   -> k_ball_fill (keys, binned positions) -> segmented sort -> k_ball_sum.
template <class F>
__device__ __forceinline__ void ball_walk(const KnnGrid &G, const CellArgs &A, int64_t c, F &&f) {
    const int nx = A.nx;
    const int ix = (int)(c % nx) + 1, jy = (int)((c / nx) % nx) + 1, kz = (int)(c / ((int64_t)nx * nx)) + 1;
    const float q[3] = {A.rad[ix - A.rad_lo], A.rad[jy - A.rad_lo], A.rad[kz - A.rad_lo]};
    const float r2 = __fmul_rn(A.dx, A.dx);                   // radius**2 in REAL*4
    const int b[3] = {bin_coord(q[0], G.origin, G.inv_bw, G.nb), bin_coord(q[1], G.origin, G.inv_bw, G.nb),
                      bin_coord(q[2], G.origin, G.inv_bw, G.nb)};
    const int sb = (int)ceilf(A.dx * G.inv_bw) + 1;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) axis_window(G, b[a], sb, lo[a], hi[a]);
    for (int dz = lo[2]; dz <= hi[2]; dz++) {
        const int bz_ = G.periodic ? wrap_bin(b[2] + dz, G.nb) : b[2] + dz;
        for (int dy = lo[1]; dy <= hi[1]; dy++) {
            const int by_ = G.periodic ? wrap_bin(b[1] + dy, G.nb) : b[1] + dy;
            for (int dx = lo[0]; dx <= hi[0]; dx++) {
                const int bx_ = G.periodic ? wrap_bin(b[0] + dx, G.nb) : b[0] + dx;
                const int bin = bx_ + G.nb * (by_ + G.nb * bz_);
                for (int64_t p = G.start[bin]; p < G.start[bin + 1]; p++) {
                    const float4 v = G.sp[p];
                    const float d2 = dist2_ref(v.x, v.y, v.z, q[0], q[1], q[2], G.box, G.periodic);
                    if (d2 <= r2) f(p, v, d2);
                }
            }
        }
    }
}

// members per ball cell, h = MAX(h, d) of every member, the largest distance
__global__ void k_ball_scan(KnnGrid G, CellArgs A, int32_t nlist, int32_t *__restrict__ cnt,
                            float *__restrict__ dmax) {
    const int32_t t = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= nlist) return;
    int32_t m = 0;
    float dm2 = -1.0f;
    ball_walk(G, A, A.ball_list[t], [&](int64_t p, const float4 &, float d2) {
        m++;
        dm2 = fmaxf(dm2, d2);
        atomic_max_pos(&A.hp_s[p], sqrtf(d2));
    });
    cnt[t] = m;
    dmax[t] = sqrtf(dm2);
}

__global__ void k_ball_fill(KnnGrid G, CellArgs A, int32_t nlist, const int64_t *__restrict__ off,
                            unsigned long long *__restrict__ keys, int32_t *__restrict__ pos) {
    const int32_t t = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= nlist) return;
    int64_t o = off[t];
    ball_walk(G, A, A.ball_list[t], [&](int64_t p, const float4 &v, float d2) {
        keys[o] = ((unsigned long long)__float_as_uint(d2) << 32) | (uint32_t)__float_as_int(v.w);
        pos[o] = (int32_t)p;
        o++;
    });
}

// the velocity sums over each ball in (distance, particle index) order, REAL*8
__global__ void k_ball_sum(CellArgs A, int32_t nlist, const int64_t *__restrict__ off,
                           const unsigned long long *__restrict__ keys, const int32_t *__restrict__ pos,
                           const float *__restrict__ dmax) {
    const int32_t t = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= nlist) return;
    const int64_t c = A.ball_list[t];
    const float hk = dmax[t];
    double bs = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
    for (int64_t o = off[t]; o < off[t + 1]; o++) {
        const int32_t p = pos[o];
        const float4 a = A.sv[p];
        float w = kernel_w(A.gauss, hk, sqrtf(__uint_as_float((uint32_t)(keys[o] >> 32))));
        w = __fmul_rn(w, __fdiv_rn(a.w, A.pd_s[p]));
        const double w8 = (double)w;
        bs = bs + w8;
        bx = bx + w8 * (double)a.x;
        by = by + w8 * (double)a.y;
        bz = bz + w8 * (double)a.z;
    }
    A.u2[c] = (float)(bx / bs);
    A.u3[c] = (float)(by / bs);
    A.u4[c] = (float)(bz / bs);
}

static void cells_ball(Ctx &c, const KnnGrid &G, const CellArgs &A, int32_t nball) {
    if (nball <= 0) return;
    int32_t *cnt = c.get_t<int32_t>(B_LIST_A, (size_t)nball + 1);
    float *dmax = c.get_t<float>(B_LIST_B, (size_t)nball);
    int64_t *off = c.get_t<int64_t>(B_SEG_A, (size_t)nball + 1);
    ++c.launches, k_ball_scan<<<grid_for(nball, 128), 128, 0, c.stream>>>(G, A, nball, cnt, dmax);
    AV_CUDA(cudaGetLastError());
    if (!A.do_vel) return;
    AV_CUDA(cudaMemsetAsync(cnt + nball, 0, sizeof(int32_t), c.stream));
    size_t tmp = 0;
    AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, off, nball + 1, c.stream));
    AV_CUDA(cub::DeviceScan::ExclusiveSum(c.get(B_CUB_TMP, tmp), tmp, cnt, off, nball + 1, c.stream));
    int64_t total = 0;
    AV_CUDA(cudaMemcpyAsync(&total, off + nball, sizeof total, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    AV_CHECK(total < (int64_t)INT32_MAX, AVISM_ERR_UNSUPPORTED, "ball fallback: more than 2^31 members");
    const int64_t m = std::max<int64_t>(total, 1);
    unsigned long long *ka = c.get_t<unsigned long long>(B_SORT_KEY, 2 * (size_t)m);
    int32_t *pa = c.get_t<int32_t>(B_SORT_IDX, 2 * (size_t)m);
    ++c.launches, k_ball_fill<<<grid_for(nball, 128), 128, 0, c.stream>>>(G, A, nball, off, ka, pa);
    AV_CUDA(cudaGetLastError());
    cub::DoubleBuffer<unsigned long long> dk(ka, ka + m);
    cub::DoubleBuffer<int32_t> dv(pa, pa + m);
    tmp = 0;
    AV_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tmp, dk, dv, (int)total, nball, off, off + 1, c.stream));
    AV_CUDA(cub::DeviceSegmentedSort::SortPairs(c.get(B_CUB_TMP, tmp), tmp, dk, dv, (int)total, nball, off,
                                                off + 1, c.stream));
    ++c.launches, k_ball_sum<<<grid_for(nball, 128), 128, 0, c.stream>>>(A, nball, off, dk.Current(),
                                                                          dv.Current(), dmax);
    AV_CUDA(cudaGetLastError());
}

// ---- warp-per-query forms of PPART_DENS and VVEL_INTERP_SPH_VW / H_DISTANCE ----
// Each warp answers SPH_QPW consecutive queries with knn_warp_exact; the sums
// over the neighbour list stay sequential in list order (REAL*8, as the
// reference's loops), done by one lane per sum from shared memory.
constexpr int SPH_WARPS = 8, SPH_QPW = 4;
constexpr int PP_QPW = 8;                      // particle queries per warp (their sums run side by side)

__device__ __forceinline__ float query_r0(const KnnGrid &G, float qx, float qy, float qz) {
    if (!G.r0) return 0.0f;
    const int b = bin_coord(qx, G.origin, G.inv_bw, G.nb) +
                  G.nb * (bin_coord(qy, G.origin, G.inv_bw, G.nb) + G.nb * bin_coord(qz, G.origin, G.inv_bw, G.nb));
    return G.r0[b];
}

// rows of staged sums: (KMAX + 2) doubles or (KMAX + 4) floats keep the
// summing lanes' 16-byte loads on distinct banks
template <int KMAX> constexpr int SPH_ROW = KMAX + 2;
template <int KMAX> constexpr int SPH_ROWF = KMAX + 4;
// the particle kernel stages its queries' neighbour masses (f32, as stored) per
// warp and sums them after the searches, one lane per query
template <int KMAX>
constexpr size_t sph_smem_bytes() {
    return (size_t)SPH_WARPS * sizeof(WarpKnnSmem<KMAX>) +
           (size_t)SPH_WARPS * PP_QPW * SPH_ROWF<KMAX> * sizeof(float);
}
template <int KMAX>
__device__ __forceinline__ float *sph_rows(unsigned char *smem, int warp) {
    return reinterpret_cast<float *>(smem + SPH_WARPS * sizeof(WarpKnnSmem<KMAX>)) +
           (size_t)warp * PP_QPW * SPH_ROWF<KMAX>;
}
// sequential REAL*8 sum of row[0..n) in order, two values per 16-byte load
__device__ __forceinline__ double seq_sum(const double *row, int n) {
    const double2 *r2 = reinterpret_cast<const double2 *>(row);
    double s = 0.0;
    int j = 0;
    for (; j + 2 <= n; j += 2) {
        const double2 v = r2[j >> 1];
        s = s + v.x;
        s = s + v.y;
    }
    if (j < n) s = s + row[j];
    return s;
}
// the same REAL*8 sum of f32 values, four per 16-byte load
__device__ __forceinline__ double seq_sum(const float *row, int n) {
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
    double s = 0.0;
    int j = 0;
    for (; j + 4 <= n; j += 4) {
        const float4 v = r4[j >> 2];
        s = s + (double)v.x;
        s = s + (double)v.y;
        s = s + (double)v.z;
        s = s + (double)v.w;
    }
    for (; j < n; j++) s = s + (double)row[j];
    return s;
}

// five blocks per SM (48 registers, a few spills): more warps in flight pay
// for the spills (171 against 187 ms with four blocks at 512^3)
template <int KMAX, bool STATS>
__global__ void __launch_bounds__(SPH_WARPS * 32, 5)
k_ppart_dens_w(KnnGrid G, int64_t n, int K, const float4 *__restrict__ sv, float *__restrict__ pd_s,
               float *__restrict__ part_dens) {
    extern __shared__ __align__(16) unsigned char wq_smem[];
    const int warp = threadIdx.x >> 5;
    WarpKnnSmem<KMAX> &S = reinterpret_cast<WarpKnnSmem<KMAX> *>(wq_smem)[warp];
    float *acc = sph_rows<KMAX>(wq_smem, warp);               // one row of masses per query
    const int lane = threadIdx.x & 31;
    const int64_t i0 = ((int64_t)blockIdx.x * SPH_WARPS + warp) * PP_QPW;
    int my_cnt = 0;                                           // lane t: query t's count and h
    float my_hk = 0.0f;
    for (int t = 0; t < PP_QPW; t++) {
        const int64_t i = i0 + t;
        if (i >= n) break;
        const float4 p = G.sp[i];
        const int cnt = knn_warp_exact<KMAX, STATS>(G, p.x, p.y, p.z, K, query_r0(G, p.x, p.y, p.z), S,
                                             reinterpret_cast<unsigned long long *>(S.d2));
        for (int j = lane; j < cnt; j += 32) acc[t * SPH_ROWF<KMAX> + j] = sv[S.res_pos[j]].w;
        const float hk = sqrtf(__uint_as_float(S.res_d2[K - 1]));
        if (lane == t) {
            my_cnt = cnt;
            my_hk = hk;
        }
    }
    __syncwarp();
    // the queries' sums side by side, one lane each
    const int64_t i = i0 + lane;
    if (lane < PP_QPW && i < n) {
        const double bas8 = seq_sum(acc + lane * SPH_ROWF<KMAX>, my_cnt);
        const double pi = 3.141592653589793;     // DACOS(-1.D0)
        const float rho = (float)(bas8 / ((4.0 / 3.0) * pi * (double)__fmul_rn(__fmul_rn(my_hk, my_hk), my_hk)));
        pd_s[i] = rho;
        if (part_dens) part_dens[__float_as_int(G.sp[i].w)] = rho;
    }
}

// the records the cell kernel reads per neighbour: velocities and m / PPART_DENS
// (the quotient of VVEL_INTERP_SPH_VW's weight, once per particle)
__global__ void k_mass_over_dens(int64_t n, const float4 *__restrict__ sv, const float *__restrict__ pd_s,
                                 float4 *__restrict__ svw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = sv[i];
    svw[i] = make_float4(a.x, a.y, a.z, __fdiv_rn(a.w, pd_s[i]));
}

// five blocks per SM (48 registers): the cell kernel gains more from the extra
// warps than it loses to spills (six blocks at 40 registers spill too much)
template <int KMAX, bool STATS>
__global__ void __launch_bounds__(SPH_WARPS * 32, 5)
k_cells_knn_w(KnnGrid G, CellArgs A) {
    extern __shared__ __align__(16) unsigned char wq_smem[];
    WarpKnnSmem<KMAX> &S = reinterpret_cast<WarpKnnSmem<KMAX> *>(wq_smem)[threadIdx.x >> 5];
    // 4 rows of SPH_ROW doubles (b, bx, by, bz) over d2, pos and the segment
    // lists, which are free after the select (res_* lie beyond them)
    static_assert(4 * SPH_ROW<KMAX> * sizeof(double) <= offsetof(WarpKnnSmem<KMAX>, res_d2), "rows overlap res_d2");
    double *acc = reinterpret_cast<double *>(S.d2);
    const int lane = threadIdx.x & 31;
    const int nx = A.nx;
    // 4x4x2 tiles of cells, one tile per block, SPH_QPW cells per warp
    const int ntx = (nx + 3) / 4, nty = (nx + 3) / 4;
    const int64_t tile = blockIdx.x;
    const int tx = (int)(tile % ntx), ty = (int)((tile / ntx) % nty), tz = (int)(tile / ((int64_t)ntx * nty));
    for (int t = 0; t < SPH_QPW; t++) {
        const int q = (threadIdx.x >> 5) * SPH_QPW + t;        // 0..31 inside the tile
        const int ix = tx * 4 + (q & 3) + 1, jy = ty * 4 + ((q >> 2) & 3) + 1, kz = tz * 2 + (q >> 4) + 1;
        if (ix > nx || jy > nx || kz > nx) continue;
        const int64_t c = (int64_t)(ix - 1) + (int64_t)nx * ((int64_t)(jy - 1) + (int64_t)nx * (kz - 1));
        if (A.smask && A.smask[c] == 0) continue;
        const float qx = A.rad[ix - A.rad_lo], qy = A.rad[jy - A.rad_lo], qz = A.rad[kz - A.rad_lo];
        const int K = A.K;
        const int cnt = knn_warp_exact<KMAX, STATS>(G, qx, qy, qz, K, query_r0(G, qx, qy, qz), S,
                                             reinterpret_cast<unsigned long long *>(S.d2));
        const float hk = sqrtf(__uint_as_float(S.res_d2[cnt - 1]));
        if (!(hk > A.dx)) {                       // ball_search(TREE, TAR, DX) branch
            if (lane == 0) {
                const int slot = atomicAdd(A.ball_count, 1);
                A.ball_list[slot] = (int32_t)c;
            }
            continue;
        }
        // HPART(j) = MAX(HPART(j), d), then the weight W(d, H) * m / PPART_DENS
        // (m / PPART_DENS per particle from k_mass_over_dens: the same quotient)
        for (int j = lane; j < cnt; j += 32) {
            const uint32_t pj = S.res_pos[j];
            const float d = sqrtf(__uint_as_float(S.res_d2[j]));
            atomic_max_pos(&A.hp_s[pj], d);
            if (!A.do_vel) continue;
            const float4 a = A.svw[pj];
            const float w = __fmul_rn(kernel_w(A.gauss, hk, d), a.w);
            const double w8 = (double)w;
            acc[j] = w8;
            acc[SPH_ROW<KMAX> + j] = w8 * (double)a.x;
            acc[2 * SPH_ROW<KMAX> + j] = w8 * (double)a.y;
            acc[3 * SPH_ROW<KMAX> + j] = w8 * (double)a.z;
        }
        if (!A.do_vel) continue;
        __syncwarp();
        double sum = 0.0;
        if (lane < 4) sum = seq_sum(acc + lane * SPH_ROW<KMAX>, cnt);
        const double b = __shfl_sync(0xffffffffu, sum, 0);
        if (lane == 1) A.u2[c] = (float)(sum / b);
        if (lane == 2) A.u3[c] = (float)(sum / b);
        if (lane == 3) A.u4[c] = (float)(sum / b);
    }
}

// ---- DDENS_INTERP_SPH: per-particle NORM in the reference's loop order, then
//      an exact scatter of m*w/NORM ----------------------------------------------
struct DdensArgs {
    int nx, rad_lo;
    float dx, rx1;
    const float *rad;
    const float *hp_s;            // h in binned order
    const float4 *sv;             // (vx, vy, vz, m) in binned order
    unsigned long long *fix;      // nlimb counters per cell (exact sums, add_exact)
    int nlimb;
    unsigned long long *norm0;    // counter of NORM = 0 particles, or null
    int gauss;                    // KERNEL_MODE = 2
};

// Exact REAL*4 sums.  Every finite f32 value is an integer multiple of 2^-149,
// so a cell's sum is kept exactly as an integer in units of 2^-149, split in
// 32-bit limbs; limb i accumulates in the cell's 64-bit counter i.  A term's
// 24-bit significand, shifted to its place, spans at most two limbs, added as
// two fire-and-forget reductions; a counter cannot overflow for fewer than 2^32
// additions per cell.  The carries between limbs are resolved once, when the
// cell is read (k_exact_to_f32).  The sum is independent of the order of the
// additions, unlike the reference's REAL*8 atomics, and as fine as REAL*4 allows
// at every magnitude (masses over many decades lose nothing).
__device__ __forceinline__ void add_exact(unsigned long long *cell, float v) {
    const uint32_t b = __float_as_uint(v);            // v >= 0
    if (b == 0) return;
    const uint32_t e = b >> 23;
    const uint32_t mant = (b & 0x7fffffu) | (e ? 0x800000u : 0u);
    const uint32_t pos = e ? e - 1 : 0;               // place of the significand's lowest bit
    const unsigned long long w = (unsigned long long)mant << (pos & 31);
    unsigned long long *c = cell + (pos >> 5);
    atomicAdd(c, w & 0xffffffffULL);
    if (w >> 32) atomicAdd(c + 1, w >> 32);
}

// DDENS weight: M4 of Q = SQRT(D2) * INV_H, or with KERNEL_MODE = 2 the Gaussian
// EXP(-D2 * INV_H_SQ), INV_H_SQ = INV_H * INV_H (src/particles.f90:522-538)
__device__ __forceinline__ float m4_q(float d2, float inv_h);
__device__ __forceinline__ float kernel_q(bool gauss, float d2, float inv_h) {
    if (gauss) return expf(-__fmul_rn(d2, __fmul_rn(inv_h, inv_h)));
    return m4_q(d2, inv_h);
}

__device__ __forceinline__ float m4_q(float d2, float inv_h) {
    const float q = __fmul_rn(sqrtf(d2), inv_h);
    if (q <= 1.0f) return __fsub_rn(1.0f, __fmul_rn(__fmul_rn(1.5f, __fmul_rn(q, q)), __fsub_rn(1.0f, __fmul_rn(0.5f, q))));
    if (q <= 2.0f) {
        const float t = __fsub_rn(2.0f, q);
        return __fmul_rn(0.25f, __fmul_rn(__fmul_rn(t, t), t));
    }
    return 0.0f;
}

// one particle with nested row loops (both passes): particles whose support
// has more rows than k_ddens holds, or offsets beyond 8 bits
__device__ __noinline__ void ddens_nested(const DdensArgs &A, const float4 p, int64_t i) {
    const int nx = A.nx;
    const float dx = A.dx;
    const int ix = (int)__fdiv_rn(__fsub_rn(p.x, A.rx1), dx) + 1;
    const int jy = (int)__fdiv_rn(__fsub_rn(p.y, A.rx1), dx) + 1;
    const int kz = (int)__fdiv_rn(__fsub_rn(p.z, A.rx1), dx) + 1;
    const float h = A.hp_s[i];
    const float inv_h = __fdiv_rn(2.0f, h);
    const float h2max = __fmul_rn(__fmul_rn(4.0f, h), h);
    const int inc = (int)__fadd_rn(__fdiv_rn(__fmul_rn(2.0f, h), dx), 0.5f);
    // M4: only cells with Q <= 2 (d <= h) carry weight; rows and planes beyond h
    // are skipped.  Gaussian: every cell with D2 <= H2_MAX (d <= 2h) does.
    const float hh = (A.gauss ? h2max : h * h) * 1.00002f + 1e-30f;
    const float inv_dx = 1.0f / dx;
    const float *rad = A.rad - A.rad_lo;
    const float m = A.sv[i].w;
    const int k_lo = max(kz - inc, 1), k_hi = min(kz + inc, nx);
    const int j_lo = max(jy - inc, 1), j_hi = min(jy + inc, nx);
    const int i_lo = max(ix - inc, 1), i_hi = min(ix + inc, nx);
    // planes and rows that can meet the support, straight from its radius (one
    // spare cell each side, as for the x range); everything else has weight 0
    const float hr = (hh > 0.0f ? hh * rsqrtf(hh) : 0.0f) * 1.00001f + 1e-6f * dx;
    int k_a = max(k_lo, (int)floorf((p.z - hr - A.rx1) * inv_dx) + 1 - 1);
    int k_b = min(k_hi, (int)ceilf((p.z + hr - A.rx1) * inv_dx) + 1 + 1);
    // trim the spare planes: the support is convex and RADX monotone, so only
    // the ends can lie outside it (dz^2 > hh, weight 0 everywhere)
    auto dz2_of = [&](int k2) { const float t = __fsub_rn(p.z, rad[k2]); return __fmul_rn(t, t); };
    while (k_a <= k_b && dz2_of(k_a) > hh) k_a++;
    while (k_b >= k_a && dz2_of(k_b) > hh) k_b--;
    float norm = 0.0f;
    for (int pass = 0; pass < 2; pass++) {
        for (int k2 = k_a; k2 <= k_b; k2++) {
            const float dz2 = dz2_of(k2);
            const float remz = hh - dz2;
            const float ry = (remz > 0.0f ? remz * rsqrtf(remz) : 0.0f) * 1.00001f + 1e-6f * dx;
            int j_a = max(j_lo, (int)floorf((p.y - ry - A.rx1) * inv_dx) + 1 - 1);
            int j_b = min(j_hi, (int)ceilf((p.y + ry - A.rx1) * inv_dx) + 1 + 1);
            auto rem_of = [&](int j2) { const float t = __fsub_rn(p.y, rad[j2]); return hh - dz2 - __fmul_rn(t, t); };
            while (j_a <= j_b && rem_of(j_a) < 0.0f) j_a++;
            while (j_b >= j_a && rem_of(j_b) < 0.0f) j_b--;
            for (int j2 = j_a; j2 <= j_b; j2++) {
                const float ty = __fsub_rn(p.y, rad[j2]);
                const float dy2 = __fmul_rn(ty, ty);
                const float rem = hh - dz2 - dy2;
                // conservative x range (one spare cell each side absorbs the rounding
                // of the approximate root and of the reciprocal), then trimmed to the
                // cells inside the support: d^2 <= hh (beyond it the weight is exactly 0)
                const float R = (rem > 0.0f ? rem * rsqrtf(rem) : 0.0f) * 1.00001f + 1e-6f * dx;
                int a = max(i_lo, (int)floorf((p.x - R - A.rx1) * inv_dx) + 1 - 1);
                int e = min(i_hi, (int)ceilf((p.x + R - A.rx1) * inv_dx) + 1 + 1);
                auto d2_of = [&](int i2) {
                    const float t = __fsub_rn(p.x, rad[i2]);
                    return __fadd_rn(__fadd_rn(__fmul_rn(t, t), dy2), dz2);
                };
                while (a <= e && d2_of(a) > hh) a++;
                while (e >= a && d2_of(e) > hh) e--;
                for (int i2 = a; i2 <= e; i2++) {
                    const float d2 = d2_of(i2);
                    if (d2 > h2max) continue;            // SKIP CUBE CORNERS (M4: never, as hh < h2max)
                    const float w = kernel_q(A.gauss, d2, inv_h);
                    if (pass == 0) {
                        norm = __fadd_rn(norm, w);
                    } else if (w != 0.0f) {
                        const float contrib = __fdiv_rn(__fmul_rn(w, m), norm);
                        const int64_t cid = (int64_t)(i2 - 1) + (int64_t)nx * ((int64_t)(j2 - 1) + (int64_t)nx * (k2 - 1));
                        add_exact(A.fix + (int64_t)A.nlimb * cid, contrib);
                    }
                }
            }
        }
        if (pass == 0 && norm == 0.0f) {
            // the particle only contributes to its own cell
            if (ix >= 1 && ix <= nx && jy >= 1 && jy <= nx && kz >= 1 && kz <= nx) {
                const int64_t cid = (int64_t)(ix - 1) + (int64_t)nx * ((int64_t)(jy - 1) + (int64_t)nx * (kz - 1));
                add_exact(A.fix + (int64_t)A.nlimb * cid, m);
            }
            break;
        }
    }
}


// DDENS_INTERP_SPH, one thread per particle.  The rows of the particle's support
// (planes and rows trimmed to d^2 <= hh, x ranges trimmed likewise) are listed
// once in shared memory, packed (k - k_lo, j - j_lo, a - i_lo, length) in 8 bits
// each; both passes then walk the cells as one flat loop, so the lanes of a warp
// stay busy until the largest support is done instead of idling at the end of
// every plane and row.  NORM still sums in the reference's (k, j, i) order.
// 28 rows per thread (28 KB per block) and six blocks per SM at 40 registers:
// occupancy pays more than the particles whose longer lists go to ddens_nested
constexpr int DD_THREADS = 256, DD_RMAX = 28;

// order: the particles (binned positions) in the order the threads take them, or
// null for the binned order itself
__global__ void __launch_bounds__(DD_THREADS, 6) k_ddens(KnnGrid G, int64_t n, DdensArgs A,
                                                        const int32_t *__restrict__ order) {
    __shared__ uint32_t rows[DD_RMAX * DD_THREADS];
    uint32_t *my = rows + threadIdx.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t i = order ? (int64_t)order[t] : t;
    const float4 p = G.sp[i];
    const int nx = A.nx;
    const float dx = A.dx;
    const int ix = (int)__fdiv_rn(__fsub_rn(p.x, A.rx1), dx) + 1;
    const int jy = (int)__fdiv_rn(__fsub_rn(p.y, A.rx1), dx) + 1;
    const int kz = (int)__fdiv_rn(__fsub_rn(p.z, A.rx1), dx) + 1;
    const float h = A.hp_s[i];
    const float inv_h = __fdiv_rn(2.0f, h);
    const int inc = (int)__fadd_rn(__fdiv_rn(__fmul_rn(2.0f, h), dx), 0.5f);
    const float h2max = __fmul_rn(__fmul_rn(4.0f, h), h);
    const float hh = (A.gauss ? h2max : h * h) * 1.00002f + 1e-30f;
    const float inv_dx = 1.0f / dx;
    const float *rad = A.rad - A.rad_lo;
    const int k_lo = max(kz - inc, 1), k_hi = min(kz + inc, nx);
    const int j_lo = max(jy - inc, 1), j_hi = min(jy + inc, nx);
    const int i_lo = max(ix - inc, 1), i_hi = min(ix + inc, nx);
    const float hr = (hh > 0.0f ? hh * rsqrtf(hh) : 0.0f) * 1.00001f + 1e-6f * dx;
    int k_a = max(k_lo, (int)floorf((p.z - hr - A.rx1) * inv_dx) + 1 - 1);
    int k_b = min(k_hi, (int)ceilf((p.z + hr - A.rx1) * inv_dx) + 1 + 1);
    auto dz2_of = [&](int k2) { const float t = __fsub_rn(p.z, rad[k2]); return __fmul_rn(t, t); };
    while (k_a <= k_b && dz2_of(k_a) > hh) k_a++;
    while (k_b >= k_a && dz2_of(k_b) > hh) k_b--;
    // the support's rows, as ddens_nested walks them
    int nrows = 0, ncell = 0;
    bool over = false;
    for (int k2 = k_a; k2 <= k_b && !over; k2++) {
        const float dz2 = dz2_of(k2);
        const float remz = hh - dz2;
        const float ry = (remz > 0.0f ? remz * rsqrtf(remz) : 0.0f) * 1.00001f + 1e-6f * dx;
        int j_a = max(j_lo, (int)floorf((p.y - ry - A.rx1) * inv_dx) + 1 - 1);
        int j_b = min(j_hi, (int)ceilf((p.y + ry - A.rx1) * inv_dx) + 1 + 1);
        auto rem_of = [&](int j2) { const float t = __fsub_rn(p.y, rad[j2]); return hh - dz2 - __fmul_rn(t, t); };
        while (j_a <= j_b && rem_of(j_a) < 0.0f) j_a++;
        while (j_b >= j_a && rem_of(j_b) < 0.0f) j_b--;
        for (int j2 = j_a; j2 <= j_b; j2++) {
            const float ty = __fsub_rn(p.y, rad[j2]);
            const float dy2 = __fmul_rn(ty, ty);
            const float rem = hh - dz2 - dy2;
            const float R = (rem > 0.0f ? rem * rsqrtf(rem) : 0.0f) * 1.00001f + 1e-6f * dx;
            int a = max(i_lo, (int)floorf((p.x - R - A.rx1) * inv_dx) + 1 - 1);
            int e = min(i_hi, (int)ceilf((p.x + R - A.rx1) * inv_dx) + 1 + 1);
            auto d2_of = [&](int i2) {
                const float t = __fsub_rn(p.x, rad[i2]);
                return __fadd_rn(__fadd_rn(__fmul_rn(t, t), dy2), dz2);
            };
            while (a <= e && d2_of(a) > hh) a++;
            while (e >= a && d2_of(e) > hh) e--;
            if (a > e) continue;
            const int len = e - a + 1;
            if (nrows == DD_RMAX || k2 - k_lo > 255 || j2 - j_lo > 255 || a - i_lo > 255 || len > 255) {
                over = true;
                break;
            }
            my[nrows * DD_THREADS] = (uint32_t)(k2 - k_lo) | (uint32_t)(j2 - j_lo) << 8 |
                                     (uint32_t)(a - i_lo) << 16 | (uint32_t)len << 24;
            nrows++;
            ncell += len;
        }
    }
    if (over) {
        ddens_nested(A, p, i);
        return;
    }
    int k2 = 0, j2 = 0, i2 = 0, ie = -1;
    float dy2 = 0.0f, dz2 = 0.0f;
    auto load_row = [&](int r) {
        const uint32_t d = my[r * DD_THREADS];
        k2 = k_lo + (int)(d & 255u);
        j2 = j_lo + (int)((d >> 8) & 255u);
        i2 = i_lo + (int)((d >> 16) & 255u);
        ie = i2 + (int)(d >> 24) - 1;
        dz2 = dz2_of(k2);
        const float ty = __fsub_rn(p.y, rad[j2]);
        dy2 = __fmul_rn(ty, ty);
    };
    // pass 0: NORM (cells outside the support add exactly 0 in the reference)
    float norm = 0.0f;
    if (ncell > 0) {
        int r = 0;
        load_row(0);
        for (int t = 0; t < ncell; t++) {
            const float tx = __fsub_rn(p.x, rad[i2]);
            const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(tx, tx), dy2), dz2);
            // listed cells beyond H2_MAX (Gaussian only: M4 lists none) add nothing
            if (!(A.gauss && d2 > h2max)) norm = __fadd_rn(norm, kernel_q(A.gauss, d2, inv_h));
            if (++i2 > ie && t + 1 < ncell) load_row(++r);
        }
    }
    const float m = A.sv[i].w;
    if (norm == 0.0f) {
        if (A.norm0) atomicAdd(A.norm0, 1ull);
        // the particle only contributes to its own cell
        if (ix >= 1 && ix <= nx && jy >= 1 && jy <= nx && kz >= 1 && kz <= nx) {
            const int64_t cid = (int64_t)(ix - 1) + (int64_t)nx * ((int64_t)(jy - 1) + (int64_t)nx * (kz - 1));
            add_exact(A.fix + (int64_t)A.nlimb * cid, m);
        }
        return;
    }
    // pass 1: m * w / NORM, exact sums per cell
    int r = 0;
    load_row(0);
    int64_t rowc = (int64_t)nx * ((int64_t)(j2 - 1) + (int64_t)nx * (k2 - 1)) - 1;
    for (int t = 0; t < ncell; t++) {
        const float tx = __fsub_rn(p.x, rad[i2]);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(tx, tx), dy2), dz2);
        const float w = (A.gauss && d2 > h2max) ? 0.0f : kernel_q(A.gauss, d2, inv_h);
        if (w != 0.0f) {
            const float contrib = __fdiv_rn(__fmul_rn(w, m), norm);
            add_exact(A.fix + (int64_t)A.nlimb * (rowc + i2), contrib);
        }
        if (++i2 > ie && t + 1 < ncell) {
            load_row(++r);
            rowc = (int64_t)nx * ((int64_t)(j2 - 1) + (int64_t)nx * (k2 - 1)) - 1;
        }
    }
}

// A cell's exact sum, rounded to REAL*8 (nearest, ties to even) and then to
// REAL*4, as the reference's U(...) = U8(...) conversion of its REAL*8 sum.
constexpr int EXACT_MAX_LIMBS = 11;

// the support class of every particle for the scatter's thread order: larger
// smoothing lengths first, in steps of a quarter cell (the scatter's sums are
// exact, so the order leaves the grid unchanged; it only gives the threads of a
// warp supports of similar size)
constexpr int DD_CLASSES = 32;
__global__ void k_ddens_class(int64_t n, const float *__restrict__ hp_s, float inv_dx, uint32_t *__restrict__ key,
                              int32_t *__restrict__ val) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float q = hp_s[i] * inv_dx * 4.0f;
    const int c = q < (float)(DD_CLASSES - 1) ? (int)q : DD_CLASSES - 1;
    key[i] = (uint32_t)(DD_CLASSES - 1 - c);
    val[i] = (int32_t)i;
}

__global__ void k_exact_to_f32(int64_t nc, const unsigned long long *__restrict__ fix, int nlimb,
                               float *__restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    uint32_t limb[EXACT_MAX_LIMBS + 1];
    unsigned long long carry = 0;
    int top = -1;
#pragma unroll
    for (int i = 0; i < EXACT_MAX_LIMBS; i++) {
        if (i < nlimb) {
            const unsigned long long v = fix[(int64_t)nlimb * c + i] + carry;   // < 2^64: counters < 2^63
            limb[i] = (uint32_t)v;
            carry = v >> 32;
        } else {
            limb[i] = (uint32_t)carry;
            carry = 0;
        }
        if (limb[i]) top = i;
    }
    if (top < 0) { out[c] = 0.0f; return; }
    // the top three limbs as one integer x; the limbs below only matter as a sticky bit
    const int base = top >= 2 ? top - 2 : 0;
    unsigned __int128 x = 0;
    for (int i = top; i >= base; i--) x = (x << 32) | limb[i];
    bool sticky = false;
    for (int i = 0; i < base; i++) sticky |= limb[i] != 0;
    const unsigned long long xh = (unsigned long long)(x >> 64), xl = (unsigned long long)x;
    const int nbits = xh ? 128 - __clzll(xh) : 64 - __clzll(xl);
    double d;
    if (nbits <= 53) {
        d = ldexp((double)xl, 32 * base - 149);           // exact (no limbs below: base = 0)
    } else {
        const int sh = nbits - 53;
        unsigned long long m = (unsigned long long)(x >> sh);
        const unsigned __int128 rem = x & (((unsigned __int128)1 << sh) - 1);
        const unsigned __int128 half = (unsigned __int128)1 << (sh - 1);
        const bool up = rem > half || (rem == half && (sticky || (m & 1)));
        int e = sh;
        if (up && ++m == (1ULL << 53)) { m >>= 1; e++; }
        d = ldexp((double)m, e + 32 * base - 149);
    }
    out[c] = __double2float_rn(d);
}

// limbs for sums of terms up to mmax: the top term's bit place, 24 significand
// bits and 32 bits of carries (fewer than 2^32 terms per cell)
static int exact_limbs(float mmax) {
    const uint32_t e = (uint32_t)(reinterpret_cast<const uint32_t &>(mmax) >> 23);
    const int top = (int)e + 1 + 24 + 32;              // one spare place for a rounded-up term
    return std::min(EXACT_MAX_LIMBS, top / 32 + 2);
}

// ---- TSC (DENS_INTERP_TSC / VEL_INTERP_TSC) as a gather over TSC cells -------
// Particles are sorted by their TSC cell I (src/particles.f90:73-75); each grid
// cell gathers from the 27 neighbouring TSC cells.
struct TscArgs {
    int nx, rad_lo, periodic;
    float dx, r1, rn, leng;
    const float *rad;
};

__device__ __forceinline__ void tsc_axis(const TscArgs &A, float xt, int &cell, float w[3]) {
    const float *rad = A.rad - A.rad_lo;
    if (A.periodic) {
        if (xt < A.r1) xt = __fadd_rn(xt, A.leng);
        if (xt >= A.rn) xt = __fsub_rn(xt, A.leng);
    }
    const int i = (int)__fadd_rn(__fdiv_rn(__fsub_rn(xt, rad[1]), A.dx), 0.49999f) + 1;
    float bas = fabsf(__fsub_rn(rad[i - 1], xt));
    float t = __fsub_rn(1.5f, __fdiv_rn(bas, A.dx));
    w[0] = __fmul_rn(0.5f, __fmul_rn(t, t));
    bas = fabsf(__fsub_rn(rad[i], xt));
    t = __fdiv_rn(bas, A.dx);
    w[1] = __fsub_rn(0.75f, __fmul_rn(t, t));
    bas = fabsf(__fsub_rn(rad[i + 1], xt));
    t = __fsub_rn(1.5f, __fdiv_rn(bas, A.dx));
    w[2] = __fmul_rn(0.5f, __fmul_rn(t, t));
    cell = i;
}

__global__ void k_tsc_keys(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                           const float *__restrict__ z, TscArgs A, uint32_t *__restrict__ keys,
                           int32_t *__restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ci, cj, ck;
    float w[3];
    tsc_axis(A, x[i], ci, w);
    tsc_axis(A, y[i], cj, w);
    tsc_axis(A, z[i], ck, w);
    keys[i] = (uint32_t)(ci - 1) + (uint32_t)A.nx * ((uint32_t)(cj - 1) + (uint32_t)A.nx * (uint32_t)(ck - 1));
    vals[i] = (int32_t)i;
}

// Each grid cell merges the 27 particle lists of the TSC cells around it (each
// ascending by particle index: stable sort) and adds the contributions in
// particle order: the order of the reference's serial loop, which the oracle
// keeps (the reference's OpenMP atomics leave it open).  Density sums in
// REAL*8, the velocity and weight sums in REAL*4 (src/particles.f90:241-248).
__global__ void __launch_bounds__(128)
k_tsc_gather(int64_t nc, const int64_t *__restrict__ start, const int32_t *__restrict__ order,
             const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
             const float *__restrict__ m, const float *__restrict__ vx, const float *__restrict__ vy,
             const float *__restrict__ vz, TscArgs A, float *__restrict__ u_mass, float *__restrict__ u2,
             float *__restrict__ u3, float *__restrict__ u4) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int nx = A.nx;
    const int ix = (int)(c % nx) + 1, jy = (int)((c / nx) % nx) + 1, kz = (int)(c / ((int64_t)nx * nx)) + 1;
    int64_t cur[27], end[27];
    int32_t head[27];
#pragma unroll
    for (int j = 0; j < 27; j++) {
        const int ox = j % 3 - 1, oy = (j / 3) % 3 - 1, oz = j / 9 - 1;
        int i = ix + ox, jj = jy + oy, k = kz + oz;
        bool ok = true;
        if (A.periodic) {
            if (i < 1) i += nx; else if (i > nx) i -= nx;
            if (jj < 1) jj += nx; else if (jj > nx) jj -= nx;
            if (k < 1) k += nx; else if (k > nx) k -= nx;
        } else {
            ok = i >= 1 && i <= nx && jj >= 1 && jj <= nx && k >= 1 && k <= nx;
        }
        cur[j] = 0;
        end[j] = 0;
        if (ok) {
            const int64_t b = (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(jj - 1) + (int64_t)nx * (k - 1));
            cur[j] = start[b];
            end[j] = start[b + 1];
        }
        head[j] = cur[j] < end[j] ? order[cur[j]] : INT_MAX;
    }
    double dm = 0.0;
    float s2 = 0.0f, s3 = 0.0f, s4 = 0.0f, sw = 0.0f;
    for (;;) {
        int32_t best = INT_MAX;
        int jb = -1;
#pragma unroll
        for (int j = 0; j < 27; j++)
            if (head[j] < best) { best = head[j]; jb = j; }
        if (jb < 0) break;
        const int ox = jb % 3 - 1, oy = (jb / 3) % 3 - 1, oz = jb / 9 - 1;
#pragma unroll
        for (int j = 0; j < 27; j++)
            if (j == jb) {
                cur[j]++;
                head[j] = cur[j] < end[j] ? order[cur[j]] : INT_MAX;
            }
        const int32_t pidx = best;
        int ci, cj, ck;
        float wx[3], wy[3], wz[3];
        tsc_axis(A, x[pidx], ci, wx);
        tsc_axis(A, y[pidx], cj, wy);
        tsc_axis(A, z[pidx], ck, wz);
        // this cell lies at -ox, -oy, -oz from the particle's TSC cell
        const float fx = wx[1 - ox], fy = wy[1 - oy], fz = wz[1 - oz];
        if (u_mass) dm += (double)__fmul_rn(__fmul_rn(__fmul_rn(m[pidx], fx), fy), fz);
        if (u2) {
            const float w = __fmul_rn(__fmul_rn(fx, fy), fz);
            s2 = __fadd_rn(s2, __fmul_rn(vx[pidx], w));
            s3 = __fadd_rn(s3, __fmul_rn(vy[pidx], w));
            s4 = __fadd_rn(s4, __fmul_rn(vz[pidx], w));
            sw = __fadd_rn(sw, w);
        }
    }
    if (u_mass) u_mass[c] = (float)dm;
    if (u2) {
        const float wei = sw == 0.0f ? 1.0f : sw;
        u2[c] = __fdiv_rn(s2, wei);
        u3[c] = __fdiv_rn(s3, wei);
        u4[c] = __fdiv_rn(s4, wei);
    }
}

// ---- starting radius of the radius-guided search: the K-th neighbour distance of
//      a uniform density equal to the particle count of the 3x3x3 bins around ----
__global__ void k_radius_estimate(KnnGrid G, int K, float fac, float *r0) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = G.nb;
    if (b >= (int64_t)nb * nb * nb) return;
    const int bx = (int)(b % nb), by = (int)((b / nb) % nb), bz = (int)(b / ((int64_t)nb * nb));
    int64_t n = 0;
    int vol = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int x = bx + dx, y = by + dy, z = bz + dz;
                if (G.periodic) { x = wrap_bin(x, nb); y = wrap_bin(y, nb); z = wrap_bin(z, nb); }
                else if (x < 0 || y < 0 || z < 0 || x >= nb || y >= nb || z >= nb) continue;
                const int bin = x + nb * (y + nb * z);
                n += G.start[bin + 1] - G.start[bin];
                vol++;
            }
    // K = n/vol per bin volume * (4/3) pi (r/bw)^3
    const float dens = fmaxf((float)n / (float)vol, 0.05f);
    r0[b] = fac * G.bw * cbrtf((float)K / (4.18879020f * dens));
}

// ---- out-of-box check (src/avism.f90:560-589) ---------------------------------
__global__ void k_box_check(int64_t n, const float *x, const float *y, const float *z, float half, int *bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (x[i] < -half || x[i] > half || y[i] < -half || y[i] > half || z[i] < -half || z[i] > half) atomicOr(bad, 1);
}

__global__ void k_zero_f32(int64_t n, float *a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0.0f;
}

// with the counters on: the ball-fallback cells and the particles left with
// h = 0 for FILL_H_ZEROS (Ctx::path_counts[0..1])
static void count_orphans(Ctx &c, const KnnGrid &G, int64_t n, const float *hp_s, int32_t nball) {
    if (!G.stats) return;
    c.path_counts[0] = nball;
    unsigned long long *d = c.get_t<unsigned long long>(B_RED2, 1);
    AV_CUDA(cudaMemsetAsync(d, 0, sizeof *d, c.stream));
    if (n > 0) ++c.launches, k_count_zero<<<grid_for(n, 256), 256, 0, c.stream>>>(n, hp_s, d);
    unsigned long long h = 0;
    AV_CUDA(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    c.path_counts[1] = (int64_t)h;
}

template <int KMAX, bool STATS>
static void run_sph_kernels_ws(Ctx &c, const KnnGrid &G, const avism_params *p, const Level &L,
                              const P2G &a, const float *rad_d, bool vel_sph, bool need_h_cells,
                              const float4 *sv, float *pd_s, float *hp_s) {
    const size_t sm = sph_smem_bytes<KMAX>();
    const int K = p->kneighbours;
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    AV_CUDA(cudaFuncSetAttribute(k_ppart_dens_w<KMAX, STATS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    // the cell kernel stages its sums inside WarpKnnSmem: no extra rows, and a
    // shared-memory carveout just large enough for its five blocks leaves the
    // rest to L1, where the candidate records are read (K <= 32: 40%, 1% faster
    // than the default at 512^3)
    const size_t sm_cells = (size_t)SPH_WARPS * sizeof(WarpKnnSmem<KMAX>);
    const int carve = std::min(100, (int)((100 * 5 * (sm_cells + 1024) + 228 * 1024 - 1) / (228 * 1024)) + 5);
    AV_CUDA(cudaFuncSetAttribute(k_cells_knn_w<KMAX, STATS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cells));
    AV_CUDA(cudaFuncSetAttribute(k_cells_knn_w<KMAX, STATS>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
    if (vel_sph) {
        ++c.launches, k_ppart_dens_w<KMAX, STATS><<<grid_for(a.n, SPH_WARPS * PP_QPW), SPH_WARPS * 32, sm, c.stream>>>(
            G, a.n, K, sv, pd_s, a.part_dens);
        AV_CUDA(cudaGetLastError());
        c.mark("ppart_dens");
    }
    if (vel_sph || need_h_cells) {
        int32_t *ball_list = c.get_t<int32_t>(B_BALL, nc);
        int32_t *cnt_d = c.get_t<int32_t>(B_SCAL, 4);
        AV_CUDA(cudaMemsetAsync(cnt_d, 0, sizeof(int32_t), c.stream));
        CellArgs A;
        A.nx = nx; A.rad_lo = L.g.rad_lo; A.K = K; A.dx = L.g.dx; A.rad = rad_d; A.smask = a.smask;
        A.sv = sv; A.pd_s = pd_s; A.svw = nullptr;
        A.hp_s = hp_s; A.u2 = a.u2; A.u3 = a.u3; A.u4 = a.u4; A.do_vel = vel_sph ? 1 : 0;
        A.gauss = p->kernel_mode == 2;
        A.ball_list = ball_list; A.ball_count = cnt_d;
        if (vel_sph) {
            sv_velocities(c);
            float4 *svw = c.get_t<float4>(B_SVW, std::max<int64_t>(a.n, 1));
            if (a.n > 0) ++c.launches, k_mass_over_dens<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, sv, pd_s, svw);
            A.svw = svw;
        }
        const int64_t nblk = (int64_t)((nx + 3) / 4) * ((nx + 3) / 4) * ((nx + 1) / 2);
        ++c.launches, k_cells_knn_w<KMAX, STATS><<<(unsigned)nblk, SPH_WARPS * 32, sm_cells, c.stream>>>(G, A);
        AV_CUDA(cudaGetLastError());
        c.mark("cells_knn");
        int32_t nball = 0;
        AV_CUDA(cudaMemcpyAsync(&nball, cnt_d, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        cells_ball(c, G, A, nball);
        AV_CUDA(cudaGetLastError());
        c.mark("cells_ball");
        count_orphans(c, G, a.n, hp_s, nball);
        {
            constexpr int KC = KMAX;
            const int T = KNN_THREADS(KC);
            const size_t smc = (size_t)KC * T * sizeof(unsigned long long);
            AV_CUDA(cudaFuncSetAttribute(k_fill_h<KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc));
            ++c.launches, k_fill_h<KC><<<grid_for(a.n, T), T, smc, c.stream>>>(G, a.n, K, hp_s);
        }
        c.mark("fill_h_zeros");
        if (a.hpart) ++c.launches, k_unbin_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, G.sp, hp_s, a.hpart);
    }
    AV_CUDA(cudaGetLastError());
}

// the counters' instantiation only when they are on
template <int KMAX>
static void run_sph_kernels_w(Ctx &c, const KnnGrid &G, const avism_params *p, const Level &L, const P2G &a,
                              const float *rad_d, bool vel_sph, bool need_h_cells, const float4 *sv, float *pd_s,
                              float *hp_s) {
    if (G.stats) run_sph_kernels_ws<KMAX, true>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
    else run_sph_kernels_ws<KMAX, false>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
}

template <int KCAP>
static void run_sph_kernels(Ctx &c, const KnnGrid &G, const avism_params *p, const Level &L,
                            const P2G &a, const float *rad_d, bool vel_sph, bool need_h_cells,
                            const float4 *sv, float *pd_s, float *hp_s) {
    const int T = KNN_THREADS(KCAP);
    const size_t sm = (size_t)KCAP * T * sizeof(unsigned long long);
    const int K = p->kneighbours;
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    AV_CUDA(cudaFuncSetAttribute(k_ppart_dens<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    AV_CUDA(cudaFuncSetAttribute(k_cells_knn<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    AV_CUDA(cudaFuncSetAttribute(k_fill_h<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    if (vel_sph) {
        ++c.launches, k_ppart_dens<KCAP><<<grid_for(a.n, T), T, sm, c.stream>>>(G, a.n, K, sv, pd_s, a.part_dens);
        c.mark("ppart_dens");
    }
    if (vel_sph || need_h_cells) {
        int32_t *ball_list = c.get_t<int32_t>(B_BALL, nc);
        int32_t *cnt_d = c.get_t<int32_t>(B_SCAL, 4);
        AV_CUDA(cudaMemsetAsync(cnt_d, 0, sizeof(int32_t), c.stream));
        CellArgs A;
        A.nx = nx; A.rad_lo = L.g.rad_lo; A.K = K; A.dx = L.g.dx; A.rad = rad_d; A.smask = a.smask;
        A.sv = sv; A.pd_s = pd_s; A.svw = nullptr;
        A.hp_s = hp_s; A.u2 = a.u2; A.u3 = a.u3; A.u4 = a.u4; A.do_vel = vel_sph ? 1 : 0;
        A.gauss = p->kernel_mode == 2;
        A.ball_list = ball_list; A.ball_count = cnt_d;
        if (vel_sph) sv_velocities(c);
        const int tx = TileDims<T>::x, ty = TileDims<T>::y, tz = TileDims<T>::z;
        const int64_t nblk = (int64_t)((nx + tx - 1) / tx) * ((nx + ty - 1) / ty) * ((nx + tz - 1) / tz);
        ++c.launches, k_cells_knn<KCAP><<<(unsigned)nblk, T, sm, c.stream>>>(G, A);
        AV_CUDA(cudaGetLastError());
        c.mark("cells_knn");
        int32_t nball = 0;
        AV_CUDA(cudaMemcpyAsync(&nball, cnt_d, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        cells_ball(c, G, A, nball);
        AV_CUDA(cudaGetLastError());
        c.mark("cells_ball");
        count_orphans(c, G, a.n, hp_s, nball);
        ++c.launches, k_fill_h<KCAP><<<grid_for(a.n, T), T, sm, c.stream>>>(G, a.n, K, hp_s);
        c.mark("fill_h_zeros");
        if (a.hpart) ++c.launches, k_unbin_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, G.sp, hp_s, a.hpart);
    }
    AV_CUDA(cudaGetLastError());
}

// per-bin starting radius (and half-width) from the learned proposal (proposal.cu)
void proposal_predict(Ctx &c, const KnnGrid &G, float *r0, float *w0);

void particles_to_grid(Ctx &c, const avism_params *p, const Level &L, const P2G &a) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    const int K = p->kneighbours;
    AV_CHECK(K >= 1 && K <= 256, AVISM_ERR_ARG, "kneighbours must be in 1..256");
    AV_CHECK(a.n >= K || (p->flag_vel_interp == 0 && p->flag_dens_interp == 0), AVISM_ERR_ARG,
             "fewer particles than kneighbours");
    // particles must lie in [-L0/2, L0/2]
    {
        int *bad = c.get_t<int>(B_SCAL, 4);
        AV_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), c.stream));
        if (a.n > 0) ++c.launches, k_box_check<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, a.x, a.y, a.z, p->lado0 / 2.0f, bad);
        int hbad = 0;
        AV_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        AV_CHECK(hbad == 0, AVISM_ERR_OUT_OF_BOX,
                 "Particles outside the bounding box! Check L0! (must be inside [-L0/2, L0/2])");
    }
    float *rad_d = c.get_t<float>(B_RAD, L.rad.size());
    AV_CUDA(cudaMemcpyAsync(rad_d, L.rad.data(), L.rad.size() * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    for (float *g : {a.u_mass, a.u2, a.u3, a.u4}) ++c.launches, k_zero_f32<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, g);
    if (a.hpart) ++c.launches, k_zero_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, a.hpart);
    if (a.part_dens) ++c.launches, k_zero_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, a.part_dens);
    c.mark("p2g_setup");
    // no velocities (FLAG_VEL_AVAILABLE = 0, src/avism.f90:1259-1306): density only,
    // with H_DISTANCE + FILL_H_ZEROS before DDENS; u2..u4 stay zero
    const bool no_vel = p->no_velocities != 0;
    const bool vel_sph = p->flag_vel_interp == 1 && !no_vel, dens_sph = p->flag_dens_interp == 1;
    TscArgs TA;
    TA.nx = nx; TA.rad_lo = L.g.rad_lo; TA.periodic = p->periodic; TA.dx = L.g.dx; TA.rad = rad_d;
    TA.r1 = L.rad_at(1) - 0.5f * L.g.dx;
    TA.rn = L.rad_at(nx) + 0.5f * L.g.dx;
    TA.leng = TA.rn - TA.r1;
    if (vel_sph || dens_sph) {
        const char *occ_env = getenv("AVISM_TUNE_OCC");
        const float occ = occ_env ? (float)atof(occ_env) : 2.0f;
        const int64_t n1 = std::max<int64_t>(a.n, 1);
        float4 *sv = c.get_t<float4>(B_SV, n1);
        const char *fine_env = getenv("AVISM_TUNE_FINE");
        const bool fine = fine_env ? atoi(fine_env) != 0 : true;
        BinnedParticles bp = bin_particles(c, a.n, a.x, a.y, a.z, p->lado0, p->periodic, occ, a.vx, a.vy, a.vz,
                                           a.m, sv, fine);
        KnnGrid G = make_knn_grid(bp);
        c.path_counts[0] = c.path_counts[1] = c.path_counts[2] = 0;
        if (c.knn_stats) {
            G.stats = c.get_t<unsigned long long>(B_KNN_STATS, 8);
            AV_CUDA(cudaMemsetAsync(G.stats, 0, 8 * sizeof(unsigned long long), c.stream));
        }
        float *pd_s = c.get_t<float>(B_PDENS_S, n1), *hp_s = c.get_t<float>(B_HPART_S, n1);
        if (a.n > 0) {
            ++c.launches, k_zero_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, hp_s);
            ++c.launches, k_zero_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, pd_s);
        }
        c.mark("bin_particles");
        if (p->learned == 1) {
            // learned proposal: starting kNN radius per bin from the MLP
            const int64_t nbins = (int64_t)bp.nb * bp.nb * bp.nb;
            float *r0 = c.get_t<float>(B_PR_R0, nbins);
            float *w0 = c.get_t<float>(B_PR_W0, nbins);
            proposal_predict(c, G, r0, w0);
            G.r0 = r0;
            if (a.wprop) {
                a.wprop->w0 = w0;
                a.wprop->nb = bp.nb;
                a.wprop->periodic = bp.periodic;
                a.wprop->origin = bp.origin;
                a.wprop->inv_bw = bp.inv_bw;
                a.wprop->box = bp.box;
            }
            c.mark("proposal");
        } else if (p->learned == 2) {
            // hand-made proposal: a starting radius per bin from the local bin density
            const int64_t nbins = (int64_t)bp.nb * bp.nb * bp.nb;
            float *r0 = c.get_t<float>(B_KNN_R0, nbins);
            const char *fac_env = getenv("AVISM_TUNE_RFAC");
            const float fac = fac_env ? (float)atof(fac_env) : 1.1f;
            ++c.launches, k_radius_estimate<<<grid_for(nbins, 256), 256, 0, c.stream>>>(G, K, fac, r0);
            AV_CUDA(cudaGetLastError());
            G.r0 = r0;
            c.mark("radius_estimate");
        }
        const bool need_h_cells = dens_sph && !vel_sph;
        if (K <= 32) run_sph_kernels_w<32>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
        else if (K <= 64) run_sph_kernels_w<64>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
        else if (K <= 128) run_sph_kernels_w<128>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
        else run_sph_kernels<256>(c, G, p, L, a, rad_d, vel_sph, need_h_cells, sv, pd_s, hp_s);
        if (dens_sph) {
            // exact per-cell sums: the limb count follows the largest mass (every
            // term m*w/NORM is at most about m)
            float mmax = 0.0f;
            {
                float *d = c.get_t<float>(B_RED0, 1);
                size_t tmp = 0;
                c.attrs_ready();
                AV_CUDA(cub::DeviceReduce::Max(nullptr, tmp, a.m, d, (int)a.n, c.stream));
                void *t = c.get(B_CUB_TMP, tmp);
                AV_CUDA(cub::DeviceReduce::Max(t, tmp, a.m, d, (int)a.n, c.stream));
                AV_CUDA(cudaMemcpyAsync(&mmax, d, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
                c.sync();
            }
            AV_CHECK(mmax > 0.0f && std::isfinite(mmax), AVISM_ERR_ARG, "particle masses must be positive");
            const int nlimb = exact_limbs(mmax);
            unsigned long long *fix = c.get_t<unsigned long long>(B_FIX0, (size_t)nlimb * nc);
            AV_CUDA(cudaMemsetAsync(fix, 0, (size_t)nlimb * nc * sizeof(unsigned long long), c.stream));
            DdensArgs D;
            D.nx = nx; D.rad_lo = L.g.rad_lo; D.dx = L.g.dx; D.rx1 = L.rad_at(1); D.rad = rad_d;
            D.hp_s = hp_s; D.sv = sv; D.fix = fix; D.nlimb = nlimb;
            D.norm0 = nullptr;
            D.gauss = p->kernel_mode == 2;
            if (G.stats) {
                D.norm0 = c.get_t<unsigned long long>(B_RED2, 1);
                AV_CUDA(cudaMemsetAsync(D.norm0, 0, sizeof(unsigned long long), c.stream));
            }
            // the threads take the particles by support size (AVISM_TUNE_DDORDER=0: binned order)
            const int32_t *order = nullptr;
            const char *ord_env = getenv("AVISM_TUNE_DDORDER");
            if ((ord_env ? atoi(ord_env) : 1) != 0 && a.n > 0) {
                uint32_t *ka = c.get_t<uint32_t>(B_KEYS_A, a.n), *kb = c.get_t<uint32_t>(B_KEYS_B, a.n);
                int32_t *va = c.get_t<int32_t>(B_VALS_A, a.n), *vb = c.get_t<int32_t>(B_VALS_B, a.n);
                ++c.launches, k_ddens_class<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, hp_s, 1.0f / L.g.dx, ka, va);
                cub::DoubleBuffer<uint32_t> dk(ka, kb);
                cub::DoubleBuffer<int32_t> dv(va, vb);
                size_t tmp = 0;
                AV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)a.n, 0, 5, c.stream));
                AV_CUDA(cub::DeviceRadixSort::SortPairs(c.get(B_CUB_TMP, tmp), tmp, dk, dv, (int)a.n, 0, 5, c.stream));
                order = dv.Current();
            }
            c.mark("ddens_setup");
            ++c.launches, k_ddens<<<grid_for(a.n, DD_THREADS), DD_THREADS, 0, c.stream>>>(G, a.n, D, order);
            AV_CUDA(cudaGetLastError());
            if (D.norm0) {
                unsigned long long h = 0;
                AV_CUDA(cudaMemcpyAsync(&h, D.norm0, sizeof h, cudaMemcpyDeviceToHost, c.stream));
                c.sync();
                c.path_counts[2] = (int64_t)h;
            }
            c.mark("ddens_scatter");
            ++c.launches, k_exact_to_f32<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, fix, nlimb, a.u_mass);
            c.mark("ddens_convert");
        }
    }
    const bool vel_tsc = !no_vel && !vel_sph;
    if (vel_tsc || !dens_sph) {
        // TSC: sort particles by their TSC cell, then gather
        uint32_t *ka = c.get_t<uint32_t>(B_KEYS_A, a.n), *kb = c.get_t<uint32_t>(B_KEYS_B, a.n);
        int32_t *va = c.get_t<int32_t>(B_VALS_A, a.n), *vb = c.get_t<int32_t>(B_VALS_B, a.n);
        ++c.launches, k_tsc_keys<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, a.x, a.y, a.z, TA, ka, va);
        cub::DoubleBuffer<uint32_t> dk(ka, kb);
        cub::DoubleBuffer<int32_t> dv(va, vb);
        int end_bit = 1;
        while ((1LL << end_bit) < nc) end_bit++;
        size_t tmp = 0;
        AV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)a.n, 0, end_bit, c.stream));
        void *t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, dk, dv, (int)a.n, 0, end_bit, c.stream));
        int64_t *start = c.get_t<int64_t>(B_BIN_START, nc + 1);
        float4 *dummy = c.get_t<float4>(B_SP, std::max<int64_t>(a.n, 1));
        ++c.launches, k_bin_gather<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, dk.Current(), dv.Current(), a.x, a.y, a.z,
                                                                dummy, start, nc);
        c.attrs_ready();
        ++c.launches, k_tsc_gather<<<grid_for(nc, 128), 128, 0, c.stream>>>(
            nc, start, dv.Current(), a.x, a.y, a.z, a.m, a.vx, a.vy, a.vz, TA,
            dens_sph ? nullptr : a.u_mass, vel_tsc ? a.u2 : nullptr, a.u3, a.u4);
        AV_CUDA(cudaGetLastError());
        c.mark("tsc");
    }
    sv_velocities(c);
}

}  // namespace avism
