// knn.cu -- particle binning and the exact k-nearest-neighbour engine.
//
// Replaces the k-d tree of src/kdtree.f90 (build_kdtree / knn_search /
// ball_search) for the SPH smoothing of src/particles.f90.  Particles are
// sorted into a uniform grid of bins (stable radix sort, bin-major order);
// each query walks shells of bins outward from its own bin and keeps an exact
// top-K list in shared memory.  The search stops once the K-th distance is
// below the distance to the nearest unvisited bin, so results are exact:
// the K smallest (squared distance, particle index) pairs, with the squared
// distance computed as distance() in src/kdtree.f90:1441-1465.
#include <cub/cub.cuh>
#include <cfloat>

#include "common.cuh"
#include "knn_core.cuh"
#include "knn_warp.cuh"

namespace avism {

// ---- binning -----------------------------------------------------------------
__global__ void k_bin_keys(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
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
__global__ void k_bin_keys_fine(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
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
__global__ void k_bin_gather(int64_t n, const uint32_t *__restrict__ keys, const int32_t *__restrict__ vals,
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

// (x, y, z, m) and (vx, vy, vz, 0) as float4 records in input order: the
// binned gather then fetches two 16-byte records per particle instead of seven
// scattered 4-byte words (one DRAM sector each)
__global__ void k_pack_particles(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                                 const float *__restrict__ z, const float *__restrict__ m,
                                 const float *__restrict__ vx, const float *__restrict__ vy,
                                 const float *__restrict__ vz, float4 *__restrict__ pa, float4 *__restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pa[i] = make_float4(x[i], y[i], z[i], m[i]);
    pb[i] = make_float4(vx[i], vy[i], vz[i], 0.0f);
}

// k_bin_gather with the attributes from the packed records (pa non-null) and,
// for FINE keys, the quarter-bin offsets as well
template <bool FINE>
__global__ void k_bin_gather2(int64_t n, const uint32_t *__restrict__ keys, const int32_t *__restrict__ vals,
                              const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                              const float4 *__restrict__ pa, const float4 *__restrict__ pb, float4 *__restrict__ sp,
                              float4 *__restrict__ sv, int64_t *__restrict__ start, int64_t nbins,
                              int32_t *__restrict__ fstart) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t v = vals[i];
    if (pa) {
        const float4 a = pa[v], b = pb[v];
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

__global__ void k_empty_start(int64_t *start, int64_t nbins) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nbins) start[i] = 0;
}

BinnedParticles bin_particles(Ctx &c, int64_t n, const float *x, const float *y, const float *z,
                              float box, int periodic, float occupancy, const float *vx, const float *vy,
                              const float *vz, const float *m, float4 *sv, bool fine) {
    BinnedParticles bp;
    bp.n = n;
    bp.periodic = periodic;
    bp.box = box;
    double nbd = std::floor(std::cbrt((double)n / (double)occupancy));
    int nb = (int)std::max(1.0, std::min(nbd, 1290.0));
    bp.nb = nb;
    bp.bw = box / (float)nb;
    bp.inv_bw = (float)nb / box;
    bp.origin = -box / 2.0f;
    const int64_t nbins = (int64_t)nb * nb * nb;
    int64_t *start = c.get_t<int64_t>(B_BIN_START, nbins + 1);
    float4 *sp = c.get_t<float4>(B_SP, std::max<int64_t>(n, 1));
    bp.sp = sp;
    bp.start = start;
    if (n == 0) {
        ++c.launches, k_empty_start<<<grid_for(nbins + 1, 256), 256, 0, c.stream>>>(start, nbins);
        return bp;
    }
    AV_CHECK(n < (int64_t)INT32_MAX, AVISM_ERR_ARG, "more than 2^31-1 particles");
    // quarter-bin keys while 4 nb^3 offsets stay below 2^31
    fine = fine && (int64_t)KNN_XF * nbins < (int64_t)INT32_MAX;
    const int64_t nkeys = fine ? (int64_t)KNN_XF * nbins : nbins;
    uint32_t *ka = c.get_t<uint32_t>(B_KEYS_A, n), *kb = c.get_t<uint32_t>(B_KEYS_B, n);
    int32_t *va = c.get_t<int32_t>(B_VALS_A, n), *vb = c.get_t<int32_t>(B_VALS_B, n);
    if (fine)
        ++c.launches, k_bin_keys_fine<<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, y, z, bp.origin, bp.inv_bw, nb,
                                                                              ka, va);
    else
        ++c.launches, k_bin_keys<<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, y, z, bp.origin, bp.inv_bw, nb, ka, va);
    AV_CUDA(cudaGetLastError());
    cub::DoubleBuffer<uint32_t> dk(ka, kb);
    cub::DoubleBuffer<int32_t> dv(va, vb);
    int end_bit = 1;
    while ((1LL << end_bit) < nkeys) end_bit++;
    size_t tmp = 0;
    AV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)n, 0, end_bit, c.stream));
    void *t = c.get(B_CUB_TMP, tmp);
    AV_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, dk, dv, (int)n, 0, end_bit, c.stream));
    float4 *pa = nullptr, *pb = nullptr;
    if (sv) {
        pa = c.get_t<float4>(B_PX4, n);
        pb = c.get_t<float4>(B_PV4, n);
        ++c.launches, k_pack_particles<<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, y, z, m, vx, vy, vz, pa, pb);
    }
    if (fine) {
        int32_t *fstart = c.get_t<int32_t>(B_FSTART, nkeys + 1);
        bp.fstart = fstart;
        ++c.launches, k_bin_gather2<true><<<grid_for(n, 256), 256, 0, c.stream>>>(
            n, dk.Current(), dv.Current(), x, y, z, pa, pb, sp, sv, start, nbins, fstart);
    } else {
        ++c.launches, k_bin_gather2<false><<<grid_for(n, 256), 256, 0, c.stream>>>(
            n, dk.Current(), dv.Current(), x, y, z, pa, pb, sp, sv, start, nbins, nullptr);
    }
    AV_CUDA(cudaGetLastError());
    return bp;
}

// ---- batch kNN (the C-ABI's avism_gpu_knn) ----------------------------------
template <int KCAP>
__global__ void __launch_bounds__(KNN_THREADS(KCAP))
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

// warp-per-query form: WQ_WARPS warps per block, WQ_QPW consecutive queries per warp
constexpr int WQ_WARPS = 8, WQ_QPW = 4;

template <int KMAX>
__global__ void __launch_bounds__(WQ_WARPS * 32)
k_knn_batch_w(KnnGrid G, int64_t nq, const float *__restrict__ qx, const float *__restrict__ qy,
              const float *__restrict__ qz, int K, int64_t *__restrict__ idx_out, float *__restrict__ dist_out) {
    extern __shared__ __align__(16) unsigned char wq_smem[];
    WarpKnnSmem<KMAX> &S = reinterpret_cast<WarpKnnSmem<KMAX> *>(wq_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t q0 = ((int64_t)blockIdx.x * WQ_WARPS + (threadIdx.x >> 5)) * WQ_QPW;
    for (int t = 0; t < WQ_QPW; t++) {
        const int64_t q = q0 + t;
        if (q >= nq) break;
        const int cnt = knn_warp_exact<KMAX>(G, qx[q], qy[q], qz[q], K, 0.0f, S,
                                             reinterpret_cast<unsigned long long *>(S.d2));
        for (int i = lane; i < K; i += 32) {
            if (i < cnt) {
                idx_out[q * K + i] = (int64_t)__float_as_int(G.sp[S.res_pos[i]].w) + 1;
                dist_out[q * K + i] = sqrtf(__uint_as_float(S.res_d2[i]));
            } else {
                idx_out[q * K + i] = -1;
                dist_out[q * K + i] = sqrtf(FLT_MAX);     // knn_search initialises dist = HUGE(0.0)
            }
        }
    }
}

template <int KMAX>
static void launch_knn_batch_w(Ctx &c, const KnnGrid &G, int64_t nq, const float *qx, const float *qy,
                               const float *qz, int k, int64_t *idx, float *dist) {
    const size_t sm = (size_t)WQ_WARPS * sizeof(WarpKnnSmem<KMAX>);
    AV_CUDA(cudaFuncSetAttribute(k_knn_batch_w<KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    ++c.launches, k_knn_batch_w<KMAX><<<grid_for(nq, WQ_WARPS * WQ_QPW), WQ_WARPS * 32, sm, c.stream>>>(
        G, nq, qx, qy, qz, k, idx, dist);
    AV_CUDA(cudaGetLastError());
}

template <int KCAP>
static void launch_knn_batch(Ctx &c, const KnnGrid &G, int64_t nq, const float *qx, const float *qy,
                             const float *qz, int k, int64_t *idx, float *dist) {
    const int T = KNN_THREADS(KCAP);
    const size_t sm = (size_t)KCAP * T * sizeof(unsigned long long);
    AV_CUDA(cudaFuncSetAttribute(k_knn_batch<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    ++c.launches, k_knn_batch<KCAP><<<grid_for(nq, T), T, sm, c.stream>>>(G, nq, qx, qy, qz, k, idx, dist);
    AV_CUDA(cudaGetLastError());
}

void knn_batch(Ctx &c, const BinnedParticles &bp, int64_t nq, const float *qx, const float *qy,
               const float *qz, int k, int64_t *idx, float *dist) {
    KnnGrid G = make_knn_grid(bp);
    if (nq == 0) return;
    if (k <= 32) launch_knn_batch_w<32>(c, G, nq, qx, qy, qz, k, idx, dist);
    else if (k <= 64) launch_knn_batch_w<64>(c, G, nq, qx, qy, qz, k, idx, dist);
    else if (k <= 128) launch_knn_batch_w<128>(c, G, nq, qx, qy, qz, k, idx, dist);
    else if (k <= 256) launch_knn_batch<256>(c, G, nq, qx, qy, qz, k, idx, dist);
    else throw Error{AVISM_ERR_ARG, "kneighbours > 256 is not supported"};
}

}  // namespace avism
