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
#include "bin_kernels.cuh"

namespace avism {

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
    float4 *pa = nullptr;
    bool with_v = false;
    if (sv) {
        if (c.attr_pending) {
            pa = c.get_t<float4>(B_PX4, n);
            // split form: the velocities are still being copied from the host;
            // the records take the masses now and the velocities in
            // sv_velocities(), before their first reader
            c.mass_ready();
            ++c.launches, k_pack_pos_mass<<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, y, z, m, pa);
            c.svp.on = true;
            c.svp.n = n;
            c.svp.sp = sp;
            c.svp.sv = sv;
            c.svp.vx = vx;
            c.svp.vy = vy;
            c.svp.vz = vz;
        } else {
            pa = c.get_t<float4>(B_PX4, 2 * (size_t)n);
            with_v = true;
            c.attrs_ready();
            ++c.launches, k_pack_particles<<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, y, z, m, vx, vy, vz, pa);
        }
    }
    if (fine) {
        int32_t *fstart = c.get_t<int32_t>(B_FSTART, nkeys + 1);
        bp.fstart = fstart;
        ++c.launches, k_bin_gather2<true><<<grid_for(n, 256), 256, 0, c.stream>>>(
            n, dk.Current(), dv.Current(), x, y, z, pa, with_v, sp, sv, start, nbins, fstart);
    } else {
        ++c.launches, k_bin_gather2<false><<<grid_for(n, 256), 256, 0, c.stream>>>(
            n, dk.Current(), dv.Current(), x, y, z, pa, with_v, sp, sv, start, nbins, nullptr);
    }
    AV_CUDA(cudaGetLastError());
    return bp;
}

void sv_velocities(Ctx &c) {
    if (!c.svp.on) return;
    const Ctx::SvPending v = c.svp;
    c.svp = Ctx::SvPending{};
    c.attrs_ready();
    if (v.n <= 0) return;
    float4 *pb = c.get_t<float4>(B_PV4, v.n);
    ++c.launches, k_pack_vel<<<grid_for(v.n, 256), 256, 0, c.stream>>>(v.n, v.vx, v.vy, v.vz, pb);
    ++c.launches, k_gather_vel<<<grid_for(v.n, 256), 256, 0, c.stream>>>(v.n, v.sp, pb, v.sv);
    AV_CUDA(cudaGetLastError());
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
