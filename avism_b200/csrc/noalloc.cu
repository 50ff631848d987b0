// noalloc.cu -- avism_gpu_knn_noalloc: the exact kNN of avism_gpu_knn with every
// scratch buffer carved from one static device array, so that a call allocates
// nothing.  The kernels are the ones of knn.cu (binning, radix sort, shell
// search); only the host orchestration differs: no context, no buffer pool, the
// caller's stream, device pointers only.
//
// Scratch layout (offsets are multiples of 256 bytes):
//   sp      float4[MAX_N]          binned particles
//   start   int64[MAX_BINS + 1]    bin offsets (every entry written by k_bin_gather)
//   keys    uint32[MAX_N] x 2      radix-sort double buffer
//   vals    int32[MAX_N] x 2
//   lim     uint32                 bounding half-width of non-periodic points,
//                                  cleared by the call before use
//   cub     CUB_BYTES              radix-sort temporary storage
#include <cub/cub.cuh>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "knn_core.cuh"
#include "bin_kernels.cuh"

namespace avism {
namespace noalloc {

constexpr int64_t MAX_N = AVISM_KNN_NOALLOC_MAX_N;
constexpr float OCCUPANCY = 4.0f;                 // particles per bin, as avism_gpu_knn
constexpr int64_t MAX_BINS = MAX_N / 4;            // nb^3 <= n / OCCUPANCY
constexpr size_t CUB_BYTES = size_t(4) << 20;

constexpr size_t up256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t OFF_SP = 0;
constexpr size_t OFF_START = OFF_SP + up256(sizeof(float4) * MAX_N);
constexpr size_t OFF_KA = OFF_START + up256(sizeof(int64_t) * (MAX_BINS + 1));
constexpr size_t OFF_KB = OFF_KA + up256(sizeof(uint32_t) * MAX_N);
constexpr size_t OFF_VA = OFF_KB + up256(sizeof(uint32_t) * MAX_N);
constexpr size_t OFF_VB = OFF_VA + up256(sizeof(int32_t) * MAX_N);
constexpr size_t OFF_LIM = OFF_VB + up256(sizeof(int32_t) * MAX_N);
constexpr size_t OFF_CUB = OFF_LIM + 256;
constexpr size_t TOTAL = OFF_CUB + CUB_BYTES;
static_assert(TOTAL < (size_t(40) << 20), "static kNN scratch above its stated 40 MiB");

static __device__ __align__(256) unsigned char g_knn_scratch[TOTAL];

constexpr int MAX_DEVICES = 64;
static std::mutex g_setup_mutex;
static unsigned char *g_scratch_addr[MAX_DEVICES];

// Largest |v| over n floats as ordered bits (non-negative floats order as
// unsigned integers); one atomicMax per warp.
__global__ void k_abs_max_bits(int64_t n, const float *__restrict__ a, unsigned *__restrict__ out) {
    unsigned m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fabsf(a[i])));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

template <int KCAP>
static void launch(cudaStream_t s, const KnnGrid &G, int64_t nq, const float *qx, const float *qy,
                   const float *qz, int k, int64_t *idx, float *dist) {
    const int T = KNN_THREADS(KCAP);
    const size_t sm = (size_t)KCAP * T * sizeof(unsigned long long);
    AV_CUDA(cudaFuncSetAttribute(k_knn_batch<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_knn_batch<KCAP><<<grid_for(nq, T), T, sm, s>>>(G, nq, qx, qy, qz, k, idx, dist);
    AV_CUDA(cudaGetLastError());
}

// Scratch address on `device`, looked up once per device.
static unsigned char *scratch_for(int device) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        int major = 0;
        AV_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
        AV_CHECK(major == 10, AVISM_ERR_NO_DEVICE, "knn_noalloc: device is not a B200 (sm_100)");
        void *p = nullptr;
        AV_CUDA(cudaGetSymbolAddress(&p, g_knn_scratch));
        g_scratch_addr[device] = (unsigned char *)p;
    }
    return g_scratch_addr[device];
}

static void check_device_ptr(const void *p, int device, const char *name) {
    cudaPointerAttributes a{};
    AV_CUDA(cudaPointerGetAttributes(&a, p));
    const bool ok = (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
    if (!ok)
        throw Error{AVISM_ERR_ARG, std::string("knn_noalloc: ") + name +
                                       " is not a device pointer on the given device (host arrays would need "
                                       "staging copies; use avism_gpu_knn for them)"};
}

static void run(int device, cudaStream_t s, int64_t n, const float *x, const float *y, const float *z,
                float box_l, int64_t nq, const float *qx, const float *qy, const float *qz, int k,
                int64_t *idx, float *dist) {
    AV_CHECK(n >= 1 && nq >= 0 && k >= 1 && k <= 256 && x && y && z, AVISM_ERR_ARG,
             "knn_noalloc: bad arguments (need n >= 1, nq >= 0, 1 <= k <= 256, non-null x, y, z)");
    if (n > MAX_N) {
        char m[200];
        std::snprintf(m, sizeof m,
                      "knn_noalloc: n = %lld particles exceeds the static scratch limit "
                      "AVISM_KNN_NOALLOC_MAX_N = %lld; use avism_gpu_knn",
                      (long long)n, (long long)MAX_N);
        throw Error{AVISM_ERR_ARG, m};
    }
    AV_CHECK(nq == 0 || (qx && qy && qz && idx && dist), AVISM_ERR_ARG, "knn_noalloc: null query or output");
    unsigned char *S = scratch_for(device);
    for (auto pr : {std::make_pair((const void *)x, "x"), std::make_pair((const void *)y, "y"),
                    std::make_pair((const void *)z, "z")})
        check_device_ptr(pr.first, device, pr.second);
    if (nq == 0) return;
    for (auto pr : {std::make_pair((const void *)qx, "qx"), std::make_pair((const void *)qy, "qy"),
                    std::make_pair((const void *)qz, "qz"), std::make_pair((const void *)idx, "idx"),
                    std::make_pair((const void *)dist, "dist")})
        check_device_ptr(pr.first, device, pr.second);

    float box = box_l;
    const int periodic = box_l > 0.0f;
    if (!periodic) {
        // bounding cube of the points and the queries, centred at 0 (as avism_gpu_knn)
        unsigned *lim = (unsigned *)(S + OFF_LIM);
        AV_CUDA(cudaMemsetAsync(lim, 0, sizeof(unsigned), s));
        for (int a = 0; a < 6; a++) {
            const float *p = a == 0 ? x : a == 1 ? y : a == 2 ? z : a == 3 ? qx : a == 4 ? qy : qz;
            const int64_t cnt = a < 3 ? n : nq;
            k_abs_max_bits<<<(int)std::min<int64_t>((cnt + 255) / 256, 4 * 148), 256, 0, s>>>(cnt, p, lim);
            AV_CUDA(cudaGetLastError());
        }
        unsigned hl = 0;
        AV_CUDA(cudaMemcpyAsync(&hl, lim, sizeof hl, cudaMemcpyDeviceToHost, s));
        AV_CUDA(cudaStreamSynchronize(s));
        float lf;
        std::memcpy(&lf, &hl, sizeof lf);
        box = 2.0f * lf * 1.0001f + 1e-6f;
    }

    BinnedParticles bp;
    bp.n = n;
    bp.periodic = periodic;
    bp.box = box;
    const double nbd = std::floor(std::cbrt((double)n / (double)OCCUPANCY));
    const int nb = (int)std::max(1.0, std::min(nbd, 1290.0));
    const int64_t nbins = (int64_t)nb * nb * nb;
    AV_CHECK(nbins <= MAX_BINS, AVISM_ERR_INTERNAL, "knn_noalloc: bin count above the scratch layout");
    bp.nb = nb;
    bp.bw = box / (float)nb;
    bp.inv_bw = (float)nb / box;
    bp.origin = -box / 2.0f;
    float4 *sp = (float4 *)(S + OFF_SP);
    int64_t *start = (int64_t *)(S + OFF_START);
    uint32_t *ka = (uint32_t *)(S + OFF_KA), *kb = (uint32_t *)(S + OFF_KB);
    int32_t *va = (int32_t *)(S + OFF_VA), *vb = (int32_t *)(S + OFF_VB);
    bp.sp = sp;
    bp.start = start;

    k_bin_keys<<<grid_for(n, 256), 256, 0, s>>>(n, x, y, z, bp.origin, bp.inv_bw, nb, ka, va);
    AV_CUDA(cudaGetLastError());
    cub::DoubleBuffer<uint32_t> dk(ka, kb);
    cub::DoubleBuffer<int32_t> dv(va, vb);
    int end_bit = 1;
    while ((1LL << end_bit) < nbins) end_bit++;
    size_t tmp = 0;
    AV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)n, 0, end_bit, s));
    AV_CHECK(tmp <= CUB_BYTES, AVISM_ERR_INTERNAL, "knn_noalloc: radix-sort storage above the scratch layout");
    AV_CUDA(cub::DeviceRadixSort::SortPairs(S + OFF_CUB, tmp, dk, dv, (int)n, 0, end_bit, s));
    k_bin_gather<<<grid_for(n, 256), 256, 0, s>>>(n, dk.Current(), dv.Current(), x, y, z, sp, start, nbins);
    AV_CUDA(cudaGetLastError());

    const KnnGrid G = make_knn_grid(bp);
    if (k <= 32) launch<32>(s, G, nq, qx, qy, qz, k, idx, dist);
    else if (k <= 64) launch<64>(s, G, nq, qx, qy, qz, k, idx, dist);
    else if (k <= 128) launch<128>(s, G, nq, qx, qy, qz, k, idx, dist);
    else launch<256>(s, G, nq, qx, qy, qz, k, idx, dist);
}

}  // namespace noalloc
}  // namespace avism

extern "C" int avism_gpu_knn_noalloc(int device, void *stream, int64_t n, const float *x, const float *y,
                                     const float *z, float box_l, int64_t nq, const float *qx,
                                     const float *qy, const float *qz, int32_t k, int64_t *idx, float *dist,
                                     char *errbuf, int32_t errlen) {
    using namespace avism;
    int status = AVISM_OK;
    std::string msg;
    int prev = -1;
    try {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
            throw Error{AVISM_ERR_NO_DEVICE, "knn_noalloc: no CUDA device"};
        AV_CHECK(device >= 0 && device < count && device < noalloc::MAX_DEVICES, AVISM_ERR_ARG,
                 "knn_noalloc: device ordinal out of range");
        AV_CUDA(cudaGetDevice(&prev));
        AV_CUDA(cudaSetDevice(device));
        noalloc::run(device, (cudaStream_t)stream, n, x, y, z, box_l, nq, qx, qy, qz, k, idx, dist);
    } catch (const Error &e) {
        status = e.code;
        msg = e.msg;
    } catch (const std::exception &e) {
        status = AVISM_ERR_INTERNAL;
        msg = std::string("knn_noalloc: ") + e.what();
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (errbuf && errlen > 0) {
        const size_t m = std::min<size_t>(msg.size(), (size_t)errlen - 1);
        std::memcpy(errbuf, msg.data(), m);
        errbuf[m] = '\0';
    }
    return status;
}
