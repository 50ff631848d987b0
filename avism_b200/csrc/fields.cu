// fields.cu -- density normalisation, divergence, ghost shell and the
// per-cell flag byte of MARK_ALL / VOIDFIND.
//
// Replaces src/avism.f90:1249-1250 and 1384-1411 (rho/rho_B, FP64 mean,
// rho/<rho>), DIVER_UNIFORM (src/divergence.f90:2-50), REAL_MAKE_PERIODIC
// (src/num.f90:89-133), MARK_ALL (src/voidfinding.f90:13-55) and the six
// directional flag grids of VOIDFIND (src/voidfinding.f90:256-432).
//
// The ext grid of U1CO / DIVERCO is never materialised on the hot path: ghost
// cells read the inner grids at wrapped coordinates.  Flags are packed into one byte per ext
// cell: bit0 FLAGV, bit1 X1, bit2 X2, bit3 Y1, bit4 Y2, bit5 Z1, bit6 Z2,
// bit7 FLAG_SUB.
#include <cub/cub.cuh>
#include <cuda.h>
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace avism {

#define UM_F 9.1717E18f
#define UL_F 10.98f

__global__ void k_rho(int64_t nc, const float *__restrict__ u_mass, float vol, float rote,
                      float *__restrict__ rho) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    float v = __fdiv_rn(u_mass[c], vol);   // U1DMCO / (DXX*DYY*DZZ*RETE**3)
    v = __fdiv_rn(v, rote);                // / ROTE
    rho[c] = __fmul_rn(v, rote);           // U1CO = U1CO*ROTE
}

__global__ void k_div_scalar(int64_t nc, float *__restrict__ a, float s) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) a[c] = __fdiv_rn(a[c], s);
}

// linear-theory divergence from the density contrast: -(coef * (U1CO - 1))
__global__ void k_lin_div(int64_t nc, const float *__restrict__ u1, float coef, float *__restrict__ dv) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) dv[c] = -__fmul_rn(coef, __fsub_rn(u1[c], 1.0f));
}

struct ToDouble {
    __host__ __device__ double operator()(float v) const { return (double)v; }
};

// d v / d axis at a face cell (pos == 1 or nx): periodic wrap or the
// reference's linear extrapolation (src/divergence.f90:15-46)
__device__ __forceinline__ float diver_edge(const float *__restrict__ v, int64_t c, int pos, int64_t stride, int nx,
                                            int periodic) {
    const float *p = v + c;
    if (pos > 1 && pos < nx) return __fdiv_rn(__fsub_rn(p[stride], p[-stride]), 2.0f);
    if (periodic) {
        const float *pp = pos == nx ? p - (int64_t)(nx - 1) * stride : p + stride;
        const float *pm = pos == 1 ? p + (int64_t)(nx - 1) * stride : p - stride;
        return __fdiv_rn(__fsub_rn(*pp, *pm), 2.0f);
    }
    if (pos == 1) {
        const float inner = __fdiv_rn(__fsub_rn(p[2 * stride], p[0]), 2.0f);
        return __fsub_rn(__fmul_rn(2.0f, __fsub_rn(p[stride], p[0])), inner);
    }
    const float inner = __fdiv_rn(__fsub_rn(p[0], p[-2 * stride]), 2.0f);
    return __fsub_rn(__fmul_rn(2.0f, __fsub_rn(p[0], p[-stride])), inner);
}

// DIVER_UNIFORM with periodic or extrapolated boundaries
__global__ void k_diver(int nx, float dx, int periodic, const float *__restrict__ v2,
                        const float *__restrict__ v3, const float *__restrict__ v4,
                        float *__restrict__ diver) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nc = (int64_t)nx * nx * nx;
    if (c >= nc) return;
    const int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    const int64_t sx = 1, sy = nx, sz = (int64_t)nx * nx;
    auto deriv = [&](const float *v, int pos, int64_t stride) -> float {
        const float *p = v + c;
        if (pos > 1 && pos < nx) return __fdiv_rn(__fsub_rn(p[stride], p[-stride]), 2.0f);
        if (periodic) {
            const float *pp = pos == nx ? p - (int64_t)(nx - 1) * stride : p + stride;
            const float *pm = pos == 1 ? p + (int64_t)(nx - 1) * stride : p - stride;
            return __fdiv_rn(__fsub_rn(*pp, *pm), 2.0f);
        }
        if (pos == 1) {
            const float inner = __fdiv_rn(__fsub_rn(p[2 * stride], p[0]), 2.0f);
            return __fsub_rn(__fmul_rn(2.0f, __fsub_rn(p[stride], p[0])), inner);
        }
        const float inner = __fdiv_rn(__fsub_rn(p[0], p[-2 * stride]), 2.0f);
        return __fsub_rn(__fmul_rn(2.0f, __fsub_rn(p[0], p[-stride])), inner);
    };
    const float ddx = deriv(v2, i, sx), ddy = deriv(v3, j, sy), ddz = deriv(v4, k, sz);
    diver[c] = __fadd_rn(__fadd_rn(__fdiv_rn(ddx, dx), __fdiv_rn(ddy, dx)), __fdiv_rn(ddz, dx));
}

// ---- DIVER_UNIFORM on TMA-staged tiles ----------------------------------------
// A CTA computes a DV_TX x DV_TY x DV_TZ tile of the inner grid.  One elected
// thread loads three boxes with cp.async.bulk.tensor (v2 with a +-4 x halo, v3
// with +-1 in y, v4 with +-1 in z; out-of-grid parts are zero-filled and
// never used) onto one mbarrier; the threads then difference from shared
// memory.  Cells on the grid's faces (periodic wrap or one-sided
// extrapolation) take their values from global memory, as k_diver does.
constexpr int DV_TX = 32, DV_TY = 8, DV_TZ = 8, DV_THREADS = 256;
constexpr uint32_t DV_WAIT_LIMIT = 1u << 22;

struct __align__(128) DvSmem {
    float v2[DV_TZ][DV_TY][DV_TX + 8];
    float v3[DV_TZ][DV_TY + 2][DV_TX];
    float v4[DV_TZ + 2][DV_TY][DV_TX];
    uint64_t mbar;
};

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(map), "r"(x), "r"(y), "r"(z),
           "r"((uint32_t)__cvta_generic_to_shared(mbar))
        : "memory");
}

__global__ void __launch_bounds__(DV_THREADS)
k_diver_tma(const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap m3,
            const __grid_constant__ CUtensorMap m4, int nx, float dx, int periodic, const float *__restrict__ v2,
            const float *__restrict__ v3, const float *__restrict__ v4, float *__restrict__ diver, int *err) {
    __shared__ DvSmem S;
    const int ntx = nx / DV_TX, nty = nx / DV_TY;
    const int bx = (int)(blockIdx.x % ntx), by = (int)((blockIdx.x / ntx) % nty), bz = (int)(blockIdx.x / (ntx * nty));
    const int X0 = bx * DV_TX, Y0 = by * DV_TY, Z0 = bz * DV_TZ;
    const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&S.mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t bytes = (uint32_t)(sizeof(S.v2) + sizeof(S.v3) + sizeof(S.v4));
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mb), "r"(bytes) : "memory");
        tma_load_3d(&S.v2[0][0][0], &m2, X0 - 4, Y0, Z0, &S.mbar);
        tma_load_3d(&S.v3[0][0][0], &m3, X0, Y0 - 1, Z0, &S.mbar);
        tma_load_3d(&S.v4[0][0][0], &m4, X0, Y0, Z0 - 1, &S.mbar);
    }
    __syncthreads();
    auto wait = [&]() {
        for (uint32_t it = 0; it < DV_WAIT_LIMIT; it++) {
            uint32_t r;
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(r) : "r"(mb) : "memory");
            if (r) return true;
        }
        return false;
    };
    if (!wait()) {                                 // report, give the copies one more bounded wait, leave
        if (threadIdx.x == 0) atomicExch(err, 1);
        wait();
        return;
    }
    const int64_t sy = nx, sz = (int64_t)nx * nx;
    for (int t = threadIdx.x; t < DV_TX * DV_TY * DV_TZ; t += DV_THREADS) {
        const int lx = t % DV_TX, ly = (t / DV_TX) % DV_TY, lz = t / (DV_TX * DV_TY);
        const int i = X0 + lx + 1, j = Y0 + ly + 1, k = Z0 + lz + 1;        // 1-based
        const int64_t c = (int64_t)(i - 1) + sy * (j - 1) + sz * (k - 1);
        float ddx, ddy, ddz;
        if (i > 1 && i < nx) ddx = __fdiv_rn(__fsub_rn(S.v2[lz][ly][lx + 5], S.v2[lz][ly][lx + 3]), 2.0f);
        else ddx = diver_edge(v2, c, i, 1, nx, periodic);
        if (j > 1 && j < nx) ddy = __fdiv_rn(__fsub_rn(S.v3[lz][ly + 2][lx], S.v3[lz][ly][lx]), 2.0f);
        else ddy = diver_edge(v3, c, j, sy, nx, periodic);
        if (k > 1 && k < nx) ddz = __fdiv_rn(__fsub_rn(S.v4[lz + 2][ly][lx], S.v4[lz][ly][lx]), 2.0f);
        else ddz = diver_edge(v4, c, k, sz, nx, periodic);
        diver[c] = __fadd_rn(__fadd_rn(__fdiv_rn(ddx, dx), __fdiv_rn(ddy, dx)), __fdiv_rn(ddz, dx));
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        AV_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        AV_CHECK(p && q == cudaDriverEntryPointSuccess, AVISM_ERR_CUDA, "cuTensorMapEncodeTiled not available");
        fn = (EncodeTiledFn)p;
    }
    return fn;
}

// f32 nx^3 grid, box bx x by x bz, zero fill outside the grid
static CUtensorMap grid_map(const float *g, int nx, int bx, int by, int bz) {
    CUtensorMap m;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)nx, (cuuint64_t)nx};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * nx * 4};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = encode_tiled_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)g, dims, strides, box, es,
                                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    AV_CHECK(r == CUDA_SUCCESS, AVISM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

// the TMA path needs whole tiles and 16-byte row pitches
static bool diver_tma_ok(int nx, const float *a, const float *b, const float *c) {
    auto al = [](const float *p) { return ((uintptr_t)p & 15) == 0; };
    return nx % DV_TX == 0 && nx % DV_TY == 0 && nx % DV_TZ == 0 && al(a) && al(b) && al(c);
}

// U1CO = (U1DMCO / (DXX*DYY*DZZ*RETE**3) / ROTE) * ROTE (src/avism.f90:1249-1250, 1386)
void rho_inner(Ctx &c, const Level &L, const float *u_mass, float *u1co_in) {
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    const float dx = L.g.dx;
    const float vol = ((dx * dx) * dx) * ((L.g.rete * L.g.rete) * L.g.rete);
    ++c.launches, k_rho<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u_mass, vol, L.g.rote, u1co_in);
    AV_CUDA(cudaGetLastError());
}

// DIVERCO from the velocity grids (DIVER_UNIFORM), or without velocities the
// linear-theory -OMEGA0**(0.6)*RETE*HTE*(U1CO - 1.0) (src/avism.f90:1647-1650),
// the REAL*4 coefficient with the host libm's powf, as the reference's
void divergence_inner(Ctx &c, const avism_params *p, const Level &L, const float *u1co_in, const float *u2,
                      const float *u3, const float *u4, float *diver_in) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    const float dx = L.g.dx;
    if (p->no_velocities) {
        const float coef = (::powf(p->omega0, 0.6f) * L.g.rete) * L.g.hte;
        ++c.launches, k_lin_div<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u1co_in, coef, diver_in);
    } else if (diver_tma_ok(nx, u2, u3, u4)) {
        const CUtensorMap m2 = grid_map(u2, nx, DV_TX + 8, DV_TY, DV_TZ);
        const CUtensorMap m3 = grid_map(u3, nx, DV_TX, DV_TY + 2, DV_TZ);
        const CUtensorMap m4 = grid_map(u4, nx, DV_TX, DV_TY, DV_TZ + 2);
        int *err = c.get_t<int>(B_SCAL, 4);
        AV_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c.stream));
        const unsigned ntiles = (unsigned)((nx / DV_TX) * (nx / DV_TY) * (nx / DV_TZ));
        ++c.launches, k_diver_tma<<<ntiles, DV_THREADS, 0, c.stream>>>(m2, m3, m4, nx, dx, p->periodic, u2, u3, u4,
                                                                       diver_in, err);
        AV_CUDA(cudaGetLastError());
        int herr = 0;
        AV_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        AV_CHECK(herr == 0, AVISM_ERR_TIMEOUT, "divergence: a TMA wait timed out");
    } else {
        ++c.launches, k_diver<<<grid_for(nc, 256), 256, 0, c.stream>>>(nx, dx, p->periodic, u2, u3, u4, diver_in);
    }
    AV_CUDA(cudaGetLastError());
}

FieldsOut fields_inner(Ctx &c, const avism_params *p, const Level &L, const float *u_mass,
                       const float *u2, const float *u3, const float *u4, float *u1co_in,
                       float *diver_in) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    rho_inner(c, L, u_mass, u1co_in);
    double *sum_d = c.get_t<double>(B_RED1, 1);
    cub::TransformInputIterator<double, ToDouble, const float *> it(u1co_in, ToDouble());
    size_t tmp = 0;
    AV_CUDA(cub::DeviceReduce::Sum(nullptr, tmp, it, sum_d, (int)nc, c.stream));
    void *t = c.get(B_CUB_TMP, tmp);
    AV_CUDA(cub::DeviceReduce::Sum(t, tmp, it, sum_d, (int)nc, c.stream));
    double sum = 0.0;
    AV_CUDA(cudaMemcpyAsync(&sum, sum_d, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const float mean = (float)(sum / (double)nc);
    ++c.launches, k_div_scalar<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u1co_in, mean);
    c.mark("normalise");
    divergence_inner(c, p, L, u1co_in, u2, u3, u4, diver_in);
    FieldsOut o;
    const float ul3 = (UL_F * UL_F) * UL_F;
    o.meandens = mean * (UM_F / ul3);
    return o;
}

// ---- survey mode: the D/(alpha R) contrast (src/avism.f90:1527-1578) ----------
// DSUM, RSUM and the MEANRATIO sum are REAL*8 sums per x-row (sequential in i),
// the rows of a plane summed in j order, the planes in k order: fixed, so ALPHA
// and the ratios do not depend on thread timing (the reference's DSUM / RSUM
// are an OpenMP reduction; its MEANRATIO a serial SUM).
__global__ void k_row_sums(int nx, const float *__restrict__ a, const int8_t *__restrict__ smask, int positive,
                           double *__restrict__ rows) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (int64_t)nx * nx) return;
    const float *ar = a + r * nx;
    const int8_t *sr = smask + r * nx;
    double s = 0.0;
    for (int i = 0; i < nx; i++) {
        const int8_t m = sr[i];
        if (positive ? m > 0 : m != 0) s = s + (double)ar[i];
    }
    rows[r] = s;
}
__global__ void k_plane_sums(int nx, const double *__restrict__ rows, double *__restrict__ planes) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nx) return;
    double s = 0.0;
    for (int j = 0; j < nx; j++) s = s + rows[(int64_t)k * nx + j];
    planes[k] = s;
}
__global__ void k_total_sum(int nx, const double *__restrict__ planes, double *__restrict__ out) {
    double s = 0.0;
    for (int k = 0; k < nx; k++) s = s + planes[k];
    *out = s;
}
// BASS8 = U1CO/(ALPHA*U1RAND) (or the floor where U1RAND = 0), floored at 1e-4,
// clamped at 1000, in REAL*8; stored as REAL*4 (src/avism.f90:1543-1566)
__global__ void k_survey_ratio(int64_t nc, float *__restrict__ u1, const float *__restrict__ ur,
                               const int8_t *__restrict__ smask, double alpha) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc || smask[c] == 0) return;
    const double floor8 = (double)1e-4f, max8 = (double)1000.0f;
    double b = (double)ur[c] > 0.0 ? __ddiv_rn((double)u1[c], __dmul_rn(alpha, (double)ur[c])) : floor8;
    b = fmax(floor8, b);
    b = fmin(max8, b);
    u1[c] = (float)b;
}
// WHERE (SMASK > 0) U1CO = U1CO / MEANRATIO
__global__ void k_survey_scale(int64_t nc, float *__restrict__ u1, const int8_t *__restrict__ smask, float meanratio) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc && smask[c] > 0) u1[c] = __fdiv_rn(u1[c], meanratio);
}
// COUNT(SMASK > 0)
__global__ void k_count_positive(int64_t nc, const int8_t *__restrict__ smask, unsigned long long *__restrict__ count) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned b = __ballot_sync(0xffffffffu, c < nc && smask[c] > 0);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, (unsigned long long)__popc(b));
}

static double blocked_sum(Ctx &c, int nx, const float *a, const int8_t *smask, int positive) {
    double *rows = c.get_t<double>(B_RED0, (size_t)nx * nx + nx + 1);
    double *planes = rows + (size_t)nx * nx, *tot = planes + nx;
    ++c.launches, k_row_sums<<<grid_for((int64_t)nx * nx, 128), 128, 0, c.stream>>>(nx, a, smask, positive, rows);
    ++c.launches, k_plane_sums<<<grid_for(nx, 128), 128, 0, c.stream>>>(nx, rows, planes);
    ++c.launches, k_total_sum<<<1, 1, 0, c.stream>>>(nx, planes, tot);
    AV_CUDA(cudaGetLastError());
    double h = 0.0;
    AV_CUDA(cudaMemcpyAsync(&h, tot, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    return h;
}

// the inner U1CO (rho/rho_B * ROTE) becomes D/(alpha R), mean 1 over SMASK > 0;
// returns MEANDENS = ROTE * (UM / UL**3)
float survey_contrast(Ctx &c, const Level &L, const int8_t *smask, const float *u1rand, float *u1co_in) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    const double dsum = blocked_sum(c, nx, u1co_in, smask, 0);
    const double rsum = blocked_sum(c, nx, u1rand, smask, 0);
    const double alpha = dsum / rsum;
    ++c.launches, k_survey_ratio<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u1co_in, u1rand, smask, alpha);
    AV_CUDA(cudaGetLastError());
    unsigned long long *cnt = c.get_t<unsigned long long>(B_RED2, 1);
    AV_CUDA(cudaMemsetAsync(cnt, 0, sizeof *cnt, c.stream));
    ++c.launches, k_count_positive<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, smask, cnt);
    unsigned long long count = 0;
    AV_CUDA(cudaMemcpyAsync(&count, cnt, sizeof count, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    AV_CHECK(count > 0, AVISM_ERR_ARG, "survey: the mask has no observed cell (SMASK > 0)");
    const float meanratio = (float)(blocked_sum(c, nx, u1co_in, smask, 1) / (double)count);
    ++c.launches, k_survey_scale<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u1co_in, smask, meanratio);
    AV_CUDA(cudaGetLastError());
    const float ul3 = (UL_F * UL_F) * UL_F;
    return L.g.rote * (UM_F / ul3);
}

// ---- grid input (FLAG_DATA = 2, src/avism.f90:1316-1362) ----------------------
// SMOOTH_2 (src/amr2uniform.f90:65-120) for levels below 0: every cell of the
// input grid (NHY^3) adds its value times WEI = (DX0*DY0*DZ0)/(DX*DY*DZ) to the
// coarse cell INT(((RX-RADX(1))/DX)+0.5)+1.  Here each coarse cell gathers its
// input cells (a contiguous range per axis, [lo, hi], from the host's map) in
// the reference's serial K, J, I order, so the REAL*4 sums match.
__global__ void k_smooth2(int nx, int nhy, const int32_t *__restrict__ lo, const int32_t *__restrict__ hi,
                          float wei, const float *__restrict__ a, float *__restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int64_t)nx * nx * nx) return;
    const int i = (int)(c % nx), j = (int)((c / nx) % nx), k = (int)(c / ((int64_t)nx * nx));
    float s = 0.0f;
    for (int kk = lo[k]; kk <= hi[k]; kk++)
        for (int jj = lo[j]; jj <= hi[j]; jj++)
            for (int ii = lo[i]; ii <= hi[i]; ii++)
                s = __fadd_rn(s, __fmul_rn(a[(int64_t)ii + (int64_t)nhy * ((int64_t)jj + (int64_t)nhy * kk)], wei));
    out[c] = s;
}

// U1CO = U1GCO, the divergence of (U2GCO, U3GCO, U4GCO), MEANDENS = ROTE*(UM/UL**3);
// u1g..u4g: the input grid (NHY^3, device), the level's grid is p->nx = NHY * 2^IR
// The level's copies of input grids given at NHY^3 (level 0): copied at
// level 0, SMOOTH_2-averaged below it (src/amr2uniform.f90:65-120).
void level_grids(Ctx &c, const Level &L, const avism_params *p, int nhy, int ngrids, const float *const *g,
                 float *const *co) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    if (nx == nhy) {                                   // IR = 0: U1GCO = U1G, ...
        for (int q = 0; q < ngrids; q++)
            AV_CUDA(cudaMemcpyAsync(co[q], g[q], sizeof(float) * (size_t)nc, cudaMemcpyDeviceToDevice, c.stream));
        return;
    }
    // the input grid's coordinates (MALLA at NHY, src/avism.f90:366-382) and
    // each input cell's coarse cell on this level
    avism_params p0 = *p;
    p0.nx = nhy;
    const Level L0 = make_level(&p0);
    const float dx = L.g.dx, dx0 = L0.g.dx, r1 = L.rad_at(1);
    std::vector<int32_t> lo(nx, INT32_MAX), hi(nx, -1);
    for (int ii = 1; ii <= nhy; ii++) {
        const int I = (int)(((L0.rad_at(ii) - r1) / dx) + 0.5f) + 1;
        AV_CHECK(I >= 1 && I <= nx, AVISM_ERR_ARG, "grid input: an input cell falls outside the level's grid");
        lo[I - 1] = std::min(lo[I - 1], ii - 1);
        hi[I - 1] = std::max(hi[I - 1], ii - 1);
    }
    const float wei = ((dx0 * dx0) * dx0) / ((dx * dx) * dx);
    int32_t *d = c.get_t<int32_t>(B_LABMAP, 2 * (size_t)nx);
    AV_CUDA(cudaMemcpyAsync(d, lo.data(), sizeof(int32_t) * nx, cudaMemcpyHostToDevice, c.stream));
    AV_CUDA(cudaMemcpyAsync(d + nx, hi.data(), sizeof(int32_t) * nx, cudaMemcpyHostToDevice, c.stream));
    for (int q = 0; q < ngrids; q++)
        ++c.launches, k_smooth2<<<grid_for(nc, 256), 256, 0, c.stream>>>(nx, nhy, d, d + nx, wei, g[q], co[q]);
    AV_CUDA(cudaGetLastError());
    c.sync();                                          // lo / hi are host vectors
}

float grid_fields_inner(Ctx &c, const avism_params *p, const Level &L, int nhy, const float *u1g, const float *u2g,
                        const float *u3g, const float *u4g, float *u1co_in, float *diver_in) {
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    const float *g[4] = {u1g, u2g, u3g, u4g};
    float *co[4] = {u1co_in, c.get_t<float>(B_U2, nc), c.get_t<float>(B_U3, nc), c.get_t<float>(B_U4, nc)};
    level_grids(c, L, p, nhy, 4, g, co);
    c.mark("grid_input");
    divergence_inner(c, p, L, u1co_in, co[1], co[2], co[3], diver_in);
    const float ul3 = (UL_F * UL_F) * UL_F;
    return L.g.rote * (UM_F / ul3);
}

// ---- MASCLET input (FLAG_DATA = 0) at levels <= 0 -----------------------------
// U1DMCO = (mass / (DXX*DYY*DZZ*RETE**3)) / ROTE (src/avism.f90:1065-1066), then
// U1CO by FLAG_DENS (1371-1373): U1DMCO + U1GCO, U1DMCO or U1GCO, times ROTE
// (1386)
__global__ void k_masclet_rho(int64_t nc, const float *__restrict__ u_mass, const float *__restrict__ u1g, float vol,
                              float rote, int flag_dens, float *__restrict__ u1) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    float dm = 0.0f;
    if (flag_dens <= 1) {
        dm = __fdiv_rn(u_mass[c], vol);
        dm = __fdiv_rn(dm, rote);
    }
    const float u = flag_dens == 0 ? __fadd_rn(dm, u1g[c]) : (flag_dens == 1 ? dm : u1g[c]);
    u1[c] = __fmul_rn(u, rote);
}
// DIVERCO = MIN(DIVERGCO, DIVERDMCO) (src/avism.f90:1636-1642)
__global__ void k_fill_i32_1(int64_t n, int32_t *__restrict__ a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 1;
}
__global__ void k_min_into(int64_t nc, float *__restrict__ a, const float *__restrict__ b) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) a[c] = b[c] < a[c] ? b[c] : a[c];
}

// ---- MASCLET level 1: DIVER_FINA_GAS (src/divergence.f90:55-340) and VMESH
//      (src/amr2uniform.f90:127-248) on the level-1 patches ----------------------
// DIVER0 inside the base grid: central differences over 2*DX0
__global__ void k_diver0(int nh, float dx0, const float *__restrict__ u2, const float *__restrict__ u3,
                         const float *__restrict__ u4, float *__restrict__ d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = nh - 2;
    if (t >= (int64_t)m * m * m) return;
    const int i = (int)(t % m) + 1, j = (int)((t / m) % m) + 1, k = (int)(t / ((int64_t)m * m)) + 1;   // 0-based 1..nh-2
    auto B = [&](int a, int b, int cc) { return (int64_t)a + (int64_t)nh * ((int64_t)b + (int64_t)nh * cc); };
    const float h = __fmul_rn(2.0f, dx0);
    const float b21 = __fdiv_rn(__fsub_rn(u2[B(i + 1, j, k)], u2[B(i - 1, j, k)]), h);
    const float b32 = __fdiv_rn(__fsub_rn(u3[B(i, j + 1, k)], u3[B(i, j - 1, k)]), h);
    const float b43 = __fdiv_rn(__fsub_rn(u4[B(i, j, k + 1)], u4[B(i, j, k - 1)]), h);
    d[B(i, j, k)] = __fadd_rn(__fadd_rn(b21, b32), b43);
}
// one face of DIVER0 copied from the plane inside it (axis a, side 0: index 1, 1: NHY)
__global__ void k_diver0_face(int nh, int a, int side, float *__restrict__ d) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nh * nh) return;
    const int u = (int)(t % nh), v = (int)(t / nh);
    const int to = side ? nh - 1 : 0, from = side ? nh - 2 : 1;
    auto B = [&](int q) {
        const int i = a == 0 ? q : u, j = a == 1 ? q : (a == 0 ? u : v), k = a == 2 ? q : v;
        return (int64_t)i + (int64_t)nh * ((int64_t)j + (int64_t)nh * k);
    };
    d[B(to)] = d[B(from)];
}
// one patch's divergence: its own central differences inside (2..N-1 over
// 2*DXR), the 2-cell rim from its parent base cells' differences (over 2*DX0),
// averaged with its own at index 2 and N-1 and in their place at 1 and N
struct PatchGeom {
    int n1, n2, n3, l1, l2, l3;
    int64_t off;
};
__global__ void k_patch_div(PatchGeom P, int nh, float dxr, float dx0, const float *__restrict__ v2,
                            const float *__restrict__ v3, const float *__restrict__ v4, const float *__restrict__ u2,
                            const float *__restrict__ u3, const float *__restrict__ u4, float *__restrict__ dv,
                            int *__restrict__ err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    if (t >= (int64_t)n1 * n2 * n3) return;
    const int i = (int)(t % n1) + 1, j = (int)((t / n1) % n2) + 1, k = (int)(t / ((int64_t)n1 * n2)) + 1;
    auto Q = [&](int a, int b, int cc) {
        return P.off + (int64_t)(a - 1) + (int64_t)n1 * ((int64_t)(b - 1) + (int64_t)n2 * (cc - 1));
    };
    float own = 0.0f;
    if (i >= 2 && i <= n1 - 1 && j >= 2 && j <= n2 - 1 && k >= 2 && k <= n3 - 1) {
        const float h = __fmul_rn(2.0f, dxr);
        const float b21 = __fdiv_rn(__fsub_rn(v2[Q(i + 1, j, k)], v2[Q(i - 1, j, k)]), h);
        const float b32 = __fdiv_rn(__fsub_rn(v3[Q(i, j + 1, k)], v3[Q(i, j - 1, k)]), h);
        const float b43 = __fdiv_rn(__fsub_rn(v4[Q(i, j, k + 1)], v4[Q(i, j, k - 1)]), h);
        own = __fadd_rn(__fadd_rn(b21, b32), b43);
    }
    float aux = 0.0f;
    if (i < 3 || i > n1 - 2 || j < 3 || j > n2 - 2 || k < 3 || k > n3 - 2) {
        const int c1 = (i + 1) / 2 + P.l1 - 1, c2 = (j + 1) / 2 + P.l2 - 1, c3 = (k + 1) / 2 + P.l3 - 1;
        if (c1 < 2 || c1 > nh - 1 || c2 < 2 || c2 > nh - 1 || c3 < 2 || c3 > nh - 1) {
            atomicOr(err, 1);                              // outside the base grid's differences
            return;
        }
        auto B = [&](int a, int b, int cc) {
            return (int64_t)(a - 1) + (int64_t)nh * ((int64_t)(b - 1) + (int64_t)nh * (cc - 1));
        };
        const float h = __fmul_rn(2.0f, dx0);
        const float b21 = __fdiv_rn(__fsub_rn(u2[B(c1 + 1, c2, c3)], u2[B(c1 - 1, c2, c3)]), h);
        const float b32 = __fdiv_rn(__fsub_rn(u3[B(c1, c2 + 1, c3)], u3[B(c1, c2 - 1, c3)]), h);
        const float b43 = __fdiv_rn(__fsub_rn(u4[B(c1, c2, c3 + 1)], u4[B(c1, c2, c3 - 1)]), h);
        aux = __fadd_rn(__fadd_rn(b21, b32), b43);
    }
    float v = own;
    if (i == 2 || i == n1 - 1 || j == 2 || j == n2 - 1 || k == 2 || k == n3 - 1) v = __fmul_rn(0.5f, __fadd_rn(aux, v));
    if (i == 1 || i == n1 || j == 1 || j == n2 || k == 1 || k == n3) v = aux;
    dv[t] = v;
}
// VMESH for one patch: its cells added into the level grid (patches in order)
__global__ void k_vmesh_add(PatchGeom P, int nx, int nh, int xr1, int yr1, int zr1, const float *__restrict__ u11,
                            const float *__restrict__ dv, int32_t *__restrict__ flagamr, float *__restrict__ ugr,
                            float *__restrict__ divr, uint8_t *__restrict__ flagr, int *__restrict__ err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = P.n1, n2 = P.n2;
    if (t >= (int64_t)n1 * n2 * P.n3) return;
    const int xr = xr1 + (int)(t % n1) + 1, yr = yr1 + (int)((t / n1) % n2) + 1, zr = zr1 + (int)(t / ((int64_t)n1 * n2)) + 1;
    if (xr < 1 || xr > nx || yr < 1 || yr > nx || zr < 1 || zr > nx) {
        atomicOr(err, 2);                                  // outside the level grid
        return;
    }
    const int64_t c = (int64_t)(xr - 1) + (int64_t)nx * ((int64_t)(yr - 1) + (int64_t)nx * (zr - 1));
    flagamr[c] += 1;
    ugr[c] = __fadd_rn(ugr[c], u11[P.off + t]);
    divr[c] = __fadd_rn(divr[c], dv[t]);
    flagr[(int64_t)((xr - 1) / 2) + (int64_t)nh * ((int64_t)((yr - 1) / 2) + (int64_t)nh * ((zr - 1) / 2))] = 1;
}
// the sums over FLAGAMR; the children of unrefined base cells take the base values
__global__ void k_vmesh_finish(int nx, int nh, const int32_t *__restrict__ flagamr, const uint8_t *__restrict__ flagr,
                               const float *__restrict__ u1g, const float *__restrict__ d0, float *__restrict__ ugr,
                               float *__restrict__ divr) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int64_t)nx * nx * nx) return;
    const int i = (int)(c % nx), j = (int)((c / nx) % nx), k = (int)(c / ((int64_t)nx * nx));
    const int64_t b = (int64_t)(i / 2) + (int64_t)nh * ((int64_t)(j / 2) + (int64_t)nh * (k / 2));
    if (!flagr[b]) {
        ugr[c] = u1g[b];
        divr[c] = d0[b];
    } else {
        const float f = (float)flagamr[c];
        ugr[c] = __fdiv_rn(ugr[c], f);
        divr[c] = __fdiv_rn(divr[c], f);
    }
}

static void amr_level1(Ctx &c, const Level &L, const avism_params *p, int nhy, const float *const *gas,
                       const AmrPatches &a, float *ugr, float *divr) {
    const int nx = L.g.nx, nh = nhy;
    const int64_t nc = (int64_t)nx * nx * nx, n0 = (int64_t)nh * nh * nh;
    avism_params p0 = *p;
    p0.nx = nhy;
    const Level L0 = make_level(&p0);
    const float dx0 = L0.g.dx, dxr_div = dx0 / 2.0f, dxr = L.g.dx, rx1 = L.rad_at(1);
    // IXR1 = INT(((PATCHRX - 0.5*DXR) - RX1)/DXR + 0.5) (src/amr2uniform.f90:170-172),
    // every corner checked before the first launch: a value beyond int is refused
    std::vector<int> r1(3 * (size_t)a.npatch);
    for (int q = 0; q < a.npatch; q++) {
        const float rc[3] = {a.rx[q], a.ry[q], a.rz[q]};
        for (int ax = 0; ax < 3; ax++) {
            const float f = (((rc[ax] - 0.5f * dxr) - rx1) / dxr) + 0.5f;
            AV_CHECK(std::isfinite(f) && std::fabs(f) < 1.0e9f, AVISM_ERR_ARG,
                     "MASCLET level 1: a patch corner lies far outside the level grid");
            r1[3 * (size_t)q + ax] = (int)f;
        }
    }
    float *d0 = c.get_t<float>(B_DIVER2, n0);
    AV_CUDA(cudaMemsetAsync(d0, 0, sizeof(float) * (size_t)n0, c.stream));
    if (nh > 2)
        ++c.launches, k_diver0<<<grid_for((int64_t)(nh - 2) * (nh - 2) * (nh - 2), 256), 256, 0, c.stream>>>(
            nh, dx0, gas[1], gas[2], gas[3], d0);
    for (int ax = 0; ax < 3; ax++)
        for (int side = 0; side < 2; side++)
            ++c.launches, k_diver0_face<<<grid_for((int64_t)nh * nh, 256), 256, 0, c.stream>>>(nh, ax, side, d0);
    int32_t *flagamr = c.get_t<int32_t>(B_LABEL_AUX, nc);
    uint8_t *flagr = c.get_t<uint8_t>(B_GAS4, n0);
    int *err = c.get_t<int>(B_SCAL, 4);
    AV_CUDA(cudaMemsetAsync(flagr, 0, (size_t)n0, c.stream));
    AV_CUDA(cudaMemsetAsync(ugr, 0, sizeof(float) * (size_t)nc, c.stream));
    AV_CUDA(cudaMemsetAsync(divr, 0, sizeof(float) * (size_t)nc, c.stream));
    AV_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c.stream));
    ++c.launches, k_fill_i32_1<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, flagamr);
    int64_t maxcells = 1;
    for (int q = 0; q < a.npatch; q++) maxcells = std::max(maxcells, (int64_t)a.nx[q] * a.ny[q] * a.nz[q]);
    float *dv = c.get_t<float>(B_GAS3, maxcells);
    for (int q = 0; q < a.npatch; q++) {
        PatchGeom P{a.nx[q], a.ny[q], a.nz[q], a.ix[q], a.iy[q], a.iz[q], a.offset[q]};
        const int64_t np = (int64_t)P.n1 * P.n2 * P.n3;
        if (np <= 0) continue;
        ++c.launches, k_patch_div<<<grid_for(np, 256), 256, 0, c.stream>>>(P, nh, dxr_div, dx0, a.u12g, a.u13g, a.u14g,
                                                                          gas[1], gas[2], gas[3], dv, err);
        const int xr1 = r1[3 * (size_t)q], yr1 = r1[3 * (size_t)q + 1], zr1 = r1[3 * (size_t)q + 2];
        ++c.launches, k_vmesh_add<<<grid_for(np, 256), 256, 0, c.stream>>>(P, nx, nh, xr1, yr1, zr1, a.u11g, dv,
                                                                          flagamr, ugr, divr, flagr, err);
    }
    ++c.launches, k_vmesh_finish<<<grid_for(nc, 256), 256, 0, c.stream>>>(nx, nh, flagamr, flagr, gas[0], d0, ugr,
                                                                         divr);
    AV_CUDA(cudaGetLastError());
    int herr = 0;
    AV_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    AV_CHECK(herr == 0, AVISM_ERR_ARG, "MASCLET level 1: a patch reaches outside the base grid's differences or "
                                       "the level grid (the reference reads or writes outside its arrays there)");
}

// DIVERCO = MIN(DIVERGCO, DIVERDMCO) with DIVERDMCO = 0 (levels above 0)
__global__ void k_min_zero(int64_t nc, float *__restrict__ a) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) a[c] = 0.0f < a[c] ? 0.0f : a[c];
}

float masclet_fields_inner(Ctx &c, const avism_params *p, const Level &L, int nhy, const float *const *gas,
                           const AmrPatches *amr, const float *u_mass, const float *du2, const float *du3,
                           const float *du4, float *u1co_in, float *diver_in) {
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    const bool amr1 = p->level == 1;
    const bool need_gas_v = !amr1 && (p->flag_div == 0 || p->flag_div == 2);
    const int ng = need_gas_v ? 4 : 1;
    float *co[4] = {c.get_t<float>(B_GAS1, nc), nullptr, nullptr, nullptr};
    if (need_gas_v) {
        co[1] = c.get_t<float>(B_GAS2, nc);
        co[2] = c.get_t<float>(B_GAS3, nc);
        co[3] = c.get_t<float>(B_GAS4, nc);
    }
    if (amr1) amr_level1(c, L, p, nhy, gas, *amr, co[0], diver_in);      // UGR, DIVR
    else if (p->flag_dens != 1 || need_gas_v) level_grids(c, L, p, nhy, ng, gas, co);
    const float dx = L.g.dx;
    const float vol = ((dx * dx) * dx) * ((L.g.rete * L.g.rete) * L.g.rete);
    ++c.launches, k_masclet_rho<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u_mass, co[0], vol, L.g.rote,
                                                                        p->flag_dens, u1co_in);
    AV_CUDA(cudaGetLastError());
    // MEANDENS8: the REAL*8 sum over the cells (1389-1405), U1CO / MEANDENS
    double *sum_d = c.get_t<double>(B_RED1, 1);
    cub::TransformInputIterator<double, ToDouble, const float *> it(u1co_in, ToDouble());
    size_t tmp = 0;
    AV_CUDA(cub::DeviceReduce::Sum(nullptr, tmp, it, sum_d, (int)nc, c.stream));
    AV_CUDA(cub::DeviceReduce::Sum(c.get(B_CUB_TMP, tmp), tmp, it, sum_d, (int)nc, c.stream));
    double sum = 0.0;
    AV_CUDA(cudaMemcpyAsync(&sum, sum_d, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    const float mean = (float)(sum / (double)nc);
    ++c.launches, k_div_scalar<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u1co_in, mean);
    c.mark("normalise");
    // DIVERCO by FLAG_DIV (1633-1650)
    avism_params pv = *p;
    pv.no_velocities = p->flag_div == -1 ? 1 : 0;
    if (p->flag_div == -1) {
        divergence_inner(c, &pv, L, u1co_in, nullptr, nullptr, nullptr, diver_in);
    } else if (amr1) {
        // DIVERGCO = DIVR (in diver_in), DIVERDMCO = 0
        if (p->flag_div == 1) AV_CUDA(cudaMemsetAsync(diver_in, 0, sizeof(float) * (size_t)nc, c.stream));
        if (p->flag_div == 0) ++c.launches, k_min_zero<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, diver_in);
    } else {
        if (need_gas_v) divergence_inner(c, &pv, L, u1co_in, co[1], co[2], co[3], diver_in);
        if (p->flag_div == 1) divergence_inner(c, &pv, L, u1co_in, du2, du3, du4, diver_in);
        if (p->flag_div == 0) {
            float *dd = c.get_t<float>(B_DIVER2, nc);
            divergence_inner(c, &pv, L, u1co_in, du2, du3, du4, dd);
            ++c.launches, k_min_into<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, diver_in, dd);
        }
    }
    AV_CUDA(cudaGetLastError());
    const float ul3 = (UL_F * UL_F) * UL_F;
    return mean * (UM_F / ul3);
}

__global__ void k_ext_copy(int nx, int low1, int ne, const float *__restrict__ inner, float *__restrict__ ext) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ne3 = (int64_t)ne * ne * ne;
    if (e >= ne3) return;
    int i = (int)(e % ne) + low1, j = (int)((e / ne) % ne) + low1, k = (int)(e / ((int64_t)ne * ne)) + low1;
    if (i < 1) i += nx; else if (i > nx) i -= nx;
    if (j < 1) j += nx; else if (j > nx) j -= nx;
    if (k < 1) k += nx; else if (k > nx) k -= nx;
    ext[e] = inner[(int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1))];
}

void ext_copy(Ctx &c, const Level &L, const float *inner, float *ext) {
    const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
    ++c.launches, k_ext_copy<<<grid_for(ne3, 256), 256, 0, c.stream>>>(L.g.nx, L.g.low1, L.g.ne, inner, ext);
    AV_CUDA(cudaGetLastError());
}

// Smallest float d with f32(f64(d) / (2*f64(dx))) >= G: the gradient test
// DDENS = (U(n+1)-U(n-1))/(2.D0*DDX) >= GRAD_THRE of src/voidfinding.f90:290
// is a monotone function of the f32 difference, so it reduces to d >= D*.
static inline int32_t f2ord(float f) {
    int32_t i;
    std::memcpy(&i, &f, 4);
    return i >= 0 ? i : (int32_t)(0x80000000u - (uint32_t)i) ;
}
static inline float ord2f(int32_t o) {
    int32_t i = o >= 0 ? o : (int32_t)(0x80000000u - (uint32_t)o);
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
static float grad_threshold(float G, float dx) {
    auto test = [&](float d) { return (float)((double)d / (2.0 * (double)dx)) >= G; };
    int64_t lo = f2ord(-INFINITY), hi = f2ord(INFINITY);
    if (test(ord2f((int32_t)lo))) return -INFINITY;
    if (!test(ord2f((int32_t)hi))) return NAN;          // never true
    while (hi - lo > 1) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (test(ord2f((int32_t)mid))) hi = mid; else lo = mid;
    }
    return ord2f((int32_t)hi);
}

struct FlagArgs {
    int nx, low1, low2, ne, ext;
    const float *u1, *dv;
    const int8_t *smask;
    const int32_t *marcap;
    float dens1, dens2, div_thre, gthr;  // DENS_THRE+1, DENS_THRE2+1, DIV_THRE, D*
};

__device__ __forceinline__ int64_t fl_index(const FlagArgs &A, int i, int j, int k) {
    if (A.ext)
        return (int64_t)(i - A.low1) + (int64_t)A.ne * ((int64_t)(j - A.low1) + (int64_t)A.ne * (k - A.low1));
    const int nx = A.nx;
    if (i < 1) i += nx; else if (i > nx) i -= nx;
    if (j < 1) j += nx; else if (j > nx) j -= nx;
    if (k < 1) k += nx; else if (k > nx) k -= nx;
    return (int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1));
}

// one direction of the flag loop; -1 = masked neighbour (CYCLE ends the cell)
__device__ __forceinline__ int dir_flag(const FlagArgs &A, const int c[3], int axis, int sgn) {
    const int pos = c[axis];
    if (sgn > 0 ? pos >= A.low2 - 1 : pos <= A.low1 + 1) return 1;
    int nb[3] = {c[0], c[1], c[2]};
    const int ii = pos + sgn;
    nb[axis] = ii;
    const int64_t en_ext = (int64_t)(nb[0] - A.low1) + (int64_t)A.ne * ((int64_t)(nb[1] - A.low1) + (int64_t)A.ne * (nb[2] - A.low1));
    if (A.smask && A.smask[en_ext] == 0) return -1;
    const int64_t en = fl_index(A, nb[0], nb[1], nb[2]);
    const float u_n = A.u1[en], d_n = A.dv[en];
    int f = 0;
    if (ii == (sgn > 0 ? A.low2 : A.low1)) {
        if (d_n < A.div_thre) f = 1;
        if (u_n >= A.dens2) f = 1;
        return f;
    }
    int a[3] = {nb[0], nb[1], nb[2]}, b[3] = {nb[0], nb[1], nb[2]};
    a[axis] = ii + sgn;
    b[axis] = ii - sgn;
    const float d1 = __fsub_rn(A.u1[fl_index(A, a[0], a[1], a[2])], A.u1[fl_index(A, b[0], b[1], b[2])]);
    if (d1 >= A.gthr) f = 1;
    if (f == 1 && (sgn > 0 ? ii < A.low2 - 1 : ii > A.low1 + 1)) {
        int a2[3] = {nb[0], nb[1], nb[2]};
        a2[axis] = ii + 2 * sgn;
        const float d2 = __fsub_rn(A.u1[fl_index(A, a2[0], a2[1], a2[2])], u_n);
        if (d2 < A.gthr) f = 0;
    }
    if (d_n < A.div_thre) f = 1;
    if (u_n >= A.dens2) f = 1;
    return f;
}

// flag byte of ext cell e at coordinates c (LOW1..LOW2)
__device__ __forceinline__ uint8_t flag_byte(const FlagArgs &A, int64_t e, const int c[3]) {
    uint8_t f = 0;
    const int32_t mp = A.marcap ? A.marcap[e] : -1;
    if ((!A.smask || A.smask[e] != 0) && mp != 0) {
        f |= 0x80;
        const int64_t ci = fl_index(A, c[0], c[1], c[2]);
        if (A.u1[ci] < A.dens1 && A.dv[ci] > 0.0f) f |= 0x01;
    }
    // +X, -X, +Y, -Y, +Z, -Z; bits X1=1 X2=2 Y1=3 Y2=4 Z1=5 Z2=6
    const int axs[6] = {0, 0, 1, 1, 2, 2};
    const int sgs[6] = {1, -1, 1, -1, 1, -1};
    const int bits[6] = {2, 1, 4, 3, 6, 5};
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const int r = dir_flag(A, c, axs[d], sgs[d]);
        if (r < 0) break;
        if (r) f |= (uint8_t)(1u << bits[d]);
    }
    return f;
}

__global__ void k_flags(FlagArgs A, uint8_t *__restrict__ flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = A.ne;
    if (e >= (int64_t)ne * ne * ne) return;
    const int c[3] = {(int)(e % ne) + A.low1, (int)((e / ne) % ne) + A.low1, (int)(e / ((int64_t)ne * ne)) + A.low1};
    flags[e] = flag_byte(A, e, c);
}

// ---- flags of the periodic inner grid, spread to the ext grid -------------------
// Away from the ext grid's faces (every coordinate at least 4 cells inside
// LOW1..LOW2) a cell's flag byte depends only on U1CO and DIVERCO at wrapped
// positions, so it equals the byte of the inner cell it wraps to (no mask, no
// parent map).  k_flags_inner computes those inner bytes once: a CTA holds a
// 32 x 8 column of cells and marches it along z, with a ring of 7 U1CO planes
// (+-3 halo) and 3 DIVERCO planes (+-1 halo) in shared memory.  k_flags_spread
// and k_flags_shell then write the ext grid.
constexpr int FL_TX = 32, FL_TY = 8, FL_TZ = 32, FL_H = 3;
constexpr int FL_UX = FL_TX + 2 * FL_H, FL_UY = FL_TY + 2 * FL_H;
constexpr int FL_DX = FL_TX + 2, FL_DY = FL_TY + 2;
constexpr int FL_UN = FL_UX * FL_UY, FL_DN = FL_DX * FL_DY;

__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__global__ void __launch_bounds__(FL_TX * FL_TY)
k_flags_inner(FlagArgs A, uint8_t *__restrict__ fin) {
    __shared__ float su[7][FL_UY][FL_UX];
    __shared__ float sd[3][FL_DY][FL_DX];
    const int nx = A.nx;
    const int ntx = nx / FL_TX, nty = nx / FL_TY;
    const int bx = (int)(blockIdx.x % ntx), by = (int)((blockIdx.x / ntx) % nty), bz = (int)(blockIdx.x / (ntx * nty));
    const int X0 = bx * FL_TX, Y0 = by * FL_TY, Z0 = bz * FL_TZ;
    const int tid = threadIdx.x, lx = tid % FL_TX, ly = tid / FL_TX;
    const int64_t plane = (int64_t)nx * nx;
    // in-plane offsets of this thread's halo loads (fixed for every plane)
    int64_t uo[3], dof[2];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const int e = tid + r * FL_TX * FL_TY;
        const int hx = e % FL_UX, hy = e / FL_UX;
        uo[r] = e < FL_UN ? (int64_t)wrapn(X0 - FL_H + hx, nx) + (int64_t)nx * wrapn(Y0 - FL_H + hy, nx) : -1;
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int e = tid + r * FL_TX * FL_TY;
        const int hx = e % FL_DX, hy = e / FL_DX;
        dof[r] = e < FL_DN ? (int64_t)wrapn(X0 - 1 + hx, nx) + (int64_t)nx * wrapn(Y0 - 1 + hy, nx) : -1;
    }
    auto load_u = [&](int z) {
        const int slot = (z - Z0 + FL_H) % 7;
        const float *src = A.u1 + plane * wrapn(z, nx);
        float *dst = &su[slot][0][0];
#pragma unroll
        for (int r = 0; r < 3; r++)
            if (uo[r] >= 0) dst[tid + r * FL_TX * FL_TY] = src[uo[r]];
    };
    auto load_d = [&](int z) {
        const int slot = (z - Z0 + 1) % 3;
        const float *src = A.dv + plane * wrapn(z, nx);
        float *dst = &sd[slot][0][0];
#pragma unroll
        for (int r = 0; r < 2; r++)
            if (dof[r] >= 0) dst[tid + r * FL_TX * FL_TY] = src[dof[r]];
    };
    for (int z = Z0 - FL_H; z < Z0 + FL_H; z++) load_u(z);
    load_d(Z0 - 1);
    load_d(Z0);
    for (int z = Z0; z < Z0 + FL_TZ; z++) {
        load_u(z + FL_H);
        load_d(z + 1);
        __syncthreads();
        auto U = [&](int dx, int dy, int dz) { return su[(z + dz - Z0 + FL_H) % 7][ly + FL_H + dy][lx + FL_H + dx]; };
        auto D = [&](int dx, int dy, int dz) { return sd[(z + dz - Z0 + 1) % 3][ly + 1 + dy][lx + 1 + dx]; };
        uint8_t f = 0x80;                                        // FLAG_SUB: no mask, no parent map
        if (U(0, 0, 0) < A.dens1 && D(0, 0, 0) > 0.0f) f |= 0x01;
        // +X, -X, +Y, -Y, +Z, -Z -> bits 2, 1, 4, 3, 6, 5
#pragma unroll
        for (int d = 0; d < 6; d++) {
            const int ax = d >> 1, sg = (d & 1) ? -1 : 1;
            const int ex = ax == 0 ? sg : 0, ey = ax == 1 ? sg : 0, ez = ax == 2 ? sg : 0;
            const float un = U(ex, ey, ez), dn = D(ex, ey, ez);
            int fl = __fsub_rn(U(2 * ex, 2 * ey, 2 * ez), U(0, 0, 0)) >= A.gthr;
            if (fl && __fsub_rn(U(3 * ex, 3 * ey, 3 * ez), un) < A.gthr) fl = 0;
            if (dn < A.div_thre) fl = 1;
            if (un >= A.dens2) fl = 1;
            const int bit = 2 * ax + (sg > 0 ? 2 : 1);
            if (fl) f |= (uint8_t)(1u << bit);
        }
        fin[(int64_t)(X0 + lx) + (int64_t)nx * (Y0 + ly) + plane * z] = f;
        __syncthreads();
    }
}

// The ext grid in two launches.  k_flags_spread writes every cell at least 4
// cells inside the faces from the inner byte it wraps to, 16 consecutive cells
// of a row per thread (one 16-byte load and store when both sides are aligned);
// k_flags_shell computes the faces' 4-cell shell directly, one cell per thread,
// so the heavier shell bytes do not hold up the copies.
__global__ void k_flags_spread(FlagArgs A, const uint8_t *__restrict__ fin, uint8_t *__restrict__ flags) {
    const int ne = A.ne, nx = A.nx;
    const int nch = (ne + 15) / 16;
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (int64_t)nch * (ne - 8) * (ne - 8)) return;
    const int ch = (int)(g % nch), y = 4 + (int)((g / nch) % (ne - 8)), z = 4 + (int)(g / ((int64_t)nch * (ne - 8)));
    const int i0 = ch * 16;
    const int cy = y + A.low1, cz = z + A.low1;
    int wy = cy, wz = cz;
    if (wy < 1) wy += nx; else if (wy > nx) wy -= nx;
    if (wz < 1) wz += nx; else if (wz > nx) wz -= nx;
    const uint8_t *frow = fin + (int64_t)nx * ((wy - 1) + (int64_t)nx * (wz - 1));
    uint8_t *erow = flags + (int64_t)ne * (y + (int64_t)ne * z);
    const int cx0 = i0 + A.low1;
    int w0 = cx0;
    if (w0 < 1) w0 += nx; else if (w0 > nx) w0 -= nx;
    if (i0 >= 4 && i0 + 16 <= ne - 4 && w0 + 15 <= nx && (reinterpret_cast<uintptr_t>(frow + w0 - 1) & 15) == 0 &&
        (reinterpret_cast<uintptr_t>(erow + i0) & 15) == 0) {
        *reinterpret_cast<uint4 *>(erow + i0) = *reinterpret_cast<const uint4 *>(frow + w0 - 1);
        return;
    }
    const int a = max(i0, 4), b = min(i0 + 16, ne - 4);
    for (int i = a; i < b; i++) {
        int wx = i + A.low1;
        if (wx < 1) wx += nx; else if (wx > nx) wx -= nx;
        erow[i] = frow[wx - 1];
    }
}

// the cells within 4 of a face: z slabs, then y slabs of the remaining planes,
// then x slabs of the remaining rows
__global__ void k_flags_shell(FlagArgs A, uint8_t *__restrict__ flags) {
    const int ne = A.ne, m = ne - 8;
    const int64_t nzs = 8 * (int64_t)ne * ne, nys = 8 * (int64_t)ne * m, nxs = 8 * (int64_t)m * m;
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (g < nzs) {
        x = (int)(g % ne); y = (int)((g / ne) % ne);
        const int s = (int)(g / ((int64_t)ne * ne));
        z = s < 4 ? s : ne - 8 + s;
    } else if ((g -= nzs) < nys) {
        x = (int)(g % ne);
        const int s = (int)((g / ne) % 8);
        y = s < 4 ? s : ne - 8 + s;
        z = 4 + (int)(g / (8 * (int64_t)ne));
    } else if ((g -= nys) < nxs) {
        const int s = (int)(g % 8);
        x = s < 4 ? s : ne - 8 + s;
        y = 4 + (int)((g / 8) % m);
        z = 4 + (int)(g / (8 * (int64_t)m));
    } else {
        return;
    }
    const int c[3] = {x + A.low1, y + A.low1, z + A.low1};
    const int64_t e = (int64_t)x + (int64_t)ne * (y + (int64_t)ne * z);
    flags[e] = flag_byte(A, e, c);
}

void make_flags(Ctx &c, const avism_params *p, const Level &L, const float *u1, const float *dv,
                int fields_are_ext, const int8_t *smask_ext, const int32_t *marcap_ext, uint8_t *flags) {
    FlagArgs A;
    A.nx = L.g.nx; A.low1 = L.g.low1; A.low2 = L.g.low2; A.ne = L.g.ne; A.ext = fields_are_ext;
    A.u1 = u1; A.dv = dv; A.smask = smask_ext; A.marcap = marcap_ext;
    A.dens1 = p->dens_thre + 1.0f;
    A.dens2 = p->dens_thre2 + 1.0f;
    A.div_thre = p->div_thre;
    A.gthr = grad_threshold(p->grad_thre, L.g.dx);
    const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
    const int nx = L.g.nx;
    const bool tiled = !fields_are_ext && !smask_ext && !marcap_ext && nx % FL_TX == 0 && nx % FL_TY == 0 &&
                       nx % FL_TZ == 0 && L.g.ne < 65536;
    if (tiled) {
        uint8_t *fin = c.get_t<uint8_t>(B_FLAGS_IN, (size_t)nx * nx * nx);
        const unsigned ntiles = (unsigned)((nx / FL_TX) * (nx / FL_TY) * (nx / FL_TZ));
        ++c.launches, k_flags_inner<<<ntiles, FL_TX * FL_TY, 0, c.stream>>>(A, fin);
        const int64_t ne = L.g.ne, m = ne - 8;
        const int64_t nth = ((ne + 15) / 16) * m * m;
        ++c.launches, k_flags_spread<<<grid_for(nth, 256), 256, 0, c.stream>>>(A, fin, flags);
        const int64_t nshell = 8 * ne * ne + 8 * ne * m + 8 * m * m;
        ++c.launches, k_flags_shell<<<grid_for(nshell, 256), 256, 0, c.stream>>>(A, flags);
    } else {
        ++c.launches, k_flags<<<grid_for(ne3, 256), 256, 0, c.stream>>>(A, flags);
    }
    AV_CUDA(cudaGetLastError());
}

}  // namespace avism
