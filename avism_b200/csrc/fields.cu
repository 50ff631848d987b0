// fields.cu -- density normalisation, divergence, ghost shell and the
// per-cell flag byte of MARK_ALL / VOIDFIND.
//
// Replaces src/avism.f90:1249-1250 and 1384-1411 (rho/rho_B, FP64 mean,
// rho/<rho>), DIVER_UNIFORM (src/divergence.f90:2-50), REAL_MAKE_PERIODIC
// (src/num.f90:89-133), MARK_ALL (src/voidfinding.f90:13-55) and the six
// directional flag grids of VOIDFIND (src/voidfinding.f90:256-432).
//
// The ext grid is never materialised on the hot path: ghost cells read the
// inner grids at wrapped coordinates.  Flags are packed into one byte per ext
// cell: bit0 FLAGV, bit1 X1, bit2 X2, bit3 Y1, bit4 Y2, bit5 Z1, bit6 Z2,
// bit7 FLAG_SUB.
#include <cub/cub.cuh>
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

struct ToDouble {
    __host__ __device__ double operator()(float v) const { return (double)v; }
};

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

FieldsOut fields_inner(Ctx &c, const avism_params *p, const Level &L, const float *u_mass,
                       const float *u2, const float *u3, const float *u4, float *u1co_in,
                       float *diver_in) {
    const int nx = L.g.nx;
    const int64_t nc = (int64_t)nx * nx * nx;
    const float dx = L.g.dx;
    const float vol = ((dx * dx) * dx) * ((L.g.rete * L.g.rete) * L.g.rete);
    ++c.launches, k_rho<<<grid_for(nc, 256), 256, 0, c.stream>>>(nc, u_mass, vol, L.g.rote, u1co_in);
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
    ++c.launches, k_diver<<<grid_for(nc, 256), 256, 0, c.stream>>>(nx, dx, p->periodic, u2, u3, u4, diver_in);
    AV_CUDA(cudaGetLastError());
    FieldsOut o;
    const float ul3 = (UL_F * UL_F) * UL_F;
    o.meandens = mean * (UM_F / ul3);
    return o;
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

__global__ void k_flags(FlagArgs A, uint8_t *__restrict__ flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = A.ne;
    if (e >= (int64_t)ne * ne * ne) return;
    const int c[3] = {(int)(e % ne) + A.low1, (int)((e / ne) % ne) + A.low1, (int)(e / ((int64_t)ne * ne)) + A.low1};
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
    flags[e] = f;
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
    ++c.launches, k_flags<<<grid_for(ne3, 256), 256, 0, c.stream>>>(A, flags);
    AV_CUDA(cudaGetLastError());
}

}  // namespace avism
