// proposal.cu -- the learned proposal: multi-scale features of the particle
// bins, a 12 -> 64 -> 64 -> 64 -> 2 ReLU MLP with BF16 weights and FP32
// accumulation, its training kernels and its tcgen05 inference kernel.
//
// No counterpart in the reference (AVISM has no learned part).  The network
// predicts, per particle bin, (0) the log of the K-th neighbour distance of a
// query at the bin, in bin widths, and (1) log(1 + w) of the half-width w of a
// cube grown from a centre in the bin.  Output 0 is the starting radius of the
// warp kNN (knn_warp.cuh) and output 1 the first shell the growth checks in
// one sweep (voidfind.cu); both are verified exactly there, so the predictions
// change the amount of work only, never a result.
//
// Features (12 per bin), from a pyramid of bin sums at cell sizes 1, 2, 4, 8
// bins (levels 0..3): per level, log(0.05 + N / (occ * 8^l)) (density), the
// central-difference divergence of the mean velocity in units of v_rms / bw,
// and the magnitude of the central-difference gradient of the density
// contrast.
//
// Parameter vector (float32, PR_NPARAM entries): mu[12], sigma[12],
// W1[64][12], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[2][64], b4[2],
// slack[2].  Forward: a0 = bf16((x - mu) / sigma); a_l = bf16(relu(W_l a + b_l))
// with W_l rounded to bf16 and FP32 sums; y = W4 a3 + b4.
#include <cub/cub.cuh>
#include <cuda_bf16.h>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "knn_core.cuh"
#include "bin_kernels.cuh"

namespace avism {

constexpr int PR_NF = 12, PR_H = 64, PR_NO = 2;
constexpr int PR_OFF_MU = 0, PR_OFF_SIG = 12, PR_OFF_W1 = 24, PR_OFF_B1 = PR_OFF_W1 + PR_H * PR_NF;
constexpr int PR_OFF_W2 = PR_OFF_B1 + PR_H, PR_OFF_B2 = PR_OFF_W2 + PR_H * PR_H;
constexpr int PR_OFF_W3 = PR_OFF_B2 + PR_H, PR_OFF_B3 = PR_OFF_W3 + PR_H * PR_H;
constexpr int PR_OFF_W4 = PR_OFF_B3 + PR_H, PR_OFF_B4 = PR_OFF_W4 + PR_NO * PR_H;
constexpr int PR_OFF_SLACK = PR_OFF_B4 + PR_NO;
constexpr int PR_NPARAM = PR_OFF_SLACK + 2;
static_assert(PR_NPARAM == 9308 && PR_NPARAM == PROPOSAL_NPARAM, "parameter layout");
constexpr int PR_LEVELS = 4;

__host__ __device__ __forceinline__ float bf16_round(float v) {
    return __bfloat162float(__float2bfloat16_rn(v));
}

// ---- feature pyramid ----------------------------------------------------------
// level l has nbl = ceil(nb / 2^l) cells per axis; each holds (count, sum vx,
// sum vy, sum vz) of the particles of its bins.
struct Pyramid {
    float4 *lev[PR_LEVELS];
    int nbl[PR_LEVELS];
    const float *cbox[4];     // counts summed over the centred (2w+1)^3 bins, w = 0, 1, 2, 4
    int periodic;
    float occ;            // mean particles per bin
    float inv_vscale;     // bw / v_rms
    int div_at_mean;      // inference: the divergence inputs held at their training mean
};
__host__ __device__ constexpr int box_w(int s) { return s == 0 ? 0 : (s == 1 ? 1 : (s == 2 ? 2 : 4)); }

__global__ void k_pyr_base(KnnGrid G, const float4 *__restrict__ sv, float4 *__restrict__ out) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nb3 = (int64_t)G.nb * G.nb * G.nb;
    if (b >= nb3) return;
    float n = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
    for (int64_t p = G.start[b]; p < G.start[b + 1]; p++) {
        const float4 a = sv[p];
        n += 1.f;
        sx += a.x;
        sy += a.y;
        sz += a.z;
    }
    out[b] = make_float4(n, sx, sy, sz);
}

__global__ void k_pyr_down(const float4 *__restrict__ in, int nin, float4 *__restrict__ out, int nout) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int64_t)nout * nout * nout) return;
    const int x = (int)(c % nout), y = (int)((c / nout) % nout), z = (int)(c / ((int64_t)nout * nout));
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
                if (X >= nin || Y >= nin || Z >= nin) continue;
                const float4 v = in[X + (int64_t)nin * (Y + (int64_t)nin * Z)];
                s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
            }
    out[c] = s;
}

__device__ __forceinline__ int pyr_wrap(int i, int n, int periodic) {
    if (periodic) return i < 0 ? i + n : (i >= n ? i - n : i);
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

__device__ __forceinline__ float4 pyr_at(const Pyramid &P, int l, int x, int y, int z) {
    const int n = P.nbl[l];
    x = pyr_wrap(x, n, P.periodic);
    y = pyr_wrap(y, n, P.periodic);
    z = pyr_wrap(z, n, P.periodic);
    return P.lev[l][(uint32_t)x + (uint32_t)n * ((uint32_t)y + (uint32_t)n * (uint32_t)z)];
}

__global__ void k_counts(int64_t nb3, const float4 *__restrict__ lev0, float *__restrict__ cnt) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb3) cnt[b] = lev0[b].x;
}
// the same counts straight from the bins' offsets (no attributes needed)
__global__ void k_bin_counts(int64_t nb3, const int64_t *__restrict__ start, float *__restrict__ cnt) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb3) cnt[b] = (float)(start[b + 1] - start[b]);
}

// one separable pass of the (2w+1)-wide box sums along `axis` (wrapped or
// clamped) for the three half-widths w = 1, 2, 4 at once (in[s] -> out[s]);
// grid (ceil(nb / blockDim), nb, nb), x along threads
struct Box3 {
    const float *in[3];
    float *out[3];
};
__global__ void k_box_pass3(int nb, int axis, int periodic, Box3 B) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nb) return;
    const int c[3] = {x, (int)blockIdx.y, (int)blockIdx.z};
    const int64_t b = (int64_t)x + (int64_t)nb * (blockIdx.y + (int64_t)nb * blockIdx.z);
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? nb : (int64_t)nb * nb);
#pragma unroll
    for (int s = 0; s < 3; s++) {
        const int w = box_w(s + 1);
        float acc = 0.f;
#pragma unroll
        for (int d = -w; d <= w; d++) {
            int q = c[axis] + d;
            if (q < 0 || q >= nb) {
                if (!periodic) continue;
                q = q < 0 ? q + nb : q - nb;
            }
            acc += B.in[s][b + (int64_t)(q - c[axis]) * stride];
        }
        B.out[s][b] = acc;
    }
}

__device__ __forceinline__ float cbox_at(const Pyramid &P, int s, int nb, int x, int y, int z) {
    x = pyr_wrap(x, nb, P.periodic);
    y = pyr_wrap(y, nb, P.periodic);
    z = pyr_wrap(z, nb, P.periodic);
    return P.cbox[s][(uint32_t)x + (uint32_t)nb * ((uint32_t)y + (uint32_t)nb * (uint32_t)z)];
}

// The 12 features of bin (bx, by, bz): f0..f3 the log density of the centred
// (2w+1)^3 boxes, w = 0, 1, 2, 4; f4..f7 the magnitude of their central
// density gradient over +-max(w, 1) bins; f8..f11 the velocity divergence of
// the pyramid cells of 1, 2, 4, 8 bins, in units of v_rms / bw.
__device__ void bin_features(const Pyramid &P, int nb, int bx, int by, int bz, float f[PR_NF]) {
    // features only steer where a search starts, so fast intrinsics are used;
    // training and inference share this function
    const float inv_occ = 1.0f / P.occ;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int w = box_w(s), sp = w > 0 ? w : 1;
        const float inv_vol = inv_occ / (float)((2 * w + 1) * (2 * w + 1) * (2 * w + 1));
        f[s] = __logf(0.05f + cbox_at(P, s, nb, bx, by, bz) * inv_vol);
        const float gx = cbox_at(P, s, nb, bx + sp, by, bz) - cbox_at(P, s, nb, bx - sp, by, bz);
        const float gy = cbox_at(P, s, nb, bx, by + sp, bz) - cbox_at(P, s, nb, bx, by - sp, bz);
        const float gz = cbox_at(P, s, nb, bx, by, bz + sp) - cbox_at(P, s, nb, bx, by, bz - sp);
        f[4 + s] = sqrtf(gx * gx + gy * gy + gz * gz) * (inv_vol * (0.5f / (float)sp));
    }
    if (P.div_at_mean) {
#pragma unroll
        for (int l = 0; l < PR_LEVELS; l++) f[8 + l] = 0.f;
        return;
    }
#pragma unroll
    for (int l = 0; l < PR_LEVELS; l++) {
        const int x = bx >> l, y = by >> l, z = bz >> l;
        float div = 0.f;
        const int d[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int a = 0; a < 3; a++) {
            const float4 p = pyr_at(P, l, x + d[a][0], y + d[a][1], z + d[a][2]);
            const float4 m = pyr_at(P, l, x - d[a][0], y - d[a][1], z - d[a][2]);
            const float vp = a == 0 ? p.y : a == 1 ? p.z : p.w, vm = a == 0 ? m.y : a == 1 ? m.z : m.w;
            const float up = p.x > 0.f ? __fdividef(vp, p.x) : 0.f, um = m.x > 0.f ? __fdividef(vm, m.x) : 0.f;
            div += up - um;
        }
        f[8 + l] = div * (P.inv_vscale * (0.5f / (float)(1 << l)));
    }
}

__global__ void k_features(Pyramid P, int nb, float *__restrict__ feat) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= (int64_t)nb * nb * nb) return;
    float f[PR_NF];
    bin_features(P, nb, (int)(b % nb), (int)((b / nb) % nb), (int)(b / ((int64_t)nb * nb)), f);
    for (int i = 0; i < PR_NF; i++) feat[b * PR_NF + i] = f[i];
}

// ---- training kernels (FP32 CUDA cores, fixed summation order) -------------------
// a0 = bf16((x - mu) / sigma), 16 wide (12 features + 4 zeros)
__global__ void k_tr_input(int B, const float *__restrict__ feat, const int32_t *__restrict__ idx,
                           const float *__restrict__ prm, float *__restrict__ a0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * 16) return;
    const int s = t / 16, k = t % 16;
    float v = 0.f;
    if (k < PR_NF) v = bf16_round(__fdiv_rn(__fsub_rn(feat[(int64_t)idx[s] * PR_NF + k], prm[PR_OFF_MU + k]),
                                            prm[PR_OFF_SIG + k]));
    a0[t] = v;
}

// z[s][o] = b[o] + sum_k bf16(W[o][k]) a[s][k]; out = bf16(relu(z)) (hidden) or z (last)
__global__ void k_tr_fwd(int B, int fin, int astride, int fout, const float *__restrict__ a, const float *__restrict__ W,
                         const float *__restrict__ bias, float *__restrict__ z, float *__restrict__ out, int last) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * fout) return;
    const int s = t / fout, o = t % fout;
    float acc = 0.f;
    for (int k = 0; k < fin; k++) acc = __fadd_rn(acc, __fmul_rn(bf16_round(W[o * fin + k]), a[(int64_t)s * astride + k]));
    acc = __fadd_rn(acc, bias[o]);
    z[t] = acc;
    out[t] = last ? acc : bf16_round(fmaxf(acc, 0.f));
}

// dy = 2 m (y - t) / den; per-sample loss terms
__global__ void k_tr_dy(int B, const float *__restrict__ y, const int32_t *__restrict__ idx,
                        const float *__restrict__ tgt, const float *__restrict__ msk, float inv_den,
                        float *__restrict__ dy, float *__restrict__ ls) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    float l = 0.f;
    for (int j = 0; j < PR_NO; j++) {
        const int64_t g = (int64_t)idx[s] * PR_NO + j;
        const float r = __fmul_rn(__fsub_rn(y[s * PR_NO + j], tgt[g]), msk[g]);
        dy[s * PR_NO + j] = __fmul_rn(__fmul_rn(2.f, r), inv_den);
        l = __fadd_rn(l, __fmul_rn(r, __fsub_rn(y[s * PR_NO + j], tgt[g])));
    }
    ls[s] = l;
}

// da[s][k] = sum_o bf16(W[o][k]) dz[s][o]; optionally dz of the layer below = da * (z > 0)
__global__ void k_tr_bwd_act(int B, int fin, int fout, const float *__restrict__ W, const float *__restrict__ dz,
                             const float *__restrict__ zbelow, float *__restrict__ dzbelow) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B * fin) return;
    const int s = t / fin, k = t % fin;
    float acc = 0.f;
    for (int o = 0; o < fout; o++) acc = __fadd_rn(acc, __fmul_rn(bf16_round(W[o * fin + k]), dz[s * fout + o]));
    dzbelow[t] = zbelow[t] > 0.f ? acc : 0.f;
}

// dW[o][k] = sum_s dz[s][o] a[s][k]; db[o] = sum_s dz[s][o]
__global__ void k_tr_gradw(int B, int fin, int astride, int fout, const float *__restrict__ a,
                           const float *__restrict__ dz, float *__restrict__ gW, float *__restrict__ gb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= fout * (fin + 1)) return;
    const int o = t / (fin + 1), k = t % (fin + 1);
    float acc = 0.f;
    if (k < fin) {
        for (int s = 0; s < B; s++) acc = __fadd_rn(acc, __fmul_rn(dz[s * fout + o], a[(int64_t)s * astride + k]));
        gW[o * fin + k] = acc;
    } else {
        for (int s = 0; s < B; s++) acc = __fadd_rn(acc, dz[s * fout + o]);
        gb[o] = acc;
    }
}

__global__ void k_tr_sum(int n, const float *__restrict__ v, float *__restrict__ out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; i++) s = __fadd_rn(s, v[i]);
        *out = s;
    }
}

// Adam on the trainable range [PR_OFF_W1, PR_OFF_SLACK)
__global__ void k_tr_adam(float *__restrict__ prm, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, float lr, float c1, float c2) {
    const int i = PR_OFF_W1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= PR_OFF_SLACK) return;
    const float b1 = 0.9f, b2 = 0.999f;
    m[i] = b1 * m[i] + (1.f - b1) * g[i];
    v[i] = b2 * v[i] + (1.f - b2) * g[i] * g[i];
    const float mh = m[i] / c1, vh = v[i] / c2;
    prm[i] = prm[i] - lr * mh / (sqrtf(vh) + 1e-8f);
}

struct TrainBufs {
    float *a0, *z1, *a1, *z2, *a2, *z3, *a3, *y, *dy, *dz3, *dz2, *dz1, *ls, *scal;
};

// forward + backward of one batch; grad receives the full gradient vector
static void tr_fwd_bwd(Ctx &c, int B, const float *feat, const int32_t *idx, const float *tgt, const float *msk,
                       float inv_den, const float *prm, float *grad, const TrainBufs &T) {
    const int TB = 256;
    ++c.launches, k_tr_input<<<grid_for((int64_t)B * 16, TB), TB, 0, c.stream>>>(B, feat, idx, prm, T.a0);
    ++c.launches, k_tr_fwd<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_NF, 16, PR_H, T.a0, prm + PR_OFF_W1, prm + PR_OFF_B1, T.z1, T.a1, 0);
    ++c.launches, k_tr_fwd<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_H, T.a1, prm + PR_OFF_W2, prm + PR_OFF_B2, T.z2, T.a2, 0);
    ++c.launches, k_tr_fwd<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_H, T.a2, prm + PR_OFF_W3, prm + PR_OFF_B3, T.z3, T.a3, 0);
    ++c.launches, k_tr_fwd<<<grid_for((int64_t)B * PR_NO, TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_NO, T.a3, prm + PR_OFF_W4, prm + PR_OFF_B4, T.y, T.y, 1);
    ++c.launches, k_tr_dy<<<grid_for(B, TB), TB, 0, c.stream>>>(B, T.y, idx, tgt, msk, inv_den, T.dy, T.ls);
    ++c.launches, k_tr_sum<<<1, 32, 0, c.stream>>>(B, T.ls, T.scal);
    AV_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * PR_NPARAM, c.stream));
    ++c.launches, k_tr_gradw<<<grid_for(PR_NO * (PR_H + 1), TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_NO, T.a3, T.dy, grad + PR_OFF_W4, grad + PR_OFF_B4);
    ++c.launches, k_tr_bwd_act<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_H, PR_NO, prm + PR_OFF_W4, T.dy, T.z3, T.dz3);
    ++c.launches, k_tr_gradw<<<grid_for(PR_H * (PR_H + 1), TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_H, T.a2, T.dz3, grad + PR_OFF_W3, grad + PR_OFF_B3);
    ++c.launches, k_tr_bwd_act<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_H, PR_H, prm + PR_OFF_W3, T.dz3, T.z2, T.dz2);
    ++c.launches, k_tr_gradw<<<grid_for(PR_H * (PR_H + 1), TB), TB, 0, c.stream>>>(B, PR_H, PR_H, PR_H, T.a1, T.dz2, grad + PR_OFF_W2, grad + PR_OFF_B2);
    ++c.launches, k_tr_bwd_act<<<grid_for((int64_t)B * PR_H, TB), TB, 0, c.stream>>>(B, PR_H, PR_H, prm + PR_OFF_W2, T.dz2, T.z1, T.dz1);
    ++c.launches, k_tr_gradw<<<grid_for(PR_H * (PR_NF + 1), TB), TB, 0, c.stream>>>(B, PR_NF, 16, PR_H, T.a0, T.dz1, grad + PR_OFF_W1, grad + PR_OFF_B1);
    AV_CUDA(cudaGetLastError());
}

static TrainBufs train_bufs(Ctx &c, int B) {
    const size_t per = (size_t)B * (16 + 7 * PR_H + 2 * PR_NO + 3 * PR_H + 1) + 16;
    float *base = c.get_t<float>(B_PR_TRAIN, per);
    TrainBufs T;
    float *p = base;
    auto take = [&](size_t n) { float *r = p; p += n; return r; };
    T.a0 = take((size_t)B * 16);
    T.z1 = take((size_t)B * PR_H); T.a1 = take((size_t)B * PR_H);
    T.z2 = take((size_t)B * PR_H); T.a2 = take((size_t)B * PR_H);
    T.z3 = take((size_t)B * PR_H); T.a3 = take((size_t)B * PR_H);
    T.y = take((size_t)B * PR_NO); T.dy = take((size_t)B * PR_NO);
    T.dz3 = take((size_t)B * PR_H); T.dz2 = take((size_t)B * PR_H); T.dz1 = take((size_t)B * PR_H);
    T.ls = take((size_t)B);
    T.scal = take(16);
    return T;
}

// one forward + backward over samples [0, ns) as one batch (the gradient check)
void proposal_grad(Ctx &c, int64_t ns, const float *feat, const float *tgt, const float *msk, const float *prm,
                   float *grad, float *loss) {
    AV_CHECK(ns >= 1 && ns <= (1 << 20), AVISM_ERR_ARG, "proposal_grad: 1 <= ns <= 2^20");
    const int B = (int)ns;
    TrainBufs T = train_bufs(c, B);
    std::vector<int32_t> hidx(B);
    for (int i = 0; i < B; i++) hidx[i] = i;
    int32_t *idx = c.get_t<int32_t>(B_PR_IDX, B);
    AV_CUDA(cudaMemcpyAsync(idx, hidx.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, c.stream));
    // the loss is normalised by the mask count
    std::vector<float> hm((size_t)B * PR_NO);
    AV_CUDA(cudaMemcpyAsync(hm.data(), msk, sizeof(float) * hm.size(), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    double den = 0.0;
    for (float v : hm) den += v;
    const float inv_den = (float)(1.0 / std::max(1.0, den));
    tr_fwd_bwd(c, B, feat, idx, tgt, msk, inv_den, prm, grad, T);
    float l = 0.f;
    AV_CUDA(cudaMemcpyAsync(&l, T.scal, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    *loss = l * inv_den;
}

// Adam over random mini-batches (seeded LCG over the sample set)
void proposal_train(Ctx &c, int64_t ns, const float *feat, const float *tgt, const float *msk, int steps, int batch,
                    float lr, uint32_t seed, float *prm, float *loss_curve) {
    AV_CHECK(ns >= 1 && ns < INT32_MAX && batch >= 1 && batch <= (1 << 20) && steps >= 0, AVISM_ERR_ARG,
             "proposal_train: bad sizes");
    const int B = batch;
    TrainBufs T = train_bufs(c, B);
    float *grad = c.get_t<float>(B_PR_GRAD, 3 * (size_t)PR_NPARAM);
    float *m = grad + PR_NPARAM, *v = grad + 2 * PR_NPARAM;
    AV_CUDA(cudaMemsetAsync(m, 0, sizeof(float) * 2 * PR_NPARAM, c.stream));
    int32_t *idx = c.get_t<int32_t>(B_PR_IDX, (size_t)B * 2);
    std::vector<int32_t> hidx(B);
    // per-sample mask counts are near constant per batch; use the expected count
    std::vector<float> hm((size_t)ns * PR_NO);
    AV_CUDA(cudaMemcpyAsync(hm.data(), msk, sizeof(float) * hm.size(), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    double msum = 0.0;
    for (float x : hm) msum += x;
    const float inv_den = (float)(1.0 / std::max(1.0, msum * (double)B / (double)ns));
    uint64_t st = 0x9E3779B97F4A7C15ULL ^ seed;
    std::vector<float> curve;
    for (int s = 1; s <= steps; s++) {
        for (int i = 0; i < B; i++) {
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            hidx[i] = (int32_t)((st >> 33) % (uint64_t)ns);
        }
        int32_t *ib = idx + (size_t)(s & 1) * B;
        AV_CUDA(cudaMemcpyAsync(ib, hidx.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice, c.stream));
        tr_fwd_bwd(c, B, feat, ib, tgt, msk, inv_den, prm, grad, T);
        const float c1 = 1.f - std::pow(0.9f, (float)s), c2 = 1.f - std::pow(0.999f, (float)s);
        const int ntr = PR_OFF_SLACK - PR_OFF_W1;
        ++c.launches, k_tr_adam<<<grid_for(ntr, 256), 256, 0, c.stream>>>(prm, grad, m, v, lr, c1, c2);
        if (loss_curve) {
            float l = 0.f;
            AV_CUDA(cudaMemcpyAsync(&l, T.scal, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
            c.sync();     // hidx is reused by the next step's copy
            loss_curve[s - 1] = l * inv_den;
        } else {
            c.sync();
        }
    }
    AV_CUDA(cudaGetLastError());
}

// ---- inference on the tensor cores (tcgen05, one CTA = 128 rows per tile) ---------
// Shared-memory operands use the no-swizzle K-major canonical layout: 8-row x
// 16-byte core matrices; core (row group g, k group j) of a tile with K
// columns sits at byte (g * K/8 + j) * 128.  LBO = 128 (next k group), SBO =
// K/8 * 128 (next row group).
constexpr int TC_M = 128;
constexpr int TC_THREADS = 128;
constexpr uint32_t TC_WAIT_LIMIT = 1u << 22;      // mbarrier polls before giving up

struct __align__(1024) TcSmem {
    __nv_bfloat16 a0[2][TC_M * 16];     // input tiles, K = 16 (double buffered)
    __nv_bfloat16 a1[TC_M * PR_H];      // hidden activations: each epilogue overwrites the
                                        // layer input its MMA has finished reading
    __nv_bfloat16 w1[PR_H * 16];        // W1, N = 64 rows, K = 16
    __nv_bfloat16 w2[PR_H * PR_H];
    __nv_bfloat16 w3[PR_H * PR_H];
    __nv_bfloat16 w4[16 * PR_H];        // W4 padded to N = 16
    float b1[PR_H], b2[PR_H], b3[PR_H], b4[2];
    float mu[PR_NF], isg[PR_NF];
    uint64_t mbar;                      // MMA completion
    uint64_t mbar_in[2];                // input tile arrival
    uint32_t tmem_base;
};

// element (r, k) of a K-major no-swizzle tile with K columns
__host__ __device__ __forceinline__ int tc_off(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t tc_desc(const void *p, uint32_t lbo, uint32_t sbo) {
    const uint64_t a = smem_u32(p);
    return ((a & 0x3FFFFull) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

// bounded wait on the mbarrier phase; false when the limit was reached
__device__ __forceinline__ bool tc_wait(uint64_t *mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < TC_WAIT_LIMIT; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive f32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// normalised bf16 features of every bin, written tile by tile (128 rows, 4 KB)
// in the input operand's core-matrix layout, so the MLP copies a tile as is
__global__ void k_features_tiles(Pyramid P, int nb, const float *__restrict__ mu, const float *__restrict__ sig,
                                 __nv_bfloat16 *__restrict__ tiles) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nb3 = (int64_t)nb * nb * nb;
    const int64_t ntile_rows = (nb3 + TC_M - 1) / TC_M * TC_M;
    if (b >= ntile_rows) return;
    float f[PR_NF];
    if (b < nb3) {
        const uint32_t u = (uint32_t)b, un = (uint32_t)nb, q = u / un;     // nb^3 < 2^32
        bin_features(P, nb, (int)(u - q * un), (int)(q % un), (int)(q / un), f);
    }
    __align__(16) __nv_bfloat16 v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const float x = (k < PR_NF && b < nb3 && !(P.div_at_mean && k >= 8))
                            ? __fdiv_rn(__fsub_rn(f[k], mu[k]), sig[k]) : 0.f;
        v[k] = __float2bfloat16_rn(x);
    }
    __nv_bfloat16 *t = tiles + (b / TC_M) * (TC_M * 16);
    const int r = (int)(b % TC_M);
    *reinterpret_cast<uint4 *>(t + tc_off(r, 0, 16)) = *reinterpret_cast<const uint4 *>(&v[0]);
    *reinterpret_cast<uint4 *>(t + tc_off(r, 8, 16)) = *reinterpret_cast<const uint4 *>(&v[8]);
}

// packed bf16 weights in the core-matrix layout + f32 biases, built once per load
struct TcWeights {
    __nv_bfloat16 w1[PR_H * 16], w2[PR_H * PR_H], w3[PR_H * PR_H], w4[16 * PR_H];
    float b1[PR_H], b2[PR_H], b3[PR_H], b4[2], mu[PR_NF], isg[PR_NF];
    float slack[2];
};

__global__ void k_pack_weights(const float *__restrict__ prm, TcWeights *__restrict__ W) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < PR_H * 16) {
        const int r = t / 16, k = t % 16;
        W->w1[tc_off(r, k, 16)] = __float2bfloat16_rn(k < PR_NF ? prm[PR_OFF_W1 + r * PR_NF + k] : 0.f);
    }
    if (t < PR_H * PR_H) {
        const int r = t / PR_H, k = t % PR_H;
        W->w2[tc_off(r, k, PR_H)] = __float2bfloat16_rn(prm[PR_OFF_W2 + t]);
        W->w3[tc_off(r, k, PR_H)] = __float2bfloat16_rn(prm[PR_OFF_W3 + t]);
    }
    if (t < 16 * PR_H) {
        const int r = t / PR_H, k = t % PR_H;
        W->w4[tc_off(r, k, PR_H)] = __float2bfloat16_rn(r < PR_NO ? prm[PR_OFF_W4 + r * PR_H + k] : 0.f);
    }
    if (t < PR_H) {
        W->b1[t] = prm[PR_OFF_B1 + t];
        W->b2[t] = prm[PR_OFF_B2 + t];
        W->b3[t] = prm[PR_OFF_B3 + t];
    }
    if (t < PR_NO) W->b4[t] = prm[PR_OFF_B4 + t];
    if (t < PR_NF) {
        W->mu[t] = prm[PR_OFF_MU + t];
        W->isg[t] = prm[PR_OFF_SIG + t];
    }
    if (t < 2) W->slack[t] = prm[PR_OFF_SLACK + t];
}

// where the rows come from and where the outputs go
struct TcIO {
    int64_t nrows;
    const float *feat;         // [nrows][12] raw features, or null: use tiles
    const __nv_bfloat16 *tiles;  // normalised bf16 rows in 4 KB core-matrix tiles (k_features_tiles)
    float *out;                // [nrows][2] raw outputs, or null
    float *r0;                 // [nrows] starting kNN radius bw * exp(y0) * slack0, or null
    float *w0;                 // [nrows] predicted half-width exp(y1) - 1 + slack1, or null
    float bw;
    int *err;                  // set to 1 when a bounded wait gave up
};

// 16 consecutive f32 columns of this thread's TMEM lane, without the wait
__device__ __forceinline__ void tc_ld16_issue(uint32_t taddr, uint32_t r[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// hidden layer epilogue: D (this thread's row, 64 columns, read from TMEM in
// four loads and one wait) + bias -> relu -> bf16 tile
__device__ __forceinline__ void tc_hidden(uint32_t taddr, const float *bias, __nv_bfloat16 *dst, int row) {
    uint32_t r[PR_H];
#pragma unroll
    for (int c0 = 0; c0 < PR_H; c0 += 16) tc_ld16_issue(taddr + c0, r + c0);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c0 = 0; c0 < PR_H; c0 += 16) {
        __align__(16) __nv_bfloat16 o[16];
#pragma unroll
        for (int i = 0; i < 16; i++)
            o[i] = __float2bfloat16_rn(fmaxf(__fadd_rn(__uint_as_float(r[c0 + i]), bias[c0 + i]), 0.f));
        *reinterpret_cast<uint4 *>(dst + tc_off(row, c0, PR_H)) = *reinterpret_cast<const uint4 *>(&o[0]);
        *reinterpret_cast<uint4 *>(dst + tc_off(row, c0 + 8, PR_H)) = *reinterpret_cast<const uint4 *>(&o[8]);
    }
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(mbar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(mbar)) : "memory");
}

__global__ void __launch_bounds__(TC_THREADS)
k_mlp_tc(TcIO io, const TcWeights *__restrict__ Wg) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem &S = *reinterpret_cast<TcSmem *>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights -> shared memory (once per CTA)
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(Wg->w1);
        uint4 *d1 = reinterpret_cast<uint4 *>(S.w1);
        for (int i = tid; i < (int)(sizeof(S.w1) / 16); i += TC_THREADS) d1[i] = src[i];
        src = reinterpret_cast<const uint4 *>(Wg->w2);
        uint4 *d2 = reinterpret_cast<uint4 *>(S.w2);
        for (int i = tid; i < (int)(sizeof(S.w2) / 16); i += TC_THREADS) d2[i] = src[i];
        src = reinterpret_cast<const uint4 *>(Wg->w3);
        uint4 *d3 = reinterpret_cast<uint4 *>(S.w3);
        for (int i = tid; i < (int)(sizeof(S.w3) / 16); i += TC_THREADS) d3[i] = src[i];
        src = reinterpret_cast<const uint4 *>(Wg->w4);
        uint4 *d4 = reinterpret_cast<uint4 *>(S.w4);
        for (int i = tid; i < (int)(sizeof(S.w4) / 16); i += TC_THREADS) d4[i] = src[i];
        for (int i = tid; i < PR_H; i += TC_THREADS) { S.b1[i] = Wg->b1[i]; S.b2[i] = Wg->b2[i]; S.b3[i] = Wg->b3[i]; }
        if (tid < PR_NO) S.b4[tid] = Wg->b4[tid];
        if (tid < PR_NF) { S.mu[tid] = Wg->mu[tid]; S.isg[tid] = Wg->isg[tid]; }
    }
    const int64_t ntiles = (io.nrows + TC_M - 1) / TC_M;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar_in[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar_in[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (io.tiles && (int64_t)blockIdx.x < ntiles)
            bulk_load(S.a0[0], io.tiles + (int64_t)blockIdx.x * TC_M * 16, TC_M * 16 * 2, &S.mbar_in[0]);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&S.tmem_base)), "r"(64) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const float slack0 = Wg->slack[0], slack1 = Wg->slack[1];
    uint32_t phase = 0;
    bool ok = true;
    int it = 0;
    const uint64_t dw1 = tc_desc(S.w1, 128, 2 * 128), dw2 = tc_desc(S.w2, 128, 8 * 128);
    const uint64_t dw3 = tc_desc(S.w3, 128, 8 * 128), dw4 = tc_desc(S.w4, 128, 8 * 128);
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, it++) {
        const int64_t row = tile * TC_M + tid;
        const int buf = it & 1;
        __nv_bfloat16 *a0 = S.a0[buf];
        if (io.tiles) {
            // this tile was prefetched; start the next one into the other buffer
            ok = __syncthreads_and(tc_wait(&S.mbar_in[buf], (uint32_t)(it >> 1) & 1u));
            if (!ok) break;
            if (tid == 0 && tile + gridDim.x < ntiles)
                bulk_load(S.a0[buf ^ 1], io.tiles + (tile + gridDim.x) * TC_M * 16, TC_M * 16 * 2, &S.mbar_in[buf ^ 1]);
        } else {
            // raw feature rows: normalise -> bf16
            float f[PR_NF];
            for (int i = 0; i < PR_NF; i++) f[i] = row < io.nrows ? io.feat[row * PR_NF + i] : 0.f;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const float v = k < PR_NF ? __fdiv_rn(__fsub_rn(f[k], S.mu[k]), S.isg[k]) : 0.f;
                a0[tc_off(tid, k, 16)] = __float2bfloat16_rn(row < io.nrows ? v : 0.f);
            }
            fence_async_smem();
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // ---- layer 1: K = 16
        if (tid == 0) {
            tc_mma(tmem, tc_desc(a0, 128, 2 * 128), dw1, tc_idesc(TC_M, PR_H), 0);
            tc_commit(&S.mbar);
        }
        ok = __syncthreads_and(tc_wait(&S.mbar, phase));
        phase ^= 1;
        tc_fence_after();
        if (!ok) break;
        tc_hidden(lane_addr, S.b1, S.a1, tid);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // ---- layers 2 and 3: K = 64 as four K = 16 steps
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                tc_mma(tmem, tc_desc(S.a1 + s * 128, 128, 8 * 128), tc_desc(S.w2 + s * 128, 128, 8 * 128),
                       tc_idesc(TC_M, PR_H), s > 0);
            tc_commit(&S.mbar);
        }
        ok = __syncthreads_and(tc_wait(&S.mbar, phase));
        phase ^= 1;
        tc_fence_after();
        if (!ok) break;
        tc_hidden(lane_addr, S.b2, S.a1, tid);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                tc_mma(tmem, tc_desc(S.a1 + s * 128, 128, 8 * 128), tc_desc(S.w3 + s * 128, 128, 8 * 128),
                       tc_idesc(TC_M, PR_H), s > 0);
            tc_commit(&S.mbar);
        }
        ok = __syncthreads_and(tc_wait(&S.mbar, phase));
        phase ^= 1;
        tc_fence_after();
        if (!ok) break;
        tc_hidden(lane_addr, S.b3, S.a1, tid);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // ---- layer 4: N = 16 (two real outputs)
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                tc_mma(tmem, tc_desc(S.a1 + s * 128, 128, 8 * 128), tc_desc(S.w4 + s * 128, 128, 8 * 128),
                       tc_idesc(TC_M, 16), s > 0);
            tc_commit(&S.mbar);
        }
        ok = __syncthreads_and(tc_wait(&S.mbar, phase));
        phase ^= 1;
        tc_fence_after();
        if (!ok) break;
        float v[16];
        tc_ld16(lane_addr, v);
        const float y0 = __fadd_rn(v[0], S.b4[0]), y1 = __fadd_rn(v[1], S.b4[1]);
        if (row < io.nrows) {
            if (io.out) { io.out[row * 2] = y0; io.out[row * 2 + 1] = y1; }
            if (io.r0) io.r0[row] = io.bw * expf(fminf(y0, 8.f)) * slack0;
            if (io.w0) io.w0[row] = expf(fminf(y1, 8.f)) - 1.f + slack1;
        }
        // every thread has read its accumulator before the next tile's MMA
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (!ok) {
        if (tid == 0) atomicExch(io.err, 1);
        tc_wait(&S.mbar, phase);      // let an MMA still in flight finish (bounded)
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(64) : "memory");
}

static TcWeights *pack_weights(Ctx &c, const float *prm_dev, BufId id = B_PR_PACKED_TMP) {
    TcWeights *W = (TcWeights *)c.get(id, sizeof(TcWeights));
    ++c.launches, k_pack_weights<<<grid_for(PR_H * PR_H, 256), 256, 0, c.stream>>>(prm_dev, W);
    AV_CUDA(cudaGetLastError());
    return W;
}

static void run_mlp_tc(Ctx &c, TcIO io, const TcWeights *W) {
    if (io.nrows == 0) return;
    const size_t sm = sizeof(TcSmem) + 1024;
    AV_CUDA(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int *err = c.get_t<int>(B_PR_ERR, 4);
    AV_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c.stream));
    io.err = err;
    const int64_t ntiles = (io.nrows + TC_M - 1) / TC_M;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, (int64_t)c.num_sms * 4);
    ++c.launches, k_mlp_tc<<<grid, TC_THREADS, sm, c.stream>>>(io, W);
    AV_CUDA(cudaGetLastError());
    int herr = 0;
    AV_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    AV_CHECK(herr == 0, AVISM_ERR_TIMEOUT, "proposal MLP: a tensor-core wait timed out");
}

// raw outputs for explicit feature rows (test entry point)
void proposal_infer(Ctx &c, int64_t ns, const float *feat, const float *prm_dev, float *out) {
    AV_CHECK(ns >= 0, AVISM_ERR_ARG, "proposal_infer: ns < 0");
    const TcWeights *W = pack_weights(c, prm_dev);
    TcIO io{};
    io.nrows = ns;
    io.feat = feat;
    io.out = out;
    run_mlp_tc(c, io, W);
}

struct V2Op {
    __host__ __device__ double operator()(const float4 &a) const {
        return (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z;
    }
};

// sv null: the density features only (the bins' counts), the divergence inputs
// held at their training mean; otherwise all twelve from the velocity pyramid
Pyramid build_pyramid(Ctx &c, const KnnGrid &G, const float4 *sv, int64_t n) {
    Pyramid P{};
    P.periodic = G.periodic;
    P.occ = G.occ;
    P.div_at_mean = sv ? 0 : 1;
    const int64_t nb3 = (int64_t)G.nb * G.nb * G.nb;
    float *cnt = c.get_t<float>(B_PR_CNT, (size_t)nb3);
    if (sv) {
        int nbl = G.nb;
        for (int l = 0; l < PR_LEVELS; l++) {
            P.nbl[l] = nbl;
            P.lev[l] = c.get_t<float4>((BufId)(B_PR_PYR0 + l), (size_t)nbl * nbl * nbl);
            nbl = (nbl + 1) / 2;
        }
        ++c.launches, k_pyr_base<<<grid_for(nb3, 256), 256, 0, c.stream>>>(G, sv, P.lev[0]);
        for (int l = 1; l < PR_LEVELS; l++) {
            const int64_t n3 = (int64_t)P.nbl[l] * P.nbl[l] * P.nbl[l];
            ++c.launches, k_pyr_down<<<grid_for(n3, 256), 256, 0, c.stream>>>(P.lev[l - 1], P.nbl[l - 1], P.lev[l],
                                                                              P.nbl[l]);
        }
        ++c.launches, k_counts<<<grid_for(nb3, 256), 256, 0, c.stream>>>(nb3, P.lev[0], cnt);
    } else {
        ++c.launches, k_bin_counts<<<grid_for(nb3, 256), 256, 0, c.stream>>>(nb3, G.start, cnt);
    }
    // centred box counts: three separable passes, each for all half-widths
    float *ta = c.get_t<float>(B_PR_TMPA, (size_t)nb3), *tb = c.get_t<float>(B_PR_TMPB, (size_t)nb3);
    P.cbox[0] = cnt;
    const BufId bid[3] = {B_PR_BOX1, B_PR_BOX2, B_PR_BOX4};
    const dim3 bg((unsigned)((G.nb + 127) / 128), (unsigned)G.nb, (unsigned)G.nb);
    {
        // x: counts -> the three outputs; y: outputs -> temporaries; z: back
        float *out[3], *tmp[3] = {ta, tb, c.get_t<float>(B_PR_TMPC, (size_t)nb3)};
        for (int s = 0; s < 3; s++) out[s] = c.get_t<float>(bid[s], (size_t)nb3);
        Box3 bx{{cnt, cnt, cnt}, {out[0], out[1], out[2]}};
        Box3 by{{out[0], out[1], out[2]}, {tmp[0], tmp[1], tmp[2]}};
        Box3 bz{{tmp[0], tmp[1], tmp[2]}, {out[0], out[1], out[2]}};
        ++c.launches, k_box_pass3<<<bg, 128, 0, c.stream>>>(G.nb, 0, G.periodic, bx);
        ++c.launches, k_box_pass3<<<bg, 128, 0, c.stream>>>(G.nb, 1, G.periodic, by);
        ++c.launches, k_box_pass3<<<bg, 128, 0, c.stream>>>(G.nb, 2, G.periodic, bz);
        for (int s = 1; s < 4; s++) P.cbox[s] = out[s - 1];
    }
    // velocity scale of the divergence features: v_rms of the particles
    if (sv) {
        double *d = c.get_t<double>(B_RED1, 1);
        auto it = cub::TransformInputIterator<double, V2Op, const float4 *>(sv, V2Op());
        size_t tmp = 0;
        AV_CUDA(cub::DeviceReduce::Sum(nullptr, tmp, it, d, (int)n, c.stream));
        void *t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceReduce::Sum(t, tmp, it, d, (int)n, c.stream));
        double s = 0.0;
        AV_CUDA(cudaMemcpyAsync(&s, d, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        const double vrms = std::sqrt(std::max(s / std::max<int64_t>(n, 1), 1e-30));
        P.inv_vscale = (float)((double)G.bw / vrms);
    }
    AV_CUDA(cudaGetLastError());
    return P;
}

void proposal_load(Ctx &c, const float *params_dev) {
    pack_weights(c, params_dev, B_PR_PACKED);
    c.sync();
    c.prop_loaded = true;
}

// the binning of particles_to_grid and its features, one row per bin
void proposal_features(Ctx &c, const avism_params *p, const P2G &a, float *feat_dev, int *nb_out, float *bw_out) {
    const char *occ_env = getenv("AVISM_TUNE_OCC");
    const float occ = occ_env ? (float)atof(occ_env) : 2.0f;
    BinnedParticles bp = bin_particles(c, a.n, a.x, a.y, a.z, p->lado0, p->periodic, occ);
    KnnGrid G = make_knn_grid(bp);
    *nb_out = bp.nb;
    *bw_out = bp.bw;
    if (!feat_dev) return;
    float4 *sv = c.get_t<float4>(B_SV, std::max<int64_t>(a.n, 1));
    c.attrs_ready();
    if (a.n > 0)
        ++c.launches, k_sorted_attrs<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, G.sp, a.vx, a.vy, a.vz, a.m, sv);
    Pyramid P = build_pyramid(c, G, sv, a.n);
    const int64_t nb3 = (int64_t)bp.nb * bp.nb * bp.nb;
    ++c.launches, k_features<<<grid_for(nb3, 256), 256, 0, c.stream>>>(P, bp.nb, feat_dev);
    AV_CUDA(cudaGetLastError());
}

// per-bin starting radius (and half-width) for a level: the density features
// from the bins' counts, the velocity-divergence inputs held at their training
// mean, fused into the tensor-core MLP.  The prediction then needs the
// positions only, so a level's velocities can still be in flight (their
// inputs gave no measurable saving in the kNN stages: 155.4 / 209.8 ms against
// 155.5 / 210.1 ms with them at 512^3 / 2^27 particles)
void proposal_predict(Ctx &c, const KnnGrid &G, float *r0, float *w0) {
    AV_CHECK(c.prop_loaded, AVISM_ERR_ARG,
             "learned proposal requested but no weights are loaded (avism_gpu_proposal_load)");
    Pyramid P = build_pyramid(c, G, nullptr, 0);
    const int64_t nb3 = (int64_t)G.nb * G.nb * G.nb;
    const int64_t rows = (nb3 + TC_M - 1) / TC_M * TC_M;
    __nv_bfloat16 *tiles = c.get_t<__nv_bfloat16>(B_PR_FEAT, (size_t)rows * 16);
    const TcWeights *W = (const TcWeights *)c.buf[B_PR_PACKED];
    ++c.launches, k_features_tiles<<<grid_for(rows, 256), 256, 0, c.stream>>>(P, G.nb, W->mu, W->isg, tiles);
    AV_CUDA(cudaGetLastError());
    c.mark("features");
    TcIO io{};
    io.nrows = nb3;
    io.feat = nullptr;
    io.tiles = tiles;
    io.r0 = r0;
    io.w0 = w0;
    io.bw = G.bw;
    run_mlp_tc(c, io, W);
}

}  // namespace avism
