// capi.cu -- the extern "C" entry points declared in include/avism_gpu.h.
#include <cub/cub.cuh>
#include <cstring>
#include <exception>
#include <vector>

#include "common.cuh"

struct avism_gpu_ctx {
    avism::Ctx c;
};

using namespace avism;

namespace {

int fail(avism_gpu_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->c.last_error = msg;
    return code;
}

template <class F>
int guarded(avism_gpu_ctx *ctx, F &&f) {
    if (!ctx) return AVISM_ERR_ARG;
    try {
        AV_CUDA(cudaSetDevice(ctx->c.device));
        ctx->c.stage_open();
        f(ctx->c);
        sv_velocities(ctx->c);
        ctx->c.attrs_ready();
        ctx->c.mark("end");
        ctx->c.stage_close();
        ctx->c.last_error.clear();
        return AVISM_OK;
    } catch (const Error &e) {
        cudaGetLastError();
        ctx->c.drop_pending_copies();
        ctx->c.stage_close();
        return fail(ctx, e.code, e.msg);
    } catch (const std::bad_alloc &) {
        ctx->c.drop_pending_copies();
        return fail(ctx, AVISM_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        ctx->c.drop_pending_copies();
        return fail(ctx, AVISM_ERR_INTERNAL, e.what());
    }
}

struct Timer {
    Ctx &c;
    cudaEvent_t a, b;
    explicit Timer(Ctx &cc) : c(cc) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, c.stream);
    }
    void lap() {
        cudaEventRecord(b, c.stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        c.stage_ms.push_back(ms);
        std::swap(a, b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// copies packed device cube arrays into the caller's avism_cubes
// the caller's cube arrays: device ones from the device records, host ones from
// the host copy (h, a HostCubes view of the same records)
void cubes_out(Ctx &c, const CubesDev &d, const avism_cubes &h, int32_t nvoid, avism_cubes *o) {
    int32_t *ints[10] = {o->inicio_x, o->final_x, o->inicio_y, o->final_y, o->inicio_z, o->final_z,
                         o->icx, o->icy, o->icz, o->father};
    float *flts[7] = {o->vol, o->rini_x, o->rfin_x, o->rini_y, o->rfin_y, o->rini_z, o->rfin_z};
    const int32_t *hi[10] = {h.inicio_x, h.final_x, h.inicio_y, h.final_y, h.inicio_z, h.final_z,
                             h.icx, h.icy, h.icz, h.father};
    const float *hf[7] = {h.vol, h.rini_x, h.rfin_x, h.rini_y, h.rfin_y, h.rini_z, h.rfin_z};
    auto one = [&](void *dst, const void *dev, const void *host, size_t bytes) {
        if (!dst || bytes == 0) return;
        if (is_device_ptr(dst)) AV_CUDA(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToDevice, c.stream));
        else std::memcpy(dst, host, bytes);
    };
    for (int k = 0; k < 10; k++) one(ints[k], d.i32 + (size_t)k * d.cap, hi[k], sizeof(int32_t) * (size_t)nvoid);
    for (int k = 0; k < 7; k++) one(flts[k], d.f32 + (size_t)k * d.cap, hf[k], sizeof(float) * (size_t)nvoid);
    c.sync();
}

// host copy of caller cube arrays (host or device memory)
struct HostCubes {
    std::vector<int32_t> i[10];
    std::vector<float> f[7];
    avism_cubes v;
    HostCubes(Ctx &c, const avism_cubes *in, int32_t n) {
        const int32_t *ints[10] = {in->inicio_x, in->final_x, in->inicio_y, in->final_y, in->inicio_z,
                                   in->final_z, in->icx, in->icy, in->icz, in->father};
        const float *flts[7] = {in->vol, in->rini_x, in->rfin_x, in->rini_y, in->rfin_y, in->rini_z, in->rfin_z};
        for (int k = 0; k < 10; k++) {
            AV_CHECK(ints[k] != nullptr || n == 0, AVISM_ERR_ARG, "null cube array");
            i[k].resize(std::max(n, 1));
            if (n) AV_CUDA(cudaMemcpyAsync(i[k].data(), ints[k], sizeof(int32_t) * n, cudaMemcpyDefault, c.stream));
        }
        for (int k = 0; k < 7; k++) {
            AV_CHECK(flts[k] != nullptr || n == 0, AVISM_ERR_ARG, "null cube array");
            f[k].resize(std::max(n, 1));
            if (n) AV_CUDA(cudaMemcpyAsync(f[k].data(), flts[k], sizeof(float) * n, cudaMemcpyDefault, c.stream));
        }
        c.sync();
        int32_t **vi[10] = {&v.inicio_x, &v.final_x, &v.inicio_y, &v.final_y, &v.inicio_z, &v.final_z,
                            &v.icx, &v.icy, &v.icz, &v.father};
        float **vf[7] = {&v.vol, &v.rini_x, &v.rfin_x, &v.rini_y, &v.rfin_y, &v.rini_z, &v.rfin_z};
        for (int k = 0; k < 10; k++) *vi[k] = i[k].data();
        for (int k = 0; k < 7; k++) *vf[k] = f[k].data();
    }
    // the device cube records (17 columns at stride cap) in two strided copies
    // into the context's pinned buffer, which the view then points into
    HostCubes(Ctx &c, const CubesDev &d, int32_t n) {
        const size_t cb = sizeof(int32_t) * (size_t)std::max(n, 1);
        char *h = (char *)c.host_pinned(17 * cb);
        if (n) {
            AV_CUDA(cudaMemcpy2DAsync(h, cb, d.i32, sizeof(int32_t) * (size_t)d.cap, cb, 10, cudaMemcpyDeviceToHost,
                                      c.stream));
            AV_CUDA(cudaMemcpy2DAsync(h + 10 * cb, cb, d.f32, sizeof(float) * (size_t)d.cap, cb, 7,
                                      cudaMemcpyDeviceToHost, c.stream));
            c.sync();
        }
        int32_t **vi[10] = {&v.inicio_x, &v.final_x, &v.inicio_y, &v.final_y, &v.inicio_z, &v.final_z,
                            &v.icx, &v.icy, &v.icz, &v.father};
        float **vf[7] = {&v.vol, &v.rini_x, &v.rfin_x, &v.rini_y, &v.rfin_y, &v.rini_z, &v.rfin_z};
        for (int k = 0; k < 10; k++) *vi[k] = reinterpret_cast<int32_t *>(h + k * cb);
        for (int k = 0; k < 7; k++) *vf[k] = reinterpret_cast<float *>(h + (10 + k) * cb);
    }
};

__global__ void k_inner_from_ext(int nx, int low1, int ne, const float *ext, float *inner) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int64_t)nx * nx * nx) return;
    const int i = (int)(c % nx) + 1, j = (int)((c / nx) % nx) + 1, k = (int)(c / ((int64_t)nx * nx)) + 1;
    inner[c] = ext[(int64_t)(i - low1) + (int64_t)ne * ((int64_t)(j - low1) + (int64_t)ne * (k - low1))];
}

P2G p2g_args(Ctx &c, const avism_params *p, const Level &L, int64_t n, const float *x, const float *y,
             const float *z, const float *vx, const float *vy, const float *vz, const float *m,
             const int8_t *smask, bool particle_out = true) {
    const size_t nb = sizeof(float) * (size_t)std::max<int64_t>(n, 1);
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    P2G a;
    a.n = n;
    a.x = (const float *)to_device(c, B_PX, x, nb);
    a.y = (const float *)to_device(c, B_PY, y, nb);
    a.z = (const float *)to_device(c, B_PZ, z, nb);
    if (p->no_velocities && !(vx && vy && vz)) {
        // READ_BINARY_PART_2 input: no velocities; zeros stand in for them
        float *zv = c.get_t<float>(B_PVX, (size_t)std::max<int64_t>(n, 1));
        AV_CUDA(cudaMemsetAsync(zv, 0, nb, c.stream));
        vx = vy = vz = zv;
    }
    // the attributes on the copy stream, after the positions' copies (the link
    // is shared): the masses first, then the velocities.  Binning's keys and
    // sort run meanwhile; every reader of a.m first calls c.mass_ready() (or
    // attrs_ready()), every reader of a.v* c.attrs_ready()
    const bool host_attr = (m && !is_device_ptr(m)) || (vx && !is_device_ptr(vx)) || (vy && !is_device_ptr(vy)) ||
                           (vz && !is_device_ptr(vz));
    if (host_attr) {
        AV_CUDA(cudaEventRecord(c.ev_pos, c.stream));
        AV_CUDA(cudaStreamWaitEvent(c.copy_stream, c.ev_pos, 0));
    }
    a.m = (const float *)to_device_on(c, c.copy_stream, B_PM, m, nb);
    if (host_attr) {
        AV_CUDA(cudaEventRecord(c.ev_mass, c.copy_stream));
        c.mass_pending = true;
    }
    a.vx = (const float *)to_device_on(c, c.copy_stream, B_PVX, vx, nb);
    a.vy = (const float *)to_device_on(c, c.copy_stream, B_PVY, vy, nb);
    a.vz = (const float *)to_device_on(c, c.copy_stream, B_PVZ, vz, nb);
    if (host_attr) {
        AV_CUDA(cudaEventRecord(c.ev_attr, c.copy_stream));
        c.attr_pending = true;
    }
    a.smask = (const int8_t *)to_device(c, B_SMASK, smask, (size_t)nc);
    a.u_mass = c.get_t<float>(B_UMASS, nc);
    a.u2 = c.get_t<float>(B_U2, nc);
    a.u3 = c.get_t<float>(B_U3, nc);
    a.u4 = c.get_t<float>(B_U4, nc);
    // per-particle outputs in input order, only when the caller wants them
    a.hpart = particle_out ? c.get_t<float>(B_HPART, std::max<int64_t>(n, 1)) : nullptr;
    a.part_dens = particle_out ? c.get_t<float>(B_PDENS, std::max<int64_t>(n, 1)) : nullptr;
    AV_CHECK(x && y && z && m && vx && vy && vz, AVISM_ERR_ARG, "null particle array");
    return a;
}

void check_params(const avism_params *p) {
    AV_CHECK(p != nullptr, AVISM_ERR_ARG, "null params");
    AV_CHECK(p->nx >= 4 && p->lado0 > 0.0f, AVISM_ERR_ARG, "nx >= 4 and lado0 > 0 required");
    AV_CHECK(p->periodic == 0 || p->periodic == 1, AVISM_ERR_ARG, "FLAG_PERIOD must be 0 or 1");
    AV_CHECK(p->flag_vel_interp == 0 || p->flag_vel_interp == 1, AVISM_ERR_ARG, "FLAG_VEL_INTERP must be 0 or 1");
    AV_CHECK(p->flag_dens_interp == 0 || p->flag_dens_interp == 1, AVISM_ERR_ARG, "FLAG_DENS_INTERP must be 0 or 1");
    AV_CHECK(p->nvoid_max >= 1, AVISM_ERR_ARG, "NVOID_MAX must be positive");
    AV_CHECK(p->kernel_mode >= 0 && p->kernel_mode <= 2, AVISM_ERR_ARG, "KERNEL_MODE must be 1 (M4) or 2 (Gaussian)");
    AV_CHECK(p->no_velocities == 0 || p->no_velocities == 1, AVISM_ERR_ARG, "no_velocities must be 0 or 1");
    AV_CHECK(p->flag_dens >= 0 && p->flag_dens <= 2, AVISM_ERR_ARG, "FLAG_DENS must be 0, 1 or 2");
    AV_CHECK(p->flag_div >= -1 && p->flag_div <= 2, AVISM_ERR_ARG, "FLAG_DIV must be 0, 1 or 2 (or -1)");
}

}  // namespace

extern "C" {

int avism_gpu_create(avism_gpu_ctx **out, int device) {
    if (!out) return AVISM_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
        cudaGetLastError();
        return AVISM_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return AVISM_ERR_NO_DEVICE;          // this library carries sm_100a code only
    }
    avism_gpu_ctx *ctx = new (std::nothrow) avism_gpu_ctx();
    if (!ctx) return AVISM_ERR_OOM;
    ctx->c.device = device;
    ctx->c.num_sms = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->c.copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->c.ev_pos, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->c.ev_mass, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->c.ev_attr, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return AVISM_ERR_CUDA;
    }
    *out = ctx;
    return AVISM_OK;
}

int avism_gpu_destroy(avism_gpu_ctx *ctx) {
    if (!ctx) return AVISM_OK;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    for (int i = 0; i < B_NUM; i++)
        if (ctx->c.buf[i]) cudaFree(ctx->c.buf[i]);
    if (ctx->c.hpin) cudaFreeHost(ctx->c.hpin);
    cudaStreamSynchronize(ctx->c.copy_stream);
    cudaEventDestroy(ctx->c.ev_pos);
    cudaEventDestroy(ctx->c.ev_mass);
    cudaEventDestroy(ctx->c.ev_attr);
    cudaStreamDestroy(ctx->c.copy_stream);
    cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return AVISM_OK;
}

const char *avism_gpu_last_error(const avism_gpu_ctx *ctx) {
    return ctx ? ctx->c.last_error.c_str() : "null context";
}

int avism_gpu_stage_times(const avism_gpu_ctx *ctx, double *ms, int n) {
    if (!ctx) return AVISM_ERR_ARG;
    const int m = (int)ctx->c.stage_ms.size();
    for (int i = 0; i < n && i < m; i++) ms[i] = ctx->c.stage_ms[i];
    return m;
}

const char *avism_gpu_stage_name(const avism_gpu_ctx *ctx, int i) {
    if (!ctx || i < 0 || i >= (int)ctx->c.stage_names.size()) return "";
    return ctx->c.stage_names[(size_t)i].c_str();
}

int64_t avism_gpu_launches(const avism_gpu_ctx *ctx) { return ctx ? ctx->c.launches : -1; }

int avism_gpu_grid_setup(const avism_params *p, avism_grid *g, float *radx) {
    return grid_setup_host(p, g, radx);
}

int avism_gpu_knn(avism_gpu_ctx *ctx, int64_t n, const float *x, const float *y, const float *z, float box_l,
                  int64_t nq, const float *qx, const float *qy, const float *qz, int32_t k, int64_t *idx,
                  float *dist) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(n >= 1 && nq >= 0 && k >= 1 && k <= 256 && x && y && z && idx && dist, AVISM_ERR_ARG,
                 "knn: bad arguments");
        const size_t nb = sizeof(float) * (size_t)n, qb = sizeof(float) * (size_t)std::max<int64_t>(nq, 1);
        const float *dx = (const float *)to_device(c, B_PX, x, nb);
        const float *dy = (const float *)to_device(c, B_PY, y, nb);
        const float *dz = (const float *)to_device(c, B_PZ, z, nb);
        const float *dqx = (const float *)to_device(c, B_PVX, qx, qb);
        const float *dqy = (const float *)to_device(c, B_PVY, qy, qb);
        const float *dqz = (const float *)to_device(c, B_PVZ, qz, qb);
        float box = box_l;
        int periodic = box_l > 0.0f;
        if (!periodic) {
            // bounding cube of the points and the queries, centred at 0
            float lim = 0.0f;
            std::vector<float> hv;
            for (const float *a : {dx, dy, dz, dqx, dqy, dqz}) {
                const int64_t cnt = (a == dqx || a == dqy || a == dqz) ? nq : n;
                if (cnt == 0) continue;
                float *d = c.get_t<float>(B_RED0, 2);
                size_t tmp = 0;
                AV_CUDA(cub::DeviceReduce::Max(nullptr, tmp, a, d, (int)cnt, c.stream));
                void *t = c.get(B_CUB_TMP, tmp);
                AV_CUDA(cub::DeviceReduce::Max(t, tmp, a, d, (int)cnt, c.stream));
                AV_CUDA(cub::DeviceReduce::Min(t, tmp, a, d + 1, (int)cnt, c.stream));
                float h2[2];
                AV_CUDA(cudaMemcpyAsync(h2, d, 8, cudaMemcpyDeviceToHost, c.stream));
                c.sync();
                lim = std::max(lim, std::max(std::fabs(h2[0]), std::fabs(h2[1])));
            }
            box = 2.0f * lim * 1.0001f + 1e-6f;
        }
        BinnedParticles bp = bin_particles(c, n, dx, dy, dz, box, periodic, 4.0f, nullptr, nullptr, nullptr,
                                           nullptr, nullptr, true);
        int64_t *di = (int64_t *)(is_device_ptr(idx) ? (void *)idx : c.get(B_LIST_A, sizeof(int64_t) * (size_t)std::max<int64_t>(nq * k, 1)));
        float *dd = (float *)(is_device_ptr(dist) ? (void *)dist : c.get(B_LIST_B, sizeof(float) * (size_t)std::max<int64_t>(nq * k, 1)));
        knn_batch(c, bp, nq, dqx, dqy, dqz, k, di, dd);
        from_device(c, idx, di, sizeof(int64_t) * (size_t)(nq * k));
        from_device(c, dist, dd, sizeof(float) * (size_t)(nq * k));
        c.sync();
    });
}

int avism_gpu_knn_counters(avism_gpu_ctx *ctx, int enable, int64_t *out, int n) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(n >= 0 && (n == 0 || out), AVISM_ERR_ARG, "knn_counters: bad arguments");
        if (n > 0) {
            unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (c.buf[B_KNN_STATS]) {
                AV_CUDA(cudaMemcpyAsync(h, c.buf[B_KNN_STATS], sizeof h, cudaMemcpyDeviceToHost, c.stream));
                c.sync();
            }
            for (int i = 0; i < n && i < 6; i++) out[i] = (int64_t)h[i];
            for (int i = 6; i < n && i < 9; i++) out[i] = c.path_counts[i - 6];
        }
        c.knn_stats = enable != 0;
    });
}

int avism_gpu_proposal_load(avism_gpu_ctx *ctx, const float *params, int32_t nparam) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(params && nparam == PROPOSAL_NPARAM, AVISM_ERR_ARG,
                 "proposal_load: params must hold AVISM_PROPOSAL_NPARAM floats");
        const float *d = (const float *)to_device(c, B_PR_PARAMS, params, sizeof(float) * PROPOSAL_NPARAM);
        if (d != c.buf[B_PR_PARAMS]) {
            float *keep = c.get_t<float>(B_PR_PARAMS, PROPOSAL_NPARAM);
            AV_CUDA(cudaMemcpyAsync(keep, d, sizeof(float) * PROPOSAL_NPARAM, cudaMemcpyDeviceToDevice, c.stream));
            d = keep;
        }
        proposal_load(c, d);
    });
}

int avism_gpu_proposal_features(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x,
                                const float *y, const float *z, const float *vx, const float *vy,
                                const float *vz, const float *m, int64_t cap_rows, float *feat, int32_t *nb,
                                float *bw) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(n >= 1 && nb && bw, AVISM_ERR_ARG, "proposal_features: bad arguments");
        Level L = make_level(p);
        P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, nullptr);
        int nbv = 0;
        float bwv = 0.f;
        proposal_features(c, p, a, nullptr, &nbv, &bwv);
        *nb = nbv;
        *bw = bwv;
        if (!feat) return;
        const int64_t rows = (int64_t)nbv * nbv * nbv;
        AV_CHECK(cap_rows >= rows, AVISM_ERR_ARG, "proposal_features: feat holds fewer rows than bins");
        float *fd = is_device_ptr(feat) ? feat : c.get_t<float>(B_PR_FEAT, (size_t)rows * 12);
        proposal_features(c, p, a, fd, &nbv, &bwv);
        from_device(c, feat, fd, sizeof(float) * 12 * (size_t)rows);
        c.sync();
    });
}

int avism_gpu_proposal_infer(avism_gpu_ctx *ctx, int64_t nrows, const float *feat, const float *params,
                             float *out) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(nrows >= 0 && feat && params && out, AVISM_ERR_ARG, "proposal_infer: bad arguments");
        const float *fd = (const float *)to_device(c, B_PR_FEAT, feat, sizeof(float) * 12 * (size_t)std::max<int64_t>(nrows, 1));
        const float *pd = (const float *)to_device(c, B_PR_TRAIN, params, sizeof(float) * PROPOSAL_NPARAM);
        float *od = is_device_ptr(out) ? out : c.get_t<float>(B_PR_R0, 2 * (size_t)std::max<int64_t>(nrows, 1));
        proposal_infer(c, nrows, fd, pd, od);
        from_device(c, out, od, sizeof(float) * 2 * (size_t)nrows);
        c.sync();
    });
}

int avism_gpu_proposal_grad(avism_gpu_ctx *ctx, int64_t ns, const float *feat, const float *target,
                            const float *mask, const float *params, float *grad, float *loss) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(ns >= 1 && feat && target && mask && params && grad && loss, AVISM_ERR_ARG,
                 "proposal_grad: bad arguments");
        const float *fd = (const float *)to_device(c, B_PR_FEAT, feat, sizeof(float) * 12 * (size_t)ns);
        const float *td = (const float *)to_device(c, B_PR_W0, target, sizeof(float) * 2 * (size_t)ns);
        const float *md = (const float *)to_device(c, B_KNN_R0, mask, sizeof(float) * 2 * (size_t)ns);
        const float *pd = (const float *)to_device(c, B_PR_PARAMS, params, sizeof(float) * PROPOSAL_NPARAM);
        float *gd = c.get_t<float>(B_PR_GRAD, 3 * (size_t)PROPOSAL_NPARAM);
        float l = 0.f;
        proposal_grad(c, ns, fd, td, md, pd, gd, &l);
        from_device(c, grad, gd, sizeof(float) * PROPOSAL_NPARAM);
        c.sync();
        *loss = l;
    });
}

int avism_gpu_proposal_train(avism_gpu_ctx *ctx, int64_t ns, const float *feat, const float *target,
                             const float *mask, int32_t steps, int32_t batch, float lr, uint32_t seed,
                             float *params, float *loss_curve) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(ns >= 1 && feat && target && mask && params, AVISM_ERR_ARG, "proposal_train: bad arguments");
        const float *fd = (const float *)to_device(c, B_PR_FEAT, feat, sizeof(float) * 12 * (size_t)ns);
        const float *td = (const float *)to_device(c, B_PR_W0, target, sizeof(float) * 2 * (size_t)ns);
        const float *md = (const float *)to_device(c, B_KNN_R0, mask, sizeof(float) * 2 * (size_t)ns);
        float *pd = c.get_t<float>(B_PR_PARAMS, PROPOSAL_NPARAM);
        AV_CUDA(cudaMemcpyAsync(pd, params, sizeof(float) * PROPOSAL_NPARAM, cudaMemcpyDefault, c.stream));
        proposal_train(c, ns, fd, td, md, steps, batch, lr, seed, pd, loss_curve);
        from_device(c, params, pd, sizeof(float) * PROPOSAL_NPARAM);
        c.sync();
    });
}

int avism_gpu_particles_to_grid(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x,
                                const float *y, const float *z, const float *vx, const float *vy,
                                const float *vz, const float *m, const int8_t *smask, float *u_mass,
                                float *u2, float *u3, float *u4, float *hpart, float *part_dens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        Level L = make_level(p);
        P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, smask, hpart || part_dens);
        particles_to_grid(c, p, L, a);
        const size_t gb = sizeof(float) * (size_t)L.g.nx * L.g.nx * L.g.nx;
        from_device(c, u_mass, a.u_mass, gb);
        from_device(c, u2, a.u2, gb);
        from_device(c, u3, a.u3, gb);
        from_device(c, u4, a.u4, gb);
        from_device(c, hpart, a.hpart, sizeof(float) * (size_t)n);
        from_device(c, part_dens, a.part_dens, sizeof(float) * (size_t)n);
        c.sync();
    });
}

int avism_gpu_fields(avism_gpu_ctx *ctx, const avism_params *p, const float *u_mass, const float *u2,
                     const float *u3, const float *u4, float *u1co_ext, float *diverco_ext, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        Level L = make_level(p);
        const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        const size_t gb = sizeof(float) * (size_t)nc;
        const float *dm = (const float *)to_device(c, B_UMASS, u_mass, gb);
        const float *d2 = (const float *)to_device(c, B_U2, u2, gb);
        const float *d3 = (const float *)to_device(c, B_U3, u3, gb);
        const float *d4 = (const float *)to_device(c, B_U4, u4, gb);
        float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
        FieldsOut fo = fields_inner(c, p, L, dm, d2, d3, d4, u1, dv);
        float *e1 = is_device_ptr(u1co_ext) ? u1co_ext : c.get_t<float>(B_U1EXT, ne3);
        float *e2 = is_device_ptr(diverco_ext) ? diverco_ext : c.get_t<float>(B_DVEXT, ne3);
        if (u1co_ext) { ext_copy(c, L, u1, e1); from_device(c, u1co_ext, e1, sizeof(float) * (size_t)ne3); }
        if (diverco_ext) { ext_copy(c, L, dv, e2); from_device(c, diverco_ext, e2, sizeof(float) * (size_t)ne3); }
        c.sync();
        if (meandens) *meandens = fo.meandens;
    });
}

int avism_gpu_voidfind(avism_gpu_ctx *ctx, const avism_params *p, const float *u1co_ext,
                       const float *diverco_ext, const int8_t *smask_ext, const int32_t *marcap_ext,
                       const float *reqp, avism_cubes *cubes, int32_t *nvoid) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(u1co_ext && diverco_ext && cubes && nvoid, AVISM_ERR_ARG, "voidfind: null argument");
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        const float *u1 = (const float *)to_device(c, B_U1EXT, u1co_ext, sizeof(float) * (size_t)ne3);
        const float *dv = (const float *)to_device(c, B_DVEXT, diverco_ext, sizeof(float) * (size_t)ne3);
        const int8_t *sm = (const int8_t *)to_device(c, B_SMASK, smask_ext, (size_t)ne3);
        const int32_t *mp = (const int32_t *)to_device(c, B_MARCAP, marcap_ext, sizeof(int32_t) * (size_t)ne3);
        // parent radii: one per parent id, as many as the largest id in marcap
        int32_t nreqp = 0;
        const float *rq = nullptr;
        if (mp && reqp) {
            int32_t *d = c.get_t<int32_t>(B_RED0, 1);
            size_t tmp = 0;
            AV_CUDA(cub::DeviceReduce::Max(nullptr, tmp, mp, d, (int)ne3, c.stream));
            void *t = c.get(B_CUB_TMP, tmp);
            AV_CUDA(cub::DeviceReduce::Max(t, tmp, mp, d, (int)ne3, c.stream));
            AV_CUDA(cudaMemcpyAsync(&nreqp, d, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            nreqp = std::max(nreqp, 0);
            rq = (const float *)to_device(c, B_REQP, reqp, sizeof(float) * (size_t)std::max(nreqp, 1));
        }
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 1, sm, mp, rq, nreqp, cd);
        HostCubes hc(c, cd, nv);
        cubes_out(c, cd, hc.v, nv, cubes);
        *nvoid = nv;
    });
}

int avism_gpu_flags(avism_gpu_ctx *ctx, const avism_params *p, const float *u1co_ext, const float *diverco_ext,
                    const int8_t *smask_ext, const int32_t *marcap_ext, uint8_t *flags_ext) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(u1co_ext && diverco_ext && flags_ext, AVISM_ERR_ARG, "flags: null argument");
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        const float *u1 = (const float *)to_device(c, B_U1EXT, u1co_ext, sizeof(float) * (size_t)ne3);
        const float *dv = (const float *)to_device(c, B_DVEXT, diverco_ext, sizeof(float) * (size_t)ne3);
        const int8_t *sm = (const int8_t *)to_device(c, B_SMASK, smask_ext, (size_t)ne3);
        const int32_t *mp = (const int32_t *)to_device(c, B_MARCAP, marcap_ext, sizeof(int32_t) * (size_t)ne3);
        uint8_t *fl = is_device_ptr(flags_ext) ? flags_ext : c.get_t<uint8_t>(B_FLAGS, ne3);
        make_flags(c, p, L, u1, dv, 1, sm, mp, fl);
        from_device(c, flags_ext, fl, (size_t)ne3);
        c.sync();
    });
}

int avism_gpu_indexx(avism_gpu_ctx *ctx, int32_t n, const float *arr, int32_t *indx) {
    return guarded(ctx, [&](Ctx &c) {
        AV_CHECK(n >= 0 && (n == 0 || (arr && indx)), AVISM_ERR_ARG, "indexx: bad arguments");
        if (n == 0) return;
        const float *k = (const float *)to_device(c, B_CAND_KEY, arr, sizeof(float) * (size_t)n);
        int32_t *o = is_device_ptr(indx) ? indx : c.get_t<int32_t>(B_CAND_POS, n);
        indexx_device(c, n, k, o);
        from_device(c, indx, o, sizeof(int32_t) * (size_t)n);
        c.sync();
    });
}

int avism_gpu_merge_post(avism_gpu_ctx *ctx, const avism_params *p, int32_t nvoid, const avism_cubes *cubes,
                         const float *u1co_ext, float meandens, avism_voids *out) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid >= 0 && cubes && u1co_ext && out, AVISM_ERR_ARG, "merge_post: null argument");
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
        const float *e1 = (const float *)to_device(c, B_U1EXT, u1co_ext, sizeof(float) * (size_t)ne3);
        float *u1 = c.get_t<float>(B_U1CO, nc);
        ++c.launches, k_inner_from_ext<<<grid_for(nc, 256), 256, 0, c.stream>>>(L.g.nx, L.g.low1, L.g.ne, e1, u1);
        HostCubes hc(c, cubes, nvoid);
        merge_post(c, p, L, nvoid, &hc.v, u1, meandens, out, out->marca);
    });
}

// a26: parent map of the next level, MARCAP(2NX)^3 = MARCA(coarse cell)
// (src/avism.f90:2137-2157), extended to the next level's ghost shell as
// MARCAP2 (src/avism.f90:1670-1674, INT_MAKE_PERIODIC src/num.f90:137-181)
__global__ void k_next_marcap(int nx, int low1, int ne, const int32_t *__restrict__ marca, int nx2, int low1n,
                              int ne2, int32_t *__restrict__ out) {
    const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
    if (i2 >= ne2) return;
    int c[3] = {i2 + low1n, (int)blockIdx.y + low1n, (int)blockIdx.z + low1n};
    for (int a = 0; a < 3; a++) {
        if (c[a] < 1) c[a] += nx2; else if (c[a] > nx2) c[a] -= nx2;
        c[a] = (c[a] - 1) / 2 + 1;                  // INT((IX-1)/2.)+1
    }
    const int64_t e = (int64_t)(c[0] - low1) + (int64_t)ne * ((int64_t)(c[1] - low1) + (int64_t)ne * (c[2] - low1));
    out[(int64_t)i2 + (int64_t)ne2 * (blockIdx.y + (int64_t)ne2 * blockIdx.z)] = marca[e];
}

int avism_gpu_next_level(avism_gpu_ctx *ctx, const avism_params *p, int32_t nvoid, const int32_t *marca_ext,
                         const int32_t *uvoid, const float *req, int32_t *marcap_next_ext, float *reqp_next) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid >= 0 && marca_ext && marcap_next_ext && (nvoid == 0 || (uvoid && req && reqp_next)),
                 AVISM_ERR_ARG, "next_level: null argument");
        Level L = make_level(p);
        avism_params pn = *p;
        pn.nx = 2 * p->nx;
        pn.level = p->level + 1;
        Level Ln = make_level(&pn);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne, ne3n = (int64_t)Ln.g.ne * Ln.g.ne * Ln.g.ne;
        AV_CHECK(Ln.g.ne < 65536 && Ln.g.nplus <= Ln.g.nx, AVISM_ERR_ARG, "next_level: grid too large");
        const int32_t *m = (const int32_t *)to_device(c, B_MARCA, marca_ext, sizeof(int32_t) * (size_t)ne3);
        int32_t *out = is_device_ptr(marcap_next_ext) ? marcap_next_ext
                                                       : c.get_t<int32_t>(B_MARCAP, (size_t)ne3n);
        const dim3 g((unsigned)((Ln.g.ne + 127) / 128), (unsigned)Ln.g.ne, (unsigned)Ln.g.ne);
        ++c.launches, k_next_marcap<<<g, 128, 0, c.stream>>>(L.g.nx, L.g.low1, L.g.ne, m, Ln.g.nx, Ln.g.low1,
                                                              Ln.g.ne, out);
        AV_CUDA(cudaGetLastError());
        from_device(c, marcap_next_ext, out, sizeof(int32_t) * (size_t)ne3n);
        // REQP(IND) = REQ(IND) for the main voids (avism.f90:2140-2144), 0 elsewhere
        if (nvoid > 0) {
            std::vector<int32_t> uv(nvoid);
            std::vector<float> rq(nvoid), rp(nvoid, 0.0f);
            AV_CUDA(cudaMemcpyAsync(uv.data(), uvoid, sizeof(int32_t) * nvoid, cudaMemcpyDefault, c.stream));
            AV_CUDA(cudaMemcpyAsync(rq.data(), req, sizeof(float) * nvoid, cudaMemcpyDefault, c.stream));
            c.sync();
            for (int32_t i = 0; i < nvoid; i++)
                if (uv[i] == -1) rp[i] = rq[i];
            AV_CUDA(cudaMemcpyAsync(reqp_next, rp.data(), sizeof(float) * nvoid, cudaMemcpyDefault, c.stream));
        }
        c.sync();
    });
}

// a level below the first (voids-in-voids): as run_level, with the parent map
// MARCAP2 and parent radii REQP of avism_gpu_next_level
int avism_gpu_run_sublevel(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                           const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                           const int32_t *marcap_ext, const float *reqp, int32_t nreqp, avism_cubes *cubes,
                           int32_t *nvoid, avism_voids *voids, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids && marcap_ext && nreqp >= 0 && (nreqp == 0 || reqp), AVISM_ERR_ARG,
                 "run_sublevel: null argument");
        Level L = make_level(p);
        const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, nullptr, false);
        const int32_t *mp = (const int32_t *)to_device(c, B_MARCAP, marcap_ext, sizeof(int32_t) * (size_t)ne3);
        const float *rq = nreqp > 0 ? (const float *)to_device(c, B_REQP, reqp, sizeof(float) * (size_t)nreqp) : nullptr;
        WidthProposal wp;
        a.wprop = &wp;
        c.mark("h2d");
        particles_to_grid(c, p, L, a);
        float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
        FieldsOut fo = fields_inner(c, p, L, a.u_mass, a.u2, a.u3, a.u4, u1, dv);
        c.mark("divergence");
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, nullptr, mp, rq, nreqp, cd, &wp);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, fo.meandens, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = fo.meandens;
    });
}

// ---- survey mode (FLAG_SURVEY = 1, src/avism.f90:1420-1596) ------------------
// the survey mask on the ext grid: the inner cells' values, 0 on the ghost shell
// (SMASK = 0 before the inner cells are set, src/avism.f90:867-869)
__global__ void k_smask_ext(int nx, int low1, int ne, const int8_t *__restrict__ inner, int8_t *__restrict__ ext) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)ne * ne * ne) return;
    const int i = (int)(e % ne) + low1, j = (int)((e / ne) % ne) + low1, k = (int)(e / ((int64_t)ne * ne)) + low1;
    const bool in = i >= 1 && i <= nx && j >= 1 && j <= nx && k >= 1 && k <= nx;
    ext[e] = in ? inner[(int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)nx * (k - 1))] : (int8_t)0;
}

namespace {

// tracers and randoms to the grid, the D/(alpha R) contrast and the divergence,
// into the inner U1CO / DIVER buffers; returns MEANDENS
float survey_fields_dev(Ctx &c, const avism_params *p, const Level &L, int64_t n, const float *x, const float *y,
                        const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                        int64_t nrand, const float *rx, const float *ry, const float *rz, const float *rw,
                        const int8_t *smask, float **u1_out, float **dv_out, const int8_t **smask_out) {
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    AV_CHECK(smask && nrand >= 1 && rx && ry && rz && rw, AVISM_ERR_ARG, "survey: mask and randoms required");
    const int8_t *sm = (const int8_t *)to_device(c, B_SMASK_IN, smask, (size_t)nc);
    // tracers (with the mask)
    P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, sm, false);
    particles_to_grid(c, p, L, a);
    float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
    rho_inner(c, L, a.u_mass, u1);
    if (!p->no_velocities) divergence_inner(c, p, L, u1, a.u2, a.u3, a.u4, dv);
    c.mark("survey_tracers");
    // randoms: no velocities; H_DISTANCE and FILL_H_ZEROS with
    // KNEIGHBOURS2 = MIN(8*KNEIGHBOURS, 256) (src/avism.f90:1516), or TSC
    avism_params pr = *p;
    pr.no_velocities = 1;
    pr.kneighbours = std::min(8 * p->kneighbours, 256);
    pr.learned = p->learned == 1 ? 2 : p->learned;     // the network predicts K = KNEIGHBOURS radii
    P2G ar = p2g_args(c, &pr, L, nrand, rx, ry, rz, nullptr, nullptr, nullptr, rw, sm, false);
    ar.u_mass = c.get_t<float>(B_U1RAND, nc);
    particles_to_grid(c, &pr, L, ar);
    c.mark("survey_randoms");
    const float meandens = survey_contrast(c, L, sm, ar.u_mass, u1);
    if (p->no_velocities) divergence_inner(c, p, L, u1, nullptr, nullptr, nullptr, dv);
    c.mark("survey_contrast");
    *u1_out = u1;
    *dv_out = dv;
    *smask_out = sm;
    return meandens;
}

}  // namespace

int avism_gpu_survey_fields(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                            const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                            int64_t nrand, const float *rx, const float *ry, const float *rz, const float *rw,
                            const int8_t *smask, float *u1co_ext, float *diverco_ext, float *meandens,
                            float *u1rand) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        Level L = make_level(p);
        const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        float *u1, *dv;
        const int8_t *sm;
        const float md = survey_fields_dev(c, p, L, n, x, y, z, vx, vy, vz, m, nrand, rx, ry, rz, rw, smask, &u1, &dv,
                                           &sm);
        float *e1 = is_device_ptr(u1co_ext) ? u1co_ext : c.get_t<float>(B_U1EXT, ne3);
        float *e2 = is_device_ptr(diverco_ext) ? diverco_ext : c.get_t<float>(B_DVEXT, ne3);
        if (u1co_ext) { ext_copy(c, L, u1, e1); from_device(c, u1co_ext, e1, sizeof(float) * (size_t)ne3); }
        if (diverco_ext) { ext_copy(c, L, dv, e2); from_device(c, diverco_ext, e2, sizeof(float) * (size_t)ne3); }
        from_device(c, u1rand, c.buf[B_U1RAND], sizeof(float) * (size_t)nc);
        c.sync();
        if (meandens) *meandens = md;
    });
}

int avism_gpu_run_level_survey(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                               const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                               int64_t nrand, const float *rx, const float *ry, const float *rz, const float *rw,
                               const int8_t *smask, avism_cubes *cubes, int32_t *nvoid, avism_voids *voids,
                               float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids, AVISM_ERR_ARG, "run_level_survey: null argument");
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        float *u1, *dv;
        const int8_t *sm;
        const float md = survey_fields_dev(c, p, L, n, x, y, z, vx, vy, vz, m, nrand, rx, ry, rz, rw, smask, &u1, &dv,
                                           &sm);
        int8_t *sme = c.get_t<int8_t>(B_SMASK, (size_t)ne3);
        ++c.launches, k_smask_ext<<<grid_for(ne3, 256), 256, 0, c.stream>>>(L.g.nx, L.g.low1, L.g.ne, sm, sme);
        AV_CUDA(cudaGetLastError());
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, sme, nullptr, nullptr, 0, cd, nullptr);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, md, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = md;
    });
}

// ---- grid input (FLAG_DATA = 2, READ_BINARY_GRID): src/avism.f90:1316-1362 --------
namespace {
float grid_fields_dev(Ctx &c, const avism_params *p, const Level &L, int32_t nhy, const float *u1g,
                      const float *u2g, const float *u3g, const float *u4g, float **u1_out, float **dv_out) {
    AV_CHECK(u1g && u2g && u3g && u4g && nhy >= 4, AVISM_ERR_ARG, "grid input: four grids of nhy >= 4 required");
    AV_CHECK(p->level <= 0, AVISM_ERR_UNSUPPORTED, "LEVEL > 0 FOR BIN_GRID NOT IMPLEMENTED YET");
    AV_CHECK((int64_t)p->nx << (-p->level) == (int64_t)nhy, AVISM_ERR_ARG,
             "grid input: params.nx must be nhy * 2^level (level <= 0)");
    const int64_t n0 = (int64_t)nhy * nhy * nhy;
    const float *g[4];
    const float *src[4] = {u1g, u2g, u3g, u4g};
    float *buf = nullptr;
    for (int q = 0; q < 4; q++) {
        if (is_device_ptr(src[q])) { g[q] = src[q]; continue; }
        if (!buf) buf = c.get_t<float>(B_GRID_IN, 4 * (size_t)n0);
        AV_CUDA(cudaMemcpyAsync(buf + q * n0, src[q], sizeof(float) * (size_t)n0, cudaMemcpyHostToDevice, c.stream));
        g[q] = buf + q * n0;
    }
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
    const float md = grid_fields_inner(c, p, L, nhy, g[0], g[1], g[2], g[3], u1, dv);
    *u1_out = u1;
    *dv_out = dv;
    return md;
}
}  // namespace

int avism_gpu_grid_fields(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g, const float *u2g,
                          const float *u3g, const float *u4g, float *u1co_ext, float *diverco_ext, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        float *u1, *dv;
        const float md = grid_fields_dev(c, p, L, nhy, u1g, u2g, u3g, u4g, &u1, &dv);
        float *e1 = is_device_ptr(u1co_ext) ? u1co_ext : c.get_t<float>(B_U1EXT, ne3);
        float *e2 = is_device_ptr(diverco_ext) ? diverco_ext : c.get_t<float>(B_DVEXT, ne3);
        if (u1co_ext) { ext_copy(c, L, u1, e1); from_device(c, u1co_ext, e1, sizeof(float) * (size_t)ne3); }
        if (diverco_ext) { ext_copy(c, L, dv, e2); from_device(c, diverco_ext, e2, sizeof(float) * (size_t)ne3); }
        c.sync();
        if (meandens) *meandens = md;
    });
}

int avism_gpu_run_level_grid(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                             const float *u2g, const float *u3g, const float *u4g, avism_cubes *cubes,
                             int32_t *nvoid, avism_voids *voids, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids, AVISM_ERR_ARG, "run_level_grid: null argument");
        Level L = make_level(p);
        float *u1, *dv;
        const float md = grid_fields_dev(c, p, L, nhy, u1g, u2g, u3g, u4g, &u1, &dv);
        c.mark("divergence");
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, nullptr, nullptr, nullptr, 0, cd, nullptr);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, md, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = md;
    });
}

// ---- MASCLET input (FLAG_DATA = 0) at levels <= 0 ------------------------------
namespace {
// the level-1 patches: geometry to host vectors, cells to the device
void host_bytes(void *dst, const void *src, size_t bytes) {
    if (bytes) AV_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
}
void host_i32(std::vector<int32_t> &dst, const int32_t *src, size_t n) {
    dst.resize(n);
    host_bytes(dst.data(), src, sizeof(int32_t) * n);
}
void host_f32(std::vector<float> &dst, const float *src, size_t n) {
    dst.resize(n);
    host_bytes(dst.data(), src, sizeof(float) * n);
}
void host_i64(std::vector<int64_t> &dst, const int64_t *src, size_t n) {
    dst.resize(n);
    host_bytes(dst.data(), src, sizeof(int64_t) * n);
}
AmrPatches amr_patches(Ctx &c, const avism_patches *a) {
    AV_CHECK(a && a->npatch >= 0 && a->offset, AVISM_ERR_ARG, "MASCLET level 1: the patches are required");
    AmrPatches r;
    const size_t np = (size_t)a->npatch;
    r.npatch = a->npatch;
    AV_CHECK(np == 0 || (a->nx && a->ny && a->nz && a->ix && a->iy && a->iz && a->rx && a->ry && a->rz),
             AVISM_ERR_ARG, "MASCLET level 1: null patch geometry");
    host_i32(r.nx, a->nx, np); host_i32(r.ny, a->ny, np); host_i32(r.nz, a->nz, np);
    host_i32(r.ix, a->ix, np); host_i32(r.iy, a->iy, np); host_i32(r.iz, a->iz, np);
    host_f32(r.rx, a->rx, np); host_f32(r.ry, a->ry, np); host_f32(r.rz, a->rz, np);
    host_i64(r.offset, a->offset, np + 1);
    AV_CHECK(r.offset[0] >= 0, AVISM_ERR_ARG, "MASCLET level 1: negative patch offset");
    for (size_t q = 0; q < np; q++)
        AV_CHECK(r.nx[q] >= 1 && r.ny[q] >= 1 && r.nz[q] >= 1 && r.nx[q] <= (1 << 20) && r.ny[q] <= (1 << 20) &&
                     r.nz[q] <= (1 << 20) && r.offset[q + 1] - r.offset[q] == (int64_t)r.nx[q] * r.ny[q] * r.nz[q],
                 AVISM_ERR_ARG, "MASCLET level 1: patch sizes and offsets disagree");
    if (r.offset[np] == 0) return r;                    // no patches: no cells to read
    const size_t cells = sizeof(float) * (size_t)r.offset[np];
    AV_CHECK(a->u11g && a->u12g && a->u13g && a->u14g, AVISM_ERR_ARG, "MASCLET level 1: null patch cells");
    r.u11g = (const float *)to_device(c, B_AMR1, a->u11g, cells);
    r.u12g = (const float *)to_device(c, B_AMR2, a->u12g, cells);
    r.u13g = (const float *)to_device(c, B_AMR3, a->u13g, cells);
    r.u14g = (const float *)to_device(c, B_AMR4, a->u14g, cells);
    return r;
}

float masclet_fields_dev(Ctx &c, const avism_params *p, const Level &L, int32_t nhy, const float *u1g,
                         const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr, int64_t n,
                         const float *x, const float *y, const float *z, const float *vx, const float *vy,
                         const float *vz, const float *m, float **u1_out, float **dv_out) {
    AV_CHECK(p->level <= 1, AVISM_ERR_UNSUPPORTED,
             "MASCLET input: levels above 1 are not implemented (the reference's VMESH indexes its base-size "
             "refinement flags beyond them there)");
    AV_CHECK(nhy >= 4 && (p->level == 1 ? p->nx == 2 * nhy : (int64_t)p->nx << (-p->level) == (int64_t)nhy),
             AVISM_ERR_ARG, "MASCLET input: params.nx must be nhy * 2^level");
    const bool need_dm = p->flag_dens <= 1 || p->flag_div == 0 || p->flag_div == 1;
    const bool need_gas_v = p->level == 1 || p->flag_div == 0 || p->flag_div == 2;
    AV_CHECK(u1g && (!need_gas_v || (u2g && u3g && u4g)), AVISM_ERR_ARG, "MASCLET input: null gas grid");
    AmrPatches ap;
    if (p->level == 1) ap = amr_patches(c, amr);
    const int64_t n0 = (int64_t)nhy * nhy * nhy;
    const float *g[4] = {nullptr, nullptr, nullptr, nullptr};
    const float *src[4] = {u1g, u2g, u3g, u4g};
    float *buf = nullptr;
    for (int q = 0; q < (need_gas_v ? 4 : 1); q++) {
        if (is_device_ptr(src[q])) { g[q] = src[q]; continue; }
        if (!buf) buf = c.get_t<float>(B_GRID_IN, 4 * (size_t)n0);
        AV_CUDA(cudaMemcpyAsync(buf + q * n0, src[q], sizeof(float) * (size_t)n0, cudaMemcpyHostToDevice, c.stream));
        g[q] = buf + q * n0;
    }
    const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
    const float *um = nullptr, *d2 = nullptr, *d3 = nullptr, *d4 = nullptr;
    if (need_dm) {
        // the DM particles as in the particle path (src/avism.f90:984-1061)
        P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, nullptr, false);
        particles_to_grid(c, p, L, a);
        um = a.u_mass; d2 = a.u2; d3 = a.u3; d4 = a.u4;
    }
    float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
    const float md = masclet_fields_inner(c, p, L, nhy, g, p->level == 1 ? &ap : nullptr, um, d2, d3, d4, u1, dv);
    *u1_out = u1;
    *dv_out = dv;
    return md;
}
}  // namespace

int avism_gpu_masclet_fields(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                             const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                             int64_t n, const float *x, const float *y, const float *z, const float *vx,
                             const float *vy, const float *vz, const float *m, float *u1co_ext,
                             float *diverco_ext, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        float *u1, *dv;
        const float md = masclet_fields_dev(c, p, L, nhy, u1g, u2g, u3g, u4g, amr, n, x, y, z, vx, vy, vz, m, &u1, &dv);
        float *e1 = is_device_ptr(u1co_ext) ? u1co_ext : c.get_t<float>(B_U1EXT, ne3);
        float *e2 = is_device_ptr(diverco_ext) ? diverco_ext : c.get_t<float>(B_DVEXT, ne3);
        if (u1co_ext) { ext_copy(c, L, u1, e1); from_device(c, u1co_ext, e1, sizeof(float) * (size_t)ne3); }
        if (diverco_ext) { ext_copy(c, L, dv, e2); from_device(c, diverco_ext, e2, sizeof(float) * (size_t)ne3); }
        c.sync();
        if (meandens) *meandens = md;
    });
}

int avism_gpu_run_level_masclet(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                                const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                                int64_t n, const float *x, const float *y, const float *z, const float *vx,
                                const float *vy, const float *vz, const float *m, avism_cubes *cubes,
                                int32_t *nvoid, avism_voids *voids, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids, AVISM_ERR_ARG, "run_level_masclet: null argument");
        Level L = make_level(p);
        float *u1, *dv;
        const float md = masclet_fields_dev(c, p, L, nhy, u1g, u2g, u3g, u4g, amr, n, x, y, z, vx, vy, vz, m, &u1, &dv);
        c.mark("divergence");
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, nullptr, nullptr, nullptr, 0, cd, nullptr);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, md, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = md;
    });
}

int avism_gpu_run_sublevel_masclet(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                                   const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                                   int64_t n, const float *x, const float *y, const float *z, const float *vx,
                                   const float *vy, const float *vz, const float *m, const int32_t *marcap_ext,
                                   const float *reqp, int32_t nreqp, avism_cubes *cubes, int32_t *nvoid,
                                   avism_voids *voids, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids && marcap_ext && nreqp >= 0 && (nreqp == 0 || reqp), AVISM_ERR_ARG,
                 "run_sublevel_masclet: null argument");
        Level L = make_level(p);
        const int64_t ne3 = (int64_t)L.g.ne * L.g.ne * L.g.ne;
        float *u1, *dv;
        const float md = masclet_fields_dev(c, p, L, nhy, u1g, u2g, u3g, u4g, amr, n, x, y, z, vx, vy, vz, m, &u1, &dv);
        const int32_t *mp = (const int32_t *)to_device(c, B_MARCAP, marcap_ext, sizeof(int32_t) * (size_t)ne3);
        const float *rq = nreqp > 0 ? (const float *)to_device(c, B_REQP, reqp, sizeof(float) * (size_t)nreqp) : nullptr;
        c.mark("divergence");
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, nullptr, mp, rq, nreqp, cd, nullptr);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, md, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = md;
    });
}

int avism_gpu_run_level(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                        const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                        avism_cubes *cubes, int32_t *nvoid, avism_voids *voids, float *meandens) {
    return guarded(ctx, [&](Ctx &c) {
        check_params(p);
        AV_CHECK(nvoid && voids, AVISM_ERR_ARG, "run_level: null argument");
        Level L = make_level(p);
        const int64_t nc = (int64_t)L.g.nx * L.g.nx * L.g.nx;
        P2G a = p2g_args(c, p, L, n, x, y, z, vx, vy, vz, m, nullptr, false);
        WidthProposal wp;
        a.wprop = &wp;
        c.mark("h2d");
        particles_to_grid(c, p, L, a);
        float *u1 = c.get_t<float>(B_U1CO, nc), *dv = c.get_t<float>(B_DIVER, nc);
        FieldsOut fo = fields_inner(c, p, L, a.u_mass, a.u2, a.u3, a.u4, u1, dv);
        c.mark("divergence");
        CubesDev cd{};
        const int32_t nv = voidfind_device(c, p, L, u1, dv, 0, nullptr, nullptr, nullptr, 0, cd, &wp);
        HostCubes hc(c, cd, nv);
        if (cubes) cubes_out(c, cd, hc.v, nv, cubes);
        c.mark("cubes_d2h");
        merge_post(c, p, L, nv, &hc.v, u1, fo.meandens, voids, voids->marca);
        c.mark("catalogue_d2h");
        *nvoid = nv;
        if (meandens) *meandens = fo.meandens;
    });
}

}  // extern "C"
