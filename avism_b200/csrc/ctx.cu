// ctx.cu -- context, pointer handling and the level geometry (host side).
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace avism {

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

const void *to_device(Ctx &c, BufId id, const void *src, size_t bytes) {
    if (!src) return nullptr;
    if (is_device_ptr(src)) return src;
    void *d = c.get(id, bytes);
    AV_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, c.stream));
    return d;
}

const void *to_device_on(Ctx &c, cudaStream_t st, BufId id, const void *src, size_t bytes) {
    if (!src) return nullptr;
    if (is_device_ptr(src)) return src;
    void *d = c.get(id, bytes);
    AV_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st));
    return d;
}

void from_device(Ctx &c, void *dst, const void *src_dev, size_t bytes) {
    if (!dst || bytes == 0) return;
    if (dst == src_dev) return;
    AV_CUDA(cudaMemcpyAsync(dst, src_dev, bytes, cudaMemcpyDefault, c.stream));
}

// Level geometry: MALLA (src/grid.f90:3-76) and the PBC extension of
// src/avism.f90:780-865, with the cosmology of src/avism.f90:476-488, 607-616.
// Host code is built with -ffp-contract=off so each REAL*4 operation rounds.
int grid_setup_host(const avism_params *p, avism_grid *g, float *radx) {
    if (!p || !g || p->nx < 4 || !(p->lado0 > 0.0f)) return AVISM_ERR_ARG;
    const int nx = p->nx;
    const float lado0 = p->lado0;
    std::memset(g, 0, sizeof(*g));
    int nplus = 0, low1 = 1, low2 = nx;
    float lado0plus = lado0;
    if (p->periodic) {
        const float dx0 = lado0 / (float)nx;
        const float sizing = std::fmin(50.0f, lado0 / 2.0f);
        const int t = (int)(sizing / dx0);
        nplus = std::max(nx / 8, t);
        low1 = -nplus + 1;
        low2 = nx + nplus;
        lado0plus = lado0 + (2.0f * (float)nplus) * dx0;
    }
    const float lado = lado0 - (lado0 / (float)nx);
    const float a = -lado / 2.0f, b = lado / 2.0f;
    const float c = (b - a) / (float)(nx - 1);
    const float r1 = a;
    const float dx = (r1 + 1.0f * c) - r1;
    const float rnx = r1 + (float)(nx - 1) * c;
    const int rad_lo = std::min(low1, 0), rad_hi = std::max(low2, nx + 1);
    if (radx) {
        for (int i = rad_lo; i <= rad_hi; i++) {
            float v;
            if (i >= 1 && i <= nx) v = r1 + (float)(i - 1) * c;
            else if (!p->periodic) v = (i == 0) ? r1 - c : rnx + c;
            else if (i < 1) v = r1 - (float)(1 - i) * dx;
            else v = rnx + (float)(i - nx) * dx;
            radx[i - rad_lo] = v;
        }
    }
    const float ache0 = (float)((double)p->ache * 3.66e-3);
    const float rodo = (float)((double)p->omega0 * 3.0 * (double)(ache0 * ache0));
    const float re0 = 1.0f / 10.98f;
    const float zeta = p->zeta < 0.0f ? 0.0f : p->zeta;
    const float t1 = 1.0f + zeta;
    const float rote = rodo * ((t1 * t1) * t1);
    const float rete = re0 / (1.0f + zeta);
    const float rr = re0 / rete;
    float hte = p->omega0 * (((rr * rr) * rr) - 1.0f) + 1.0f;
    hte = p->ache * std::sqrt(hte);
    g->nx = nx; g->nplus = nplus; g->low1 = low1; g->low2 = low2; g->ne = low2 - low1 + 1;
    g->rad_lo = rad_lo; g->rad_hi = rad_hi;
    g->dx = dx; g->rx1 = r1; g->lado = lado; g->lado0plus = lado0plus;
    g->rete = rete; g->rote = rote; g->hte = hte;
    return AVISM_OK;
}

Level make_level(const avism_params *p) {
    Level L;
    int st = grid_setup_host(p, &L.g, nullptr);
    AV_CHECK(st == AVISM_OK, st, "invalid grid parameters (nx >= 4 and lado0 > 0 required)");
    L.rad.resize((size_t)(L.g.rad_hi - L.g.rad_lo + 1));
    grid_setup_host(p, &L.g, L.rad.data());
    return L;
}

}  // namespace avism
