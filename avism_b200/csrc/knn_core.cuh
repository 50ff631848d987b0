// knn_core.cuh -- device-side exact kNN on binned particles.
//
// One thread per query.  The current best K keys live in a shared-memory
// column (stride = blockDim.x, conflict-free), sorted ascending.  A key is
// (float bits of the squared distance) << 32 | particle index, so ties in
// distance are broken by the smaller particle index.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace avism {

#define KNN_THREADS(KCAP) ((KCAP) <= 32 ? 256 : (KCAP) <= 64 ? 128 : (KCAP) <= 128 ? 64 : 32)

struct KnnGrid {
    const float4 *sp;
    const int64_t *start;
    int nb;
    float origin, bw, inv_bw, box, margin;
    int periodic;
};

inline KnnGrid make_knn_grid(const BinnedParticles &bp) {
    KnnGrid G;
    G.sp = bp.sp;
    G.start = bp.start;
    G.nb = bp.nb;
    G.origin = bp.origin;
    G.bw = bp.bw;
    G.inv_bw = bp.inv_bw;
    G.box = bp.box;
    G.periodic = bp.periodic;
    G.margin = 2e-3f * bp.bw + 1e-6f * bp.box;
    return G;
}

__host__ __device__ __forceinline__ int bin_coord(float x, float origin, float inv_bw, int nb) {
    int b = (int)floorf((x - origin) * inv_bw);
    return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

// squared distance exactly as distance() in src/kdtree.f90:1441-1465:
// dx = p - q, periodic dx = min(|dx|, L-|dx|), d2 = ((0 + dx^2) + dy^2) + dz^2
__device__ __forceinline__ float dist2_ref(float px, float py, float pz, float qx, float qy, float qz,
                                           float L, int periodic) {
    float dx = __fsub_rn(px, qx), dy = __fsub_rn(py, qy), dz = __fsub_rn(pz, qz);
    if (periodic) {
        float a = fabsf(dx);
        dx = fminf(a, __fsub_rn(L, a));
        a = fabsf(dy);
        dy = fminf(a, __fsub_rn(L, a));
        a = fabsf(dz);
        dz = fminf(a, __fsub_rn(L, a));
    }
    float d = __fmul_rn(dx, dx);
    d = __fadd_rn(d, __fmul_rn(dy, dy));
    d = __fadd_rn(d, __fmul_rn(dz, dz));
    return d;
}

__device__ __forceinline__ unsigned long long knn_key(float d2, uint32_t idx) {
    return ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned long long)idx;
}
__device__ __forceinline__ float key_d2(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t key_idx(unsigned long long k) { return (uint32_t)(k & 0xffffffffu); }

// allowed bin offsets along one axis for shell radius s
__device__ __forceinline__ void axis_window(const KnnGrid &G, int b, int s, int &lo, int &hi) {
    if (G.periodic) {
        lo = -min(s, (G.nb - 1) / 2);
        hi = min(s, G.nb / 2);
    } else {
        lo = max(-s, -b);
        hi = min(s, G.nb - 1 - b);
    }
}

__device__ __forceinline__ int wrap_bin(int b, int nb) {
    b %= nb;
    return b < 0 ? b + nb : b;
}

template <int KCAP>
__device__ __forceinline__ void topk_insert(unsigned long long *col, int S, int K, int &cnt,
                                            unsigned long long key) {
    int i;
    if (cnt < K) {
        i = cnt++;
    } else {
        if (key >= col[(size_t)(K - 1) * S]) return;
        i = K - 1;
    }
    while (i > 0) {
        const unsigned long long prev = col[(size_t)(i - 1) * S];
        if (prev <= key) break;
        col[(size_t)i * S] = prev;
        i--;
    }
    col[(size_t)i * S] = key;
}

__device__ __forceinline__ void scan_bin(const KnnGrid &G, int bin, float qx, float qy, float qz,
                                         unsigned long long *col, int S, int K, int &cnt) {
    const int64_t a = G.start[bin], e = G.start[bin + 1];
    for (int64_t p = a; p < e; p++) {
        const float4 v = G.sp[p];
        const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, G.periodic);
        const unsigned long long key = knn_key(d2, (uint32_t)__float_as_int(v.w));
        if (cnt < K || key < col[(size_t)(K - 1) * S]) topk_insert<0>(col, S, K, cnt, key);
    }
}

// Distance from q to the boundary of the visited block of bins after shell s.
// Returns +inf when no particle can lie outside (every bin visited on the
// relevant sides); *all_done set when every bin has been visited.
__device__ __forceinline__ float guaranteed_radius(const KnnGrid &G, const int b[3], const float q[3],
                                                   int s, bool *all_done) {
    float r = FLT_MAX;
    bool done = true;
    for (int a = 0; a < 3; a++) {
        if (G.periodic) {
            if (2 * s + 1 >= G.nb) continue;
            const float lo = G.origin + (float)(b[a] - s) * G.bw;
            const float hi = G.origin + (float)(b[a] + s + 1) * G.bw;
            r = fminf(r, fminf(q[a] - lo, hi - q[a]));
            done = false;
        } else {
            if (b[a] - s > 0) {
                r = fminf(r, q[a] - (G.origin + (float)(b[a] - s) * G.bw));
                done = false;
            }
            if (b[a] + s < G.nb - 1) {
                r = fminf(r, (G.origin + (float)(b[a] + s + 1) * G.bw) - q[a]);
                done = false;
            }
        }
    }
    *all_done = done;
    return r - G.margin;
}

// Exact K nearest of q; returns the number found (K unless fewer particles).
template <int KCAP>
__device__ int knn_query(const KnnGrid &G, float qx, float qy, float qz, int K,
                         unsigned long long *col, int S) {
    const int b[3] = {bin_coord(qx, G.origin, G.inv_bw, G.nb), bin_coord(qy, G.origin, G.inv_bw, G.nb),
                      bin_coord(qz, G.origin, G.inv_bw, G.nb)};
    const float q[3] = {qx, qy, qz};
    int cnt = 0;
    for (int s = 0;; s++) {
        int lz, hz, ly, hy, lx, hx;
        axis_window(G, b[2], s, lz, hz);
        axis_window(G, b[1], s, ly, hy);
        axis_window(G, b[0], s, lx, hx);
        for (int dz = lz; dz <= hz; dz++) {
            const int bz = G.periodic ? wrap_bin(b[2] + dz, G.nb) : b[2] + dz;
            for (int dy = ly; dy <= hy; dy++) {
                const int by = G.periodic ? wrap_bin(b[1] + dy, G.nb) : b[1] + dy;
                const bool face = (dz == s || dz == -s || dy == s || dy == -s);
                const int row = G.nb * (by + G.nb * bz);
                if (face) {
                    for (int dx = lx; dx <= hx; dx++) {
                        const int bx = G.periodic ? wrap_bin(b[0] + dx, G.nb) : b[0] + dx;
                        scan_bin(G, row + bx, qx, qy, qz, col, S, K, cnt);
                    }
                } else {
                    if (lx == -s) {
                        const int bx = G.periodic ? wrap_bin(b[0] - s, G.nb) : b[0] - s;
                        scan_bin(G, row + bx, qx, qy, qz, col, S, K, cnt);
                    }
                    if (hx == s && s > 0) {
                        const int bx = G.periodic ? wrap_bin(b[0] + s, G.nb) : b[0] + s;
                        scan_bin(G, row + bx, qx, qy, qz, col, S, K, cnt);
                    }
                }
            }
        }
        bool all_done;
        const float r = guaranteed_radius(G, b, q, s, &all_done);
        if (all_done) break;
        if (cnt == K && r > 0.0f) {
            const float kth = key_d2(col[(size_t)(K - 1) * S]);
            if (kth < __fmul_rn(r, r)) break;
        }
    }
    return cnt;
}

}  // namespace avism
