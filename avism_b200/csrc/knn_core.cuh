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
    const float *r0;          // per-bin starting radius of the radius-guided search, or null
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
    G.r0 = nullptr;
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

// candidates [a, e) of the binned array; tau = current K-th key (or ~0)
__device__ __forceinline__ void scan_range(const KnnGrid &G, int64_t a, int64_t e, float qx, float qy, float qz,
                                           unsigned long long *col, int S, int K, int &cnt,
                                           unsigned long long &tau) {
    int64_t p = a;
    for (; p + 1 < e; p += 2) {                    // two independent loads in flight
        const float4 v0 = G.sp[p], v1 = G.sp[p + 1];
        const float d0 = dist2_ref(v0.x, v0.y, v0.z, qx, qy, qz, G.box, G.periodic);
        const float d1 = dist2_ref(v1.x, v1.y, v1.z, qx, qy, qz, G.box, G.periodic);
        const unsigned long long k0 = knn_key(d0, (uint32_t)__float_as_int(v0.w));
        const unsigned long long k1 = knn_key(d1, (uint32_t)__float_as_int(v1.w));
        if (k0 < tau) {
            topk_insert<0>(col, S, K, cnt, k0);
            if (cnt == K) tau = col[(size_t)(K - 1) * S];
        }
        if (k1 < tau) {
            topk_insert<0>(col, S, K, cnt, k1);
            if (cnt == K) tau = col[(size_t)(K - 1) * S];
        }
    }
    if (p < e) {
        const float4 v = G.sp[p];
        const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, G.periodic);
        const unsigned long long key = knn_key(d2, (uint32_t)__float_as_int(v.w));
        if (key < tau) {
            topk_insert<0>(col, S, K, cnt, key);
            if (cnt == K) tau = col[(size_t)(K - 1) * S];
        }
    }
}

__device__ __forceinline__ void scan_bin(const KnnGrid &G, int bin, float qx, float qy, float qz,
                                         unsigned long long *col, int S, int K, int &cnt) {
    unsigned long long tau = cnt == K ? col[(size_t)(K - 1) * S] : ~0ULL;
    scan_range(G, G.start[bin], G.start[bin + 1], qx, qy, qz, col, S, K, cnt, tau);
}

// bins bx0..bx1 (unwrapped, at most nb of them) of one (by, bz) row
__device__ __forceinline__ void scan_row(const KnnGrid &G, int row, int bx0, int bx1, float qx, float qy, float qz,
                                         unsigned long long *col, int S, int K, int &cnt, unsigned long long &tau) {
    if (!G.periodic) {
        scan_range(G, G.start[row + bx0], G.start[row + bx1 + 1], qx, qy, qz, col, S, K, cnt, tau);
        return;
    }
    const int w0 = wrap_bin(bx0, G.nb), n = bx1 - bx0 + 1;
    if (w0 + n <= G.nb) {
        scan_range(G, G.start[row + w0], G.start[row + w0 + n], qx, qy, qz, col, S, K, cnt, tau);
    } else {                                       // the run wraps around x
        scan_range(G, G.start[row + w0], G.start[row + G.nb], qx, qy, qz, col, S, K, cnt, tau);
        scan_range(G, G.start[row], G.start[row + (w0 + n - G.nb)], qx, qy, qz, col, S, K, cnt, tau);
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
    unsigned long long tau = ~0ULL;
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
                    scan_row(G, row, b[0] + lx, b[0] + hx, qx, qy, qz, col, S, K, cnt, tau);
                } else {
                    if (lx == -s) scan_row(G, row, b[0] - s, b[0] - s, qx, qy, qz, col, S, K, cnt, tau);
                    if (hx == s && s > 0) scan_row(G, row, b[0] + s, b[0] + s, qx, qy, qz, col, S, K, cnt, tau);
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


// min distance from q to the bin with unwrapped coordinates (bx, by, bz)
__device__ __forceinline__ float bin_mindist2(const KnnGrid &G, const float q[3], int bx, int by, int bz) {
    const int b[3] = {bx, by, bz};
    float d2 = 0.0f;
    for (int a = 0; a < 3; a++) {
        const float lo = G.origin + (float)b[a] * G.bw, hi = lo + G.bw;
        const float g = fmaxf(fmaxf(lo - q[a], q[a] - hi), 0.0f);
        d2 += g * g;
    }
    return d2;
}

// Exact K nearest of q, starting from the radius estimate r0: scan every bin
// that meets the ball of radius r (bins met by the previous ball skipped),
// stop once the K-th distance is <= r (every particle not scanned is farther
// than r), else grow r by 1.5.  Same results as knn_query.
template <int KCAP>
__device__ int knn_query_radius(const KnnGrid &G, float qx, float qy, float qz, int K,
                                unsigned long long *col, int S, float r0) {
    const float q[3] = {qx, qy, qz};
    const int bq[3] = {bin_coord(qx, G.origin, G.inv_bw, G.nb), bin_coord(qy, G.origin, G.inv_bw, G.nb),
                       bin_coord(qz, G.origin, G.inv_bw, G.nb)};
    int cnt = 0;
    float r = fmaxf(r0, 0.5f * G.bw);
    float rprev2 = -1.0f;                    // bins with mindist2 <= rprev2 were scanned
    for (int it = 0;; it++) {
        const float rm = r + G.margin;
        const float rm2 = rm * rm;
        int lo[3], hi[3];
        bool wraps = false, full_all = true;
        for (int a = 0; a < 3; a++) {
            // one extra bin each side: the min-distance test decides, so the box
            // only has to contain every bin that test can accept
            lo[a] = (int)floorf((q[a] - rm - G.origin) * G.inv_bw) - 1;
            hi[a] = (int)floorf((q[a] + rm - G.origin) * G.inv_bw) + 1;
            if (G.periodic) {
                if (hi[a] - lo[a] + 2 >= G.nb) wraps = true;
            } else {
                lo[a] = max(lo[a], 0);
                hi[a] = min(hi[a], G.nb - 1);
                if (lo[a] > 0 || hi[a] < G.nb - 1) full_all = false;
            }
        }
        if (wraps) {
            // the ball reaches around a periodic box: scan every bin once, exactly
            cnt = 0;
            const int64_t nbins = (int64_t)G.nb * G.nb * G.nb;
            for (int64_t bb = 0; bb < nbins; bb++) scan_bin(G, (int)bb, qx, qy, qz, col, S, K, cnt);
            break;
        }
        for (int bz = lo[2]; bz <= hi[2]; bz++)
            for (int by = lo[1]; by <= hi[1]; by++)
                for (int bx = lo[0]; bx <= hi[0]; bx++) {
                    const float md = bin_mindist2(G, q, bx, by, bz);
                    if (md > rm2 || md <= rprev2) continue;
                    const int wx = G.periodic ? wrap_bin(bx, G.nb) : bx;
                    const int wy = G.periodic ? wrap_bin(by, G.nb) : by;
                    const int wz = G.periodic ? wrap_bin(bz, G.nb) : bz;
                    scan_bin(G, wx + G.nb * (wy + G.nb * wz), qx, qy, qz, col, S, K, cnt);
                }
        if (!G.periodic && full_all) break;           // every bin scanned
        if (cnt == K && key_d2(col[(size_t)(K - 1) * S]) <= __fmul_rn(r, r)) break;
        rprev2 = rm2;
        r *= 1.5f;
    }
    return cnt;
}

// exact kNN: shells of bins, or the radius-guided search when a starting
// radius is available for q's bin
template <int KCAP>
__device__ __forceinline__ int knn_any(const KnnGrid &G, float qx, float qy, float qz, int K,
                                       unsigned long long *col, int S) {
    if (G.r0) {
        const int b = bin_coord(qx, G.origin, G.inv_bw, G.nb) +
                      G.nb * (bin_coord(qy, G.origin, G.inv_bw, G.nb) + G.nb * bin_coord(qz, G.origin, G.inv_bw, G.nb));
        return knn_query_radius<KCAP>(G, qx, qy, qz, K, col, S, G.r0[b]);
    }
    return knn_query<KCAP>(G, qx, qy, qz, K, col, S);
}

}  // namespace avism
