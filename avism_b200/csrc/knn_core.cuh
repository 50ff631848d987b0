// knn_core.cuh -- device-side exact kNN on binned particles.
//
// One thread per query.  The current best K keys live in a shared-memory
// column (stride = blockDim.x, conflict-free), sorted ascending.  A key is
// (float bits of the squared distance) << 32 | position in the binned array;
// keys order by squared distance, and equal distances by the smaller original
// particle index (held in sp[pos].w), so the order does not depend on binning.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace avism {

#define KNN_THREADS(KCAP) ((KCAP) <= 32 ? 256 : (KCAP) <= 64 ? 128 : (KCAP) <= 128 ? 64 : 32)

struct KnnGrid {
    const float4 *sp;
    const int64_t *start;
    const int32_t *fstart;    // quarter-bin x offsets (BinnedParticles::fstart) or null
    int nb;
    float origin, bw, inv_bw, box, margin;
    int periodic;
    const float *r0;          // per-bin starting radius of the radius-guided search, or null
    float occ;                // mean particles per bin
    float dmax;               // no two particles are farther apart than this
    unsigned long long *stats;  // warp kNN counters or null: queries, attempts, scanned, kept, fallbacks
};

inline KnnGrid make_knn_grid(const BinnedParticles &bp) {
    KnnGrid G;
    G.sp = bp.sp;
    G.start = bp.start;
    G.fstart = bp.fstart;
    G.nb = bp.nb;
    G.origin = bp.origin;
    G.bw = bp.bw;
    G.inv_bw = bp.inv_bw;
    G.box = bp.box;
    G.periodic = bp.periodic;
    G.margin = 2e-3f * bp.bw + 1e-6f * bp.box;
    G.r0 = nullptr;
    G.occ = (float)((double)bp.n / ((double)bp.nb * bp.nb * bp.nb));
    G.dmax = 1.7321f * bp.box * 1.001f;
    G.stats = nullptr;
    return G;
}

__host__ __device__ __forceinline__ int bin_coord(float x, float origin, float inv_bw, int nb) {
    int b = (int)floorf((x - origin) * inv_bw);
    return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}
// quarter-bin cell along x: 4t is exact, so fine_coord / 4 == bin_coord
constexpr int KNN_XF = 4;
__host__ __device__ __forceinline__ int fine_coord(float x, float origin, float inv_bw, int nb) {
    const float f = ((x - origin) * inv_bw) * (float)KNN_XF;
    return f < 0.0f ? 0 : (f >= (float)(KNN_XF * nb) ? KNN_XF * nb - 1 : (int)floorf(f));
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

__device__ __forceinline__ unsigned long long knn_key(float d2, uint32_t pos) {
    return ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned long long)pos;
}
__device__ __forceinline__ float key_d2(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }
// position of the particle in the binned array
__device__ __forceinline__ uint32_t key_pos(unsigned long long k) { return (uint32_t)(k & 0xffffffffu); }
// original (input-order, 0-based) index of the particle
__device__ __forceinline__ uint32_t key_orig(const float4 *sp, unsigned long long k) {
    return (uint32_t)__float_as_int(sp[key_pos(k)].w);
}
// equal squared distances: the smaller original index first (kept out of line,
// ties are rare and the hot comparisons stay two instructions)
static __device__ __noinline__ bool key_tie_lt(const float4 *sp, unsigned long long a, unsigned long long b) {
    if (a == b) return false;
    return key_orig(sp, a) < key_orig(sp, b);
}
// a < b in (squared distance, original index) order; ~0 (no key) is above all
__device__ __forceinline__ bool key_lt(const float4 *sp, unsigned long long a, unsigned long long b) {
    if ((uint32_t)(a >> 32) != (uint32_t)(b >> 32)) return a < b;
    return key_tie_lt(sp, a, b);
}

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

// The current best K keys of one query: a sorted shared-memory column (stride
// S), its count, and tau = the K-th key once the column is full (before that the
// proposed-radius bound, or ~0).
struct TopK {
    unsigned long long *col;
    int S, K, cnt;
    unsigned long long tau;
    bool tie;                 // a tie in squared distance may decide the result
};

// Key order of the fast pass is (squared distance, binned position): one 64-bit
// compare.  It can differ from the exact order (squared distance, original
// index) only when two keys with equal squared distance are compared, so the
// fast pass flags every comparison against tau with an equal squared distance
// and every eviction that leaves tau at the evicted distance; a flagged query
// is searched again with the exact order.
template <bool EXACT>
__device__ __forceinline__ bool key_before(const float4 *sp, unsigned long long a, unsigned long long b) {
    if constexpr (EXACT) return key_lt(sp, a, b);
    else return a < b;
}

template <bool EXACT>
__device__ __forceinline__ void topk_offer(const float4 *sp, TopK &T, unsigned long long key) {
    if constexpr (!EXACT) T.tie |= (uint32_t)(key >> 32) == (uint32_t)(T.tau >> 32);
    if (!key_before<EXACT>(sp, key, T.tau)) return;
    int i = T.cnt < T.K ? T.cnt++ : T.K - 1;
    while (i > 0) {
        const unsigned long long prev = T.col[(size_t)(i - 1) * T.S];
        if (!key_before<EXACT>(sp, key, prev)) break;
        T.col[(size_t)i * T.S] = prev;
        i--;
    }
    T.col[(size_t)i * T.S] = key;
    if (T.cnt == T.K) {
        const unsigned long long nt = T.col[(size_t)(T.K - 1) * T.S];
        if constexpr (!EXACT) T.tie |= (uint32_t)(nt >> 32) == (uint32_t)(T.tau >> 32);
        T.tau = nt;
    }
}

// candidates [a, e) of the binned array
template <bool EXACT>
__device__ __forceinline__ void scan_range(const KnnGrid &G, int64_t a, int64_t e, float qx, float qy, float qz,
                                           TopK &T) {
    int64_t p = a;
    for (; p + 1 < e; p += 2) {                    // two independent loads in flight
        const float4 v0 = G.sp[p], v1 = G.sp[p + 1];
        const float d0 = dist2_ref(v0.x, v0.y, v0.z, qx, qy, qz, G.box, G.periodic);
        const float d1 = dist2_ref(v1.x, v1.y, v1.z, qx, qy, qz, G.box, G.periodic);
        topk_offer<EXACT>(G.sp, T, knn_key(d0, (uint32_t)p));
        topk_offer<EXACT>(G.sp, T, knn_key(d1, (uint32_t)(p + 1)));
    }
    if (p < e) {
        const float4 v = G.sp[p];
        const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, G.periodic);
        topk_offer<EXACT>(G.sp, T, knn_key(d2, (uint32_t)p));
    }
}

// bins bx0..bx1 (unwrapped, at most nb of them) of one (by, bz) row
template <bool EXACT>
__device__ __forceinline__ void scan_row(const KnnGrid &G, int row, int bx0, int bx1, float qx, float qy, float qz,
                                         TopK &T) {
    if (!G.periodic) {
        scan_range<EXACT>(G, G.start[row + bx0], G.start[row + bx1 + 1], qx, qy, qz, T);
        return;
    }
    const int w0 = wrap_bin(bx0, G.nb), n = bx1 - bx0 + 1;
    if (w0 + n <= G.nb) {
        scan_range<EXACT>(G, G.start[row + w0], G.start[row + w0 + n], qx, qy, qz, T);
    } else {                                       // the run wraps around x
        scan_range<EXACT>(G, G.start[row + w0], G.start[row + G.nb], qx, qy, qz, T);
        scan_range<EXACT>(G, G.start[row], G.start[row + (w0 + n - G.nb)], qx, qy, qz, T);
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

// Lower bound of |q - p| along one axis for any particle p binned into the bin
// with unwrapped index bu: the gap to the bin's slab less the rounding margin.
__device__ __forceinline__ float axis_gap(const KnnGrid &G, float q, int bu) {
    const float lo = G.origin + (float)bu * G.bw, hi = lo + G.bw;
    return fmaxf(fmaxf(fmaxf(lo - q, q - hi), 0.0f) - G.margin, 0.0f);
}

// K nearest of q in the order of key_before<EXACT>; returns the number found
// (K unless fewer particles).  Shells of bins outward from q's bin.  While tau
// is finite, a row of bins whose (y, z) gap exceeds it is skipped, and in a kept
// row only the bins within the remaining x reach are scanned: tau only
// decreases, so a skipped bin can never hold a closer particle later.
// r0 > 0 is a proposed search radius: tau starts just above r0^2, so only
// particles within r0 are ever inserted.  If the visited block covers the ball
// of radius r0 and fewer than K particles were found, the search is repeated
// without the bound; the result is the same either way.
// The fast pass (EXACT false) sets *tie when equal squared distances may have
// been ordered by binned position (see topk_offer).
template <int KCAP, bool EXACT>
__device__ int knn_search(const KnnGrid &G, float qx, float qy, float qz, int K,
                          unsigned long long *col, int S, float r0, bool *tie) {
    const int b[3] = {bin_coord(qx, G.origin, G.inv_bw, G.nb), bin_coord(qy, G.origin, G.inv_bw, G.nb),
                      bin_coord(qz, G.origin, G.inv_bw, G.nb)};
    const float q[3] = {qx, qy, qz};
    TopK T;
    T.col = col;
    T.S = S;
    T.K = K;
    T.tie = false;
    for (int attempt = 0; attempt < 2; attempt++) {
        const bool bounded = attempt == 0 && r0 > 0.0f;
        const float r02 = __fmul_rn(r0, r0);
        // smallest key with a squared distance above r0^2 (position 0 is a valid index)
        T.tau = bounded ? knn_key(__uint_as_float(__float_as_uint(r02) + 1u), 0u) : ~0ULL;
        T.cnt = 0;
        T.tie = false;
        bool retry = false;
        for (int s = 0;; s++) {
            int lz, hz, ly, hy, lx, hx;
            axis_window(G, b[2], s, lz, hz);
            axis_window(G, b[1], s, ly, hy);
            axis_window(G, b[0], s, lx, hx);
            // pruning needs the unwrapped geometry to stand for the periodic images
            const bool prune = !G.periodic || 2 * s + 3 < G.nb;
            for (int dz = lz; dz <= hz; dz++) {
                const int bz = G.periodic ? wrap_bin(b[2] + dz, G.nb) : b[2] + dz;
                const float gz = axis_gap(G, qz, b[2] + dz);
                const float gz2 = __fmul_rn(gz, gz);
                if (prune && T.tau != ~0ULL && gz2 > key_d2(T.tau)) continue;
                for (int dy = ly; dy <= hy; dy++) {
                    const bool face = (dz == s || dz == -s || dy == s || dy == -s);
                    int xl = lx, xh = hx;
                    if (prune && T.tau != ~0ULL) {
                        const float gy = axis_gap(G, qy, b[1] + dy);
                        const float yz2 = __fadd_rn(gz2, __fmul_rn(gy, gy));
                        const float t = key_d2(T.tau);
                        if (yz2 > t) continue;
                        const float rx = __fadd_rn(__fsqrt_rn(__fsub_rn(t, yz2)), G.margin);
                        const int cl = (int)floorf(__fmul_rn(__fsub_rn(__fsub_rn(qx, rx), G.origin), G.inv_bw));
                        const int ch = (int)floorf(__fmul_rn(__fsub_rn(__fadd_rn(qx, rx), G.origin), G.inv_bw));
                        // near the periodic seam the images' bins are not monotone in x: keep the shell range
                        if (!G.periodic || (cl >= 0 && ch <= G.nb - 1)) {
                            xl = max(xl, cl - b[0]);
                            xh = min(xh, ch - b[0]);
                        }
                    }
                    const int by = G.periodic ? wrap_bin(b[1] + dy, G.nb) : b[1] + dy;
                    const int row = G.nb * (by + G.nb * bz);
                    if (face) {
                        if (xl <= xh) scan_row<EXACT>(G, row, b[0] + xl, b[0] + xh, qx, qy, qz, T);
                    } else {
                        if (lx == -s && xl <= -s) scan_row<EXACT>(G, row, b[0] - s, b[0] - s, qx, qy, qz, T);
                        if (hx == s && xh >= s) scan_row<EXACT>(G, row, b[0] + s, b[0] + s, qx, qy, qz, T);
                    }
                }
            }
            bool all_done;
            const float r = guaranteed_radius(G, b, q, s, &all_done);
            if (all_done) {
                retry = bounded && T.cnt < K;
                break;
            }
            if (T.cnt == K && r > 0.0f) {
                const float kth = key_d2(col[(size_t)(K - 1) * S]);
                if (kth < __fmul_rn(r, r)) break;
            }
            if (bounded && T.cnt < K && r > 0.0f && key_d2(T.tau) < __fmul_rn(r, r)) {
                retry = true;                  // fewer than K particles within r0
                break;
            }
        }
        if (!retry) break;
    }
    if constexpr (!EXACT) {
        // equal squared distances inside the list are ordered by position
        for (int i = 1; i < T.cnt; i++)
            T.tie |= (uint32_t)(col[(size_t)i * S] >> 32) == (uint32_t)(col[(size_t)(i - 1) * S] >> 32);
        *tie = T.tie;
    }
    return T.cnt;
}

// Exact K nearest of q in (squared distance, original index) order: the fast
// pass, repeated with the exact order when a tie may have decided it.
template <int KCAP>
__device__ __forceinline__ int knn_query(const KnnGrid &G, float qx, float qy, float qz, int K,
                                         unsigned long long *col, int S, float r0 = 0.0f) {
    bool tie = false;
    const int cnt = knn_search<KCAP, false>(G, qx, qy, qz, K, col, S, r0, &tie);
    if (!tie) return cnt;
    return knn_search<KCAP, true>(G, qx, qy, qz, K, col, S, r0, nullptr);
}

// exact kNN; with a per-bin proposed radius when one is available
template <int KCAP>
__device__ __forceinline__ int knn_any(const KnnGrid &G, float qx, float qy, float qz, int K,
                                       unsigned long long *col, int S) {
    float r0 = 0.0f;
    if (G.r0) {
        const int b = bin_coord(qx, G.origin, G.inv_bw, G.nb) +
                      G.nb * (bin_coord(qy, G.origin, G.inv_bw, G.nb) + G.nb * bin_coord(qz, G.origin, G.inv_bw, G.nb));
        r0 = G.r0[b];
    }
    return knn_query<KCAP>(G, qx, qy, qz, K, col, S, r0);
}

}  // namespace avism
