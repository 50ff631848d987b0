// knn_warp.cuh -- warp-cooperative exact kNN from a proposed search radius.
//
// One warp answers one query.  Given a radius R, the warp lists every row of
// bins that the ball of radius R around the query can touch (one row per lane,
// pruned in y/z by the row's gap and in x by the remaining reach, exactly as
// knn_search prunes; with quarter-bin offsets the x range is cut at a quarter
// of a bin), concatenates the rows' particle ranges and scans them 32
// candidates at a time with all lanes busy.  Candidates with squared distance
// <= R^2 are kept in a shared-memory buffer.  If at least K were kept, the K
// nearest overall are the K smallest kept ones (nothing outside the ball can be
// closer), and they are ranked exactly by (squared distance, original particle
// index) -- the order of knn_search -- by a bitonic sort verified on the full
// squared distances, or by a counting select when that check fails.  If fewer than K
// were kept the radius grows; if more than the buffer holds it shrinks; after a
// bounded number of attempts the query falls back to knn_search.  The radius is
// therefore only a starting point: the neighbour lists do not depend on it.
#pragma once

#include <climits>

#include "knn_core.cuh"

namespace avism {

constexpr int WQ_SEGS = 64;          // row segments per batch of 32 rows (two per row when x wraps)
constexpr int WQ_ATTEMPTS = 12;      // radius attempts before falling back to knn_search

template <int KMAX>
struct __align__(16) WarpKnnSmem {
    static constexpr int CAP = 4 * KMAX;    // kept candidates per attempt
    uint32_t d2[CAP];                       // float bits of the squared distance
    uint32_t pos[CAP];                      // position in the binned array
    uint32_t seg_base[WQ_SEGS];             // binned position of each segment's first candidate
                                            // minus its offset in the batch (mod 2^32)
    int32_t seg_end[WQ_SEGS];               // running end offset of each segment
    uint32_t res_d2[KMAX];                  // result, ascending (squared distance, index)
    uint32_t res_pos[KMAX];
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// default starting radius: the K-th neighbour distance of a uniform density
// equal to the mean bin occupancy
__device__ __forceinline__ float knn_uniform_radius(const KnnGrid &G, int K) {
    return 1.15f * G.bw * cbrtf((float)K / (4.18879020f * fmaxf(G.occ, 1e-3f)));
}

// One batch of up to 32 rows (row r = rbase + lane): write their particle
// segments to smem and return the total number of candidates.
// b in [-nb, 2nb): the bin it wraps to
__device__ __forceinline__ int wrap_near(int b, int nb) { return b < 0 ? b + nb : (b >= nb ? b - nb : b); }

__device__ __forceinline__ int wq_rows(const KnnGrid &G, const int b[3], float qx, float qy, float qz,
                                       float R2, bool prune, int lx, int hx, int ly, int ny, float inv_ny, int lz,
                                       int nrows, int rbase, uint32_t *seg_base, int32_t *seg_end,
                                       int *nseg_out) {
    const int lane = threadIdx.x & 31;
    const int r = rbase + lane;
    uint32_t s0 = 0, s1 = 0;
    int l0 = 0, l1 = 0;
    if (r < nrows) {
        // r = ry + ny * rz; the float quotient is exact here (r, ny < 2^12)
        const int rz = (int)(((float)r + 0.5f) * inv_ny);
        const int dy = ly + (r - rz * ny), dz = lz + rz;
        bool keep = true;
        int xl = lx, xh = hx;
        int fl = INT_MIN, fh = INT_MAX;                 // quarter-bin x range (G.fstart)
        if (prune) {
            const float gz = axis_gap(G, qz, b[2] + dz);
            const float gz2 = __fmul_rn(gz, gz);
            const float gy = axis_gap(G, qy, b[1] + dy);
            const float yz2 = __fadd_rn(gz2, __fmul_rn(gy, gy));
            if (gz2 > R2 || yz2 > R2) {
                keep = false;
            } else {
                // the reach only prunes (with the margin), so an approximate root does
                const float rem = R2 - yz2;
                const float rx = (rem > 0.0f ? rem * rsqrtf(rem) * 1.000001f : 0.0f) + G.margin;
                const float tl = __fmul_rn(__fsub_rn(__fsub_rn(qx, rx), G.origin), G.inv_bw);
                const float th = __fmul_rn(__fsub_rn(__fadd_rn(qx, rx), G.origin), G.inv_bw);
                const int cl = (int)floorf(tl), ch = (int)floorf(th);
                // near the periodic seam the images' bins are not monotone in x: keep the window
                if (!G.periodic || (cl >= 0 && ch <= G.nb - 1)) {
                    xl = max(xl, cl - b[0]);
                    xh = min(xh, ch - b[0]);
                    // particles' quarter-bin cells are floor(4 t) of the same t: monotone in x
                    fl = (int)floorf(tl * (float)KNN_XF);
                    fh = (int)floorf(th * (float)KNN_XF);
                }
            }
        }
        if (keep && xl <= xh) {
            const int bz = G.periodic ? wrap_near(b[2] + dz, G.nb) : b[2] + dz;
            const int by = G.periodic ? wrap_near(b[1] + dy, G.nb) : b[1] + dy;
            const int64_t row = (int64_t)G.nb * (by + (int64_t)G.nb * bz);
            const int bx0 = b[0] + xl, n = xh - xl + 1;
            if (G.fstart) {
                // the same rows at a quarter of a bin along x; the cells' offsets are
                // in bin order, so a wrapped window splits as the bins' does
                const int nf = KNN_XF * G.nb;
                const int f0 = max(KNN_XF * bx0, fl), f1 = min(KNN_XF * (bx0 + n) - 1, fh);
                const int fn = f1 - f0 + 1;
                const int64_t frow = (int64_t)nf * (by + (int64_t)G.nb * bz);
                const int32_t *F = G.fstart + frow;
                if (fn <= 0) {
                } else if (!G.periodic) {
                    s0 = (uint32_t)F[f0];
                    l0 = F[f0 + fn] - F[f0];
                } else {
                    const int w0 = wrap_near(f0, nf);
                    if (w0 + fn <= nf) {
                        s0 = (uint32_t)F[w0];
                        l0 = F[w0 + fn] - F[w0];
                    } else {
                        s0 = (uint32_t)F[w0];
                        l0 = F[nf] - F[w0];
                        s1 = (uint32_t)F[0];
                        l1 = F[w0 + fn - nf] - F[0];
                    }
                }
            } else if (!G.periodic) {
                s0 = (uint32_t)G.start[row + bx0];
                l0 = (int)(G.start[row + bx0 + n] - G.start[row + bx0]);
            } else {
                const int w0 = wrap_near(bx0, G.nb);
                if (w0 + n <= G.nb) {
                    s0 = (uint32_t)G.start[row + w0];
                    l0 = (int)(G.start[row + w0 + n] - G.start[row + w0]);
                } else {
                    s0 = (uint32_t)G.start[row + w0];
                    l0 = (int)(G.start[row + G.nb] - G.start[row + w0]);
                    s1 = (uint32_t)G.start[row];
                    l1 = (int)(G.start[row + (w0 + n - G.nb)] - G.start[row]);
                }
            }
        }
    }
    // segment slots and candidate offsets: warp-inclusive scans
    const int ns = (l0 > 0) + (l1 > 0);
    const int lt = l0 + l1;
    int si = ns, li = lt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, si, o), c = __shfl_up_sync(0xffffffffu, li, o);
        if (lane >= o) { si += a; li += c; }
    }
    int k = si - ns, off = li - lt;
    if (l0 > 0) { seg_base[k] = s0 - (uint32_t)off; seg_end[k] = off + l0; k++; off += l0; }
    if (l1 > 0) { seg_base[k] = s1 - (uint32_t)off; seg_end[k] = off + l1; }
    *nseg_out = __shfl_sync(0xffffffffu, si, 31);
    __syncwarp();
    return __shfl_sync(0xffffffffu, li, 31);
}

// Bitonic sort of one 32-bit key per lane, ascending (DESC: descending).  The
// keys carry their payload in the low bits, so a stage is one shuffle and a
// min or max.
template <bool DESC>
__device__ __forceinline__ void warp_sort32(uint32_t &key) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, key, j);
            const bool keep_min = (((lane & j) == 0) == ((lane & k) == 0)) != DESC;
            key = keep_min ? min(key, o) : max(key, o);
        }
    }
}
// a ascending and b descending in lockstep: one lane predicate per stage and two
// independent shuffle chains
__device__ __forceinline__ void warp_sort32x2(uint32_t &a, uint32_t &b) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t oa = __shfl_xor_sync(0xffffffffu, a, j), ob = __shfl_xor_sync(0xffffffffu, b, j);
            const bool lo = ((lane & j) == 0) == ((lane & k) == 0);
            a = lo ? min(a, oa) : max(a, oa);
            b = lo ? max(b, ob) : min(b, ob);
        }
    }
}
// a ascending, b descending: the 32 smallest of both, ascending (DESC: descending).
// The lane-wise minimum is a bitonic sequence holding them; half-cleaners sort it.
template <bool DESC>
__device__ __forceinline__ void warp_merge32(uint32_t &a, uint32_t b) {
    const int lane = threadIdx.x & 31;
    a = min(a, b);
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const uint32_t o = __shfl_xor_sync(0xffffffffu, a, j);
        const bool keep_min = ((lane & j) == 0) != DESC;
        a = keep_min ? min(a, o) : max(a, o);
    }
}

// The K <= 32 nearest of the n <= 128 kept candidates.  Each key packs the
// squared distance's bits (shifted past the always-zero sign bit, low seven
// bits dropped) above the candidate's 7-bit slot, and the keys are sorted with
// warp bitonic networks.  The result is then verified on the full squared
// distances: the first m = min(n, K) must be strictly ascending (no tie, no pair
// misordered by the dropped bits) and exactly m kept candidates may lie at or
// below the m-th.  Then they are the m nearest in the exact order; otherwise it
// returns false and the caller ranks exactly.
template <int KMAX>
__device__ __forceinline__ bool bitonic_select(const KnnGrid &G, int n, int K, WarpKnnSmem<KMAX> &S) {
    static_assert(WarpKnnSmem<KMAX>::CAP <= 128, "slots must fit in 7 bits");
    const int lane = threadIdx.x & 31;
    uint32_t k[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int e = q * 32 + lane;
        k[q] = e < n ? (((S.d2[e] << 1) & ~0x7fu) | (uint32_t)e) : 0xffffffffu;
    }
    const int ns = (n + 31) >> 5;
    if (ns > 1) {
        warp_sort32x2(k[0], k[1]);
        warp_merge32<false>(k[0], k[1]);
    } else {
        warp_sort32<false>(k[0]);
    }
    if (ns > 2) {
        if (ns > 3) {
            warp_sort32x2(k[2], k[3]);
            warp_merge32<true>(k[2], k[3]);
        } else {
            warp_sort32<true>(k[2]);
        }
        warp_merge32<false>(k[0], k[2]);
    }
    const int m = min(n, K);
    const uint32_t slot = k[0] & 0x7fu;
    const uint32_t d = lane < m ? S.d2[slot] : 0xffffffffu;
    const uint32_t dn = __shfl_down_sync(0xffffffffu, d, 1);
    const uint32_t dk = __shfl_sync(0xffffffffu, d, m - 1);
    const bool bad = lane < m - 1 && !(d < dn);
    int le = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int e = q * 32 + lane;
        le += __popc(__ballot_sync(0xffffffffu, e < n && S.d2[e] <= dk));
    }
    if (__any_sync(0xffffffffu, bad) || le > m) return false;
    if (lane < m) {
        S.res_d2[lane] = d;
        S.res_pos[lane] = S.pos[slot];
    }
    __syncwarp();
    return true;
}

// Exact K nearest of q (K <= KMAX) by the warp; all 32 lanes must call it with
// the same arguments.  Returns the neighbour count (K unless fewer particles)
// with S.res_d2 / S.res_pos holding them in ascending order, or -1 when the
// attempts ran out (the caller then runs knn_search).
// STATS: count queries, attempts and candidates into G.stats (a separate
// instantiation, so the counters cost nothing when they are off)
template <int KMAX, bool STATS = false>
__device__ int knn_warp(const KnnGrid &G, float qx, float qy, float qz, int K, float r0, WarpKnnSmem<KMAX> &S) {
    constexpr int CAP = WarpKnnSmem<KMAX>::CAP;
    const int lane = threadIdx.x & 31;
    __syncwarp();                              // the previous query's results have been read
    const int b[3] = {bin_coord(qx, G.origin, G.inv_bw, G.nb), bin_coord(qy, G.origin, G.inv_bw, G.nb),
                      bin_coord(qz, G.origin, G.inv_bw, G.nb)};
    float R = r0 > 0.0f ? r0 : knn_uniform_radius(G, K);
    float r_lo = 0.0f, r_hi = FLT_MAX;       // known too small / known too large
    for (int attempt = 0; attempt < WQ_ATTEMPTS; attempt++) {
        const float R2 = __fmul_rn(R, R);
        const float reach = __fmul_rn(__fadd_rn(R, G.margin), G.inv_bw);
        const int s = reach >= (float)G.nb ? G.nb : (int)ceilf(reach);
        int lz, hz, ly, hy, lx, hx;
        axis_window(G, b[2], s, lz, hz);
        axis_window(G, b[1], s, ly, hy);
        axis_window(G, b[0], s, lx, hx);
        const int ny = hy - ly + 1, nz = hz - lz + 1;
        const int nrows = ny * nz;
        const float inv_ny = 1.0f / (float)ny;
        // no wrapped image inside the window: |dx| < L/2 for every candidate, so
        // min(|dx|, L - |dx|) = |dx| and the plain distance has the same bits
        const bool plain_d = !G.periodic || (b[0] + lx >= 0 && b[0] + hx < G.nb && b[1] + ly >= 0 &&
                                             b[1] + hy < G.nb && b[2] + lz >= 0 && b[2] + hz < G.nb &&
                                             4 * s + 2 <= G.nb);
        bool all_done;
        if (G.periodic) all_done = 2 * s + 1 >= G.nb;
        else all_done = b[0] + lx == 0 && b[0] + hx == G.nb - 1 && b[1] + ly == 0 && b[1] + hy == G.nb - 1 &&
                        b[2] + lz == 0 && b[2] + hz == G.nb - 1;
        const bool prune = !G.periodic || 2 * s + 3 < G.nb;
        int count = 0;
        for (int rbase = 0; rbase < nrows; rbase += 32) {
            int nseg;
            const int T = wq_rows(G, b, qx, qy, qz, R2, prune, lx, hx, ly, ny, inv_ny, lz, nrows, rbase,
                                  S.seg_base, S.seg_end, &nseg);
            int k0 = 0;                                  // first segment ending after this chunk's start
            for (int cb = 0; cb < T; cb += 32) {
                const int g = cb + lane;
                // segment of candidate g = number of segment ends <= g: the ends in
                // [cb, cb + 31] as one OR-reduced mask (ends are distinct, so at most 32)
                const int e = k0 + lane < nseg ? S.seg_end[k0 + lane] : INT_MAX;
                const unsigned endmask = __reduce_or_sync(0xffffffffu, e - cb <= 31 ? 1u << (e - cb) : 0u);
                const int seg = k0 + __popc(endmask & ((2u << lane) - 1u));
                k0 += __popc(endmask);
                bool pass = false;
                uint32_t d2b = 0, p = 0;
                if (g < T) {
                    p = S.seg_base[seg] + (uint32_t)g;
                    const float4 v = G.sp[p];
                    const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, plain_d ? 0 : 1);
                    pass = d2 <= R2;
                    d2b = __float_as_uint(d2);
                }
                const uint32_t m = __ballot_sync(0xffffffffu, pass);
                if (pass) {
                    const int slot = count + __popc(m & lanemask_lt());
                    if (slot < CAP) { S.d2[slot] = d2b; S.pos[slot] = p; }
                }
                count += __popc(m);
            }
            if (STATS && lane == 0) atomicAdd(&G.stats[2], (unsigned long long)T);
            __syncwarp();
        }
        if (count > CAP) {                               // too many: shrink
            r_hi = R;
            float Rn = __fmul_rn(R, cbrtf(0.5f * (float)(K + CAP) / (float)count));
            if (!(Rn > r_lo)) Rn = 0.5f * (r_lo + R);
            R = Rn;
            continue;
        }
        if (count < K && !(all_done && R >= G.dmax)) {   // too few: grow
            r_lo = R;
            float Rn = __fmul_rn(R, fmaxf(1.26f, cbrtf(1.5f * (float)K / (float)max(count, 1))));
            if (!(Rn < r_hi)) Rn = 0.5f * (R + r_hi);
            R = Rn;
            continue;
        }
        const int n = count;
        if (STATS && lane == 0) {
            atomicAdd(&G.stats[0], 1ULL);
            atomicAdd(&G.stats[1], (unsigned long long)(attempt + 1));
            atomicAdd(&G.stats[3], (unsigned long long)n);
        }
        if constexpr (KMAX == 32) {
            if (bitonic_select(G, n, K, S)) return min(n, K);
            if (STATS && lane == 0) atomicAdd(&G.stats[5], 1ULL);
        }
        // counting select: rank = #smaller squared distances + #equal ones with a smaller index
        for (int e = lane; e < n; e += 32) {
            const uint32_t de = S.d2[e];
            int rank = 0, eq = 0;
            for (int f = 0; f < n; f++) {
                const uint32_t df = S.d2[f];
                rank += df < de;
                eq += df == de;
            }
            if (eq > 1) {                                // a tie in squared distance: order by index
                const uint32_t oe = (uint32_t)__float_as_int(G.sp[S.pos[e]].w);
                for (int f = 0; f < n; f++)
                    if (S.d2[f] == de && f != e && (uint32_t)__float_as_int(G.sp[S.pos[f]].w) < oe) rank++;
            }
            if (rank < K) { S.res_d2[rank] = de; S.res_pos[rank] = S.pos[e]; }
        }
        __syncwarp();
        return min(n, K);
    }
    if (STATS && lane == 0) atomicAdd(&G.stats[4], 1ULL);
    return -1;
}

// knn_search for lane 0 when knn_warp gave up; results copied to S.res_*.
template <int KMAX>
__device__ int knn_warp_fallback(const KnnGrid &G, float qx, float qy, float qz, int K, WarpKnnSmem<KMAX> &S,
                                 unsigned long long *col) {
    int cnt = 0;
    if ((threadIdx.x & 31) == 0) {
        cnt = knn_query<KMAX>(G, qx, qy, qz, K, col, 1, 0.0f);
        for (int i = 0; i < cnt; i++) {
            S.res_d2[i] = (uint32_t)(col[i] >> 32);
            S.res_pos[i] = key_pos(col[i]);
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, cnt, 0);
}

// exact kNN of one query by the whole warp
template <int KMAX, bool STATS = false>
__device__ __forceinline__ int knn_warp_exact(const KnnGrid &G, float qx, float qy, float qz, int K, float r0,
                                              WarpKnnSmem<KMAX> &S, unsigned long long *col) {
    const int cnt = knn_warp<KMAX, STATS>(G, qx, qy, qz, K, r0, S);
    if (cnt >= 0) return cnt;
    return knn_warp_fallback<KMAX>(G, qx, qy, qz, K, S, col);
}

}  // namespace avism
