// knn_warp.cuh -- warp-cooperative exact kNN from a proposed search radius.
//
// One warp answers one query.  Given a radius R, the warp lists every row of
// bins that the ball of radius R around the query can touch (one row per lane,
// pruned in y/z by the row's gap and in x by the remaining reach, exactly as
// knn_search prunes), concatenates the rows' particle ranges and scans them 32
// candidates at a time with all lanes busy.  Candidates with squared distance
// <= R^2 are kept in a shared-memory buffer.  If at least K were kept, the K
// nearest overall are the K smallest kept ones (nothing outside the ball can be
// closer), and they are ranked exactly by (squared distance, original particle
// index) -- the order of knn_search -- with a counting select.  If fewer than K
// were kept the radius grows; if more than the buffer holds it shrinks; after a
// bounded number of attempts the query falls back to knn_search.  The radius is
// therefore only a starting point: the neighbour lists do not depend on it.
#pragma once

#include "knn_core.cuh"

namespace avism {

constexpr int WQ_SEGS = 64;          // row segments per batch of 32 rows (two per row when x wraps)
constexpr int WQ_ATTEMPTS = 12;      // radius attempts before falling back to knn_search

template <int KMAX>
struct __align__(16) WarpKnnSmem {
    static constexpr int CAP = 4 * KMAX;    // kept candidates per attempt
    uint32_t d2[CAP];                       // float bits of the squared distance
    uint32_t pos[CAP];                      // position in the binned array
    uint32_t seg_start[WQ_SEGS];            // first binned position of each segment
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
__device__ __forceinline__ int wq_rows(const KnnGrid &G, const int b[3], float qx, float qy, float qz,
                                       float R2, bool prune, int lx, int hx, int ly, int ny, int lz,
                                       int nrows, int rbase, uint32_t *seg_start, int32_t *seg_end,
                                       int *nseg_out) {
    const int lane = threadIdx.x & 31;
    const int r = rbase + lane;
    uint32_t s0 = 0, s1 = 0;
    int l0 = 0, l1 = 0;
    if (r < nrows) {
        const int dy = ly + r % ny, dz = lz + r / ny;
        bool keep = true;
        int xl = lx, xh = hx;
        if (prune) {
            const float gz = axis_gap(G, qz, b[2] + dz);
            const float gz2 = __fmul_rn(gz, gz);
            const float gy = axis_gap(G, qy, b[1] + dy);
            const float yz2 = __fadd_rn(gz2, __fmul_rn(gy, gy));
            if (gz2 > R2 || yz2 > R2) {
                keep = false;
            } else {
                const float rx = __fadd_rn(__fsqrt_rn(__fsub_rn(R2, yz2)), G.margin);
                const int cl = (int)floorf(__fmul_rn(__fsub_rn(__fsub_rn(qx, rx), G.origin), G.inv_bw));
                const int ch = (int)floorf(__fmul_rn(__fsub_rn(__fadd_rn(qx, rx), G.origin), G.inv_bw));
                // near the periodic seam the images' bins are not monotone in x: keep the window
                if (!G.periodic || (cl >= 0 && ch <= G.nb - 1)) {
                    xl = max(xl, cl - b[0]);
                    xh = min(xh, ch - b[0]);
                }
            }
        }
        if (keep && xl <= xh) {
            const int bz = G.periodic ? wrap_bin(b[2] + dz, G.nb) : b[2] + dz;
            const int by = G.periodic ? wrap_bin(b[1] + dy, G.nb) : b[1] + dy;
            const int64_t row = (int64_t)G.nb * (by + (int64_t)G.nb * bz);
            const int bx0 = b[0] + xl, n = xh - xl + 1;
            if (!G.periodic) {
                s0 = (uint32_t)G.start[row + bx0];
                l0 = (int)(G.start[row + bx0 + n] - G.start[row + bx0]);
            } else {
                const int w0 = wrap_bin(bx0, G.nb);
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
    if (l0 > 0) { seg_start[k] = s0; seg_end[k] = off + l0; k++; off += l0; }
    if (l1 > 0) { seg_start[k] = s1; seg_end[k] = off + l1; }
    *nseg_out = __shfl_sync(0xffffffffu, si, 31);
    __syncwarp();
    return __shfl_sync(0xffffffffu, li, 31);
}

// Exact K nearest of q (K <= KMAX) by the warp; all 32 lanes must call it with
// the same arguments.  Returns the neighbour count (K unless fewer particles)
// with S.res_d2 / S.res_pos holding them in ascending order, or -1 when the
// attempts ran out (the caller then runs knn_search).
template <int KMAX>
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
        bool all_done;
        if (G.periodic) all_done = 2 * s + 1 >= G.nb;
        else all_done = b[0] + lx == 0 && b[0] + hx == G.nb - 1 && b[1] + ly == 0 && b[1] + hy == G.nb - 1 &&
                        b[2] + lz == 0 && b[2] + hz == G.nb - 1;
        const bool prune = !G.periodic || 2 * s + 3 < G.nb;
        int count = 0;
        for (int rbase = 0; rbase < nrows; rbase += 32) {
            int nseg;
            const int T = wq_rows(G, b, qx, qy, qz, R2, prune, lx, hx, ly, ny, lz, nrows, rbase, S.seg_start,
                                  S.seg_end, &nseg);
            for (int cb = 0; cb < T; cb += 32) {
                const int g = cb + lane;
                bool pass = false;
                uint32_t d2b = 0, p = 0;
                if (g < T) {
                    int lo = 0, hi = nseg - 1;           // first segment whose end exceeds g
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (S.seg_end[mid] > g) hi = mid; else lo = mid + 1;
                    }
                    const int begin = lo == 0 ? 0 : S.seg_end[lo - 1];
                    p = S.seg_start[lo] + (uint32_t)(g - begin);
                    const float4 v = G.sp[p];
                    const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, G.periodic);
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
        // counting select: rank = #smaller squared distances + #equal ones with a smaller index
        const int n = count;
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
template <int KMAX>
__device__ __forceinline__ int knn_warp_exact(const KnnGrid &G, float qx, float qy, float qz, int K, float r0,
                                              WarpKnnSmem<KMAX> &S, unsigned long long *col) {
    const int cnt = knn_warp<KMAX>(G, qx, qy, qz, K, r0, S);
    if (cnt >= 0) return cnt;
    return knn_warp_fallback<KMAX>(G, qx, qy, qz, K, S, col);
}

}  // namespace avism
