// knn_group.cuh -- exact kNN of 32 neighbouring queries per warp, one per lane,
// over particle tiles staged in shared memory.
//
// The queries of a warp lie close together (a 4x4x2 tile of grid cells, or 32
// consecutive particles of the binned order), so their searches read nearly the
// same particles.  The warp walks the rows of bins that any of its queries can
// reach once: 32 candidates at a time are staged in shared memory, and every
// lane tests all of them against its own query (a broadcast read per
// candidate) and appends those within its radius R to its own column of kept
// candidates.  A lane whose column ends with K to CAP candidates holds its K
// nearest (nothing outside its ball can be closer); it ranks them exactly by
// (squared distance, original particle index), the order of knn_search
// (src/kdtree.f90:504-540, distance() at 1441-1465), with an insertion sort of
// its column.  A lane with fewer than K or more than CAP kept candidates is
// answered afterwards by the whole warp with knn_warp_exact.  The radius is a
// starting point only: the neighbour lists do not depend on it.
#pragma once

#include <climits>

#include "knn_core.cuh"
#include "knn_warp.cuh"

namespace avism {

template <int KMAX>
struct __align__(16) GroupKnnSmem {
    static constexpr int CAP = 2 * KMAX;          // kept candidates per lane
    uint32_t d2[CAP][32];                         // lane l's column: [j][l]
    uint32_t pos[CAP][32];
    float4 stage[32];                             // the batch of candidates under test
    uint32_t stage_pos[32];
    uint32_t seg_base[WQ_SEGS];
    int32_t seg_end[WQ_SEGS];
    WarpKnnSmem<KMAX> w;                          // the warp search of the lanes that need one
};

__device__ __forceinline__ float warp_min_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// (squared distance, original index) order of two kept candidates
__device__ __forceinline__ bool cand_lt(const KnnGrid &G, uint32_t da, uint32_t pa, uint32_t db, uint32_t pb) {
    if (da != db) return da < db;
    return __float_as_int(G.sp[pa].w) < __float_as_int(G.sp[pb].w);
}

// One batch of up to 32 rows of the group window (row r = rbase + lane; rows
// y = ly + r % ny, z = lz + r / ny, in bins, possibly outside [0, nb) when the
// window wraps): their particle segments over the x range [fx0, fx1] of quarter
// bins (or bins [bx0, bx1] without quarter-bin offsets) go to smem; returns the
// candidate count.
__device__ __forceinline__ int group_rows(const KnnGrid &G, int ly, int ny, float inv_ny, int lz, int nrows,
                                          int rbase, int bx0, int bx1, int fx0, int fx1, uint32_t *seg_base,
                                          int32_t *seg_end, int *nseg_out) {
    const int lane = threadIdx.x & 31;
    const int r = rbase + lane;
    uint32_t s0 = 0, s1 = 0;
    int l0 = 0, l1 = 0;
    if (r < nrows) {
        const int rz = (int)(((float)r + 0.5f) * inv_ny);       // exact: r, ny < 2^12
        const int y = ly + (r - rz * ny), z = lz + rz;
        const int by = G.periodic ? wrap_near(y, G.nb) : y;
        const int bz = G.periodic ? wrap_near(z, G.nb) : z;
        if (G.fstart) {
            const int nf = KNN_XF * G.nb;
            const int32_t *F = G.fstart + (int64_t)nf * (by + (int64_t)G.nb * bz);
            const int fn = fx1 - fx0 + 1;
            if (!G.periodic || (fx0 >= 0 && fx1 < nf)) {
                s0 = (uint32_t)F[fx0];
                l0 = F[fx1 + 1] - F[fx0];
            } else {
                const int w0 = wrap_near(fx0, nf);
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
        } else {
            const int64_t row = (int64_t)G.nb * (by + (int64_t)G.nb * bz);
            const int n = bx1 - bx0 + 1;
            if (!G.periodic || (bx0 >= 0 && bx1 < G.nb)) {
                s0 = (uint32_t)G.start[row + bx0];
                l0 = (int)(G.start[row + bx1 + 1] - G.start[row + bx0]);
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

// bin window of one axis covering [lo, hi] (coordinates); periodic windows of
// more than nb bins are cut to one period (no bin twice)
__device__ __forceinline__ void group_axis(const KnnGrid &G, float lo, float hi, int &b0, int &b1) {
    b0 = (int)floorf(__fmul_rn(__fsub_rn(lo, G.origin), G.inv_bw));
    b1 = (int)floorf(__fmul_rn(__fsub_rn(hi, G.origin), G.inv_bw));
    if (G.periodic) {
        if (b1 - b0 + 1 >= G.nb) { b0 = 0; b1 = G.nb - 1; }
    } else {
        b0 = max(b0, 0);
        b1 = min(b1, G.nb - 1);
    }
}

// bins apart along one axis (the shorter way round when periodic)
__device__ __forceinline__ int bin_apart(const KnnGrid &G, int a, int b) {
    const int d = abs(a - b);
    return G.periodic ? min(d, G.nb - d) : d;
}

// Scan of one subgroup (the member lanes): every member lane's candidates
// within its radius go to its column; returns the lane's kept count.
template <int KMAX, bool STATS>
__device__ int group_scan(const KnnGrid &G, bool member, float qx, float qy, float qz, float R,
                          GroupKnnSmem<KMAX> &S) {
    constexpr int CAP = GroupKnnSmem<KMAX>::CAP;
    const int lane = threadIdx.x & 31;
    const float reach = __fadd_rn(R, G.margin);
    const float R2 = __fmul_rn(R, R);
    // the window holding every member's ball
    const float BIG = 3.0e38f;
    const float xlo = warp_min_f(member ? qx - reach : BIG), xhi = warp_max_f(member ? qx + reach : -BIG);
    const float ylo = warp_min_f(member ? qy - reach : BIG), yhi = warp_max_f(member ? qy + reach : -BIG);
    const float zlo = warp_min_f(member ? qz - reach : BIG), zhi = warp_max_f(member ? qz + reach : -BIG);
    int bx0, bx1, by0, by1, bz0, bz1;
    group_axis(G, xlo, xhi, bx0, bx1);
    group_axis(G, ylo, yhi, by0, by1);
    group_axis(G, zlo, zhi, bz0, bz1);
    // quarter bins along x: the particles' quarter-bin cells are monotone in x
    int fx0 = KNN_XF * bx0, fx1 = KNN_XF * bx1 + KNN_XF - 1;
    if (G.fstart && !(G.periodic && bx1 - bx0 + 1 == G.nb)) {
        fx0 = max(fx0, (int)floorf(__fmul_rn(__fsub_rn(xlo, G.origin), G.inv_bw) * (float)KNN_XF));
        fx1 = min(fx1, (int)floorf(__fmul_rn(__fsub_rn(xhi, G.origin), G.inv_bw) * (float)KNN_XF));
    }
    // no image of a candidate closer than the plain difference: the window
    // spans less than half the box along every axis and does not wrap
    const bool plain_d = !G.periodic ||
                         (bx0 >= 0 && bx1 < G.nb && by0 >= 0 && by1 < G.nb && bz0 >= 0 && bz1 < G.nb &&
                          2 * (bx1 - bx0 + 1) + 2 <= G.nb && 2 * (by1 - by0 + 1) + 2 <= G.nb &&
                          2 * (bz1 - bz0 + 1) + 2 <= G.nb);
    const int ny = by1 - by0 + 1, nz = bz1 - bz0 + 1, nrows = ny * nz;
    const float inv_ny = 1.0f / (float)ny;
    int n = 0;
    for (int rbase = 0; rbase < nrows; rbase += 32) {
        int nseg;
        const int T = group_rows(G, by0, ny, inv_ny, bz0, nrows, rbase, bx0, bx1, fx0, fx1, S.seg_base,
                                 S.seg_end, &nseg);
        int k0 = 0;
        for (int cb = 0; cb < T; cb += 32) {
            const int g = cb + lane;
            const int e = k0 + lane < nseg ? S.seg_end[k0 + lane] : INT_MAX;
            const unsigned endmask = __reduce_or_sync(0xffffffffu, e - cb <= 31 ? 1u << (e - cb) : 0u);
            const int seg = k0 + __popc(endmask & ((2u << lane) - 1u));
            k0 += __popc(endmask);
            if (g < T) {
                const uint32_t p = S.seg_base[seg] + (uint32_t)g;
                S.stage[lane] = G.sp[p];
                S.stage_pos[lane] = p;
            }
            __syncwarp();
            const int m = min(32, T - cb);
            if (plain_d) {
                for (int t = 0; t < m; t++) {
                    const float4 v = S.stage[t];
                    const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, 0);
                    if (member && d2 <= R2) {
                        if (n < CAP) { S.d2[n][lane] = __float_as_uint(d2); S.pos[n][lane] = S.stage_pos[t]; }
                        n++;
                    }
                }
            } else {
                for (int t = 0; t < m; t++) {
                    const float4 v = S.stage[t];
                    const float d2 = dist2_ref(v.x, v.y, v.z, qx, qy, qz, G.box, 1);
                    if (member && d2 <= R2) {
                        if (n < CAP) { S.d2[n][lane] = __float_as_uint(d2); S.pos[n][lane] = S.stage_pos[t]; }
                        n++;
                    }
                }
            }
            __syncwarp();
        }
        if (STATS && lane == 0) atomicAdd(&G.stats[2], (unsigned long long)T * 32ull);
    }
    return n;
}

// Exact K nearest (K <= KMAX) of every active lane's query q, from radius R.
// All 32 lanes call it.  Returns the lane's neighbour count; its neighbours are
// S.d2[0..cnt)[lane] / S.pos[0..cnt)[lane], ascending.  Lanes scan together
// in subgroups of queries within GROUP_SPAN bins of each other per axis and
// radii within a factor 2, so that one far or wide query cannot blow up the
// window of the rest (the end of a row of bins in the binned order, a void
// cell next to a cluster).
constexpr int GROUP_SPAN = 4;

template <int KMAX, bool STATS = false>
__device__ int group_knn(const KnnGrid &G, bool active, float qx, float qy, float qz, float R, int K,
                         GroupKnnSmem<KMAX> &S) {
    constexpr int CAP = GroupKnnSmem<KMAX>::CAP;
    const int lane = threadIdx.x & 31;
    __syncwarp();                                  // the previous group's columns have been read
    const int bx = bin_coord(qx, G.origin, G.inv_bw, G.nb), by = bin_coord(qy, G.origin, G.inv_bw, G.nb);
    const int bz = bin_coord(qz, G.origin, G.inv_bw, G.nb);
    int n = 0;
    unsigned pending = __ballot_sync(0xffffffffu, active);
    while (pending) {
        const int L = __ffs(pending) - 1;
        const int lx = __shfl_sync(0xffffffffu, bx, L), ly = __shfl_sync(0xffffffffu, by, L);
        const int lz = __shfl_sync(0xffffffffu, bz, L);
        const float lr = __shfl_sync(0xffffffffu, R, L);
        const bool member = ((pending >> lane) & 1u) && bin_apart(G, bx, lx) <= GROUP_SPAN &&
                            bin_apart(G, by, ly) <= GROUP_SPAN && bin_apart(G, bz, lz) <= GROUP_SPAN &&
                            R <= 2.0f * lr && lr <= 2.0f * R;
        pending &= ~__ballot_sync(0xffffffffu, member);
        const int nm = group_scan<KMAX, STATS>(G, member, qx, qy, qz, R, S);
        if (member) n = nm;
    }
    bool fail = active && (n < K || n > CAP);
    if (active && !fail) {
        // the K smallest of the column, ascending: insertion into a sorted prefix
        // of at most K entries (later candidates beyond the K-th are dropped)
        int len = 0;
        for (int i = 0; i < n; i++) {
            const uint32_t d = S.d2[i][lane], p = S.pos[i][lane];
            if (len == K && !cand_lt(G, d, p, S.d2[K - 1][lane], S.pos[K - 1][lane])) continue;
            int j = len < K ? len++ : K - 1;
            while (j > 0 && cand_lt(G, d, p, S.d2[j - 1][lane], S.pos[j - 1][lane])) {
                S.d2[j][lane] = S.d2[j - 1][lane];
                S.pos[j][lane] = S.pos[j - 1][lane];
                j--;
            }
            S.d2[j][lane] = d;
            S.pos[j][lane] = p;
        }
        n = K;
    }
    if (STATS) {
        const unsigned act = __ballot_sync(0xffffffffu, active);
        unsigned s = (unsigned)(active ? min(n, CAP) : 0);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            atomicAdd(&G.stats[0], (unsigned long long)__popc(act));
            atomicAdd(&G.stats[1], (unsigned long long)__popc(act));
            atomicAdd(&G.stats[3], (unsigned long long)s);
        }
    }
    // lanes whose radius did not fit: the whole warp searches for each in turn
    unsigned todo = __ballot_sync(0xffffffffu, fail);
    if (STATS && lane == 0 && todo) atomicAdd(&G.stats[4], (unsigned long long)__popc(todo));
    __syncwarp();
    while (todo) {
        const int L = __ffs(todo) - 1;
        todo &= todo - 1;
        const float x = __shfl_sync(0xffffffffu, qx, L), y = __shfl_sync(0xffffffffu, qy, L);
        const float z = __shfl_sync(0xffffffffu, qz, L), r = __shfl_sync(0xffffffffu, R, L);
        const int cnt = knn_warp_exact<KMAX, STATS>(G, x, y, z, K, r, S.w,
                                                    reinterpret_cast<unsigned long long *>(S.w.d2));
        for (int j = lane; j < cnt; j += 32) {
            S.d2[j][L] = S.w.res_d2[j];
            S.pos[j][L] = S.w.res_pos[j];
        }
        if (lane == L) n = cnt;
        __syncwarp();
    }
    __syncwarp();
    return active ? n : 0;
}

}  // namespace avism
