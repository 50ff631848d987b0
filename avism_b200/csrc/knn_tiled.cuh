// knn_tiled.cuh -- exact kNN for spatial tiles of queries, candidates staged in
// shared memory.
//
// A CTA owns a tile of queries (a block of grid cells, or the particles of a
// block of bins).  It loads the particles of the bins covering the tile, then
// shells of bins around that block, chunk by chunk, into shared memory; every
// thread scans the same chunk (broadcast reads) for its own query.  A thread
// keeps its current best K keys sorted in a shared-memory column; candidates
// below its K-th key go to a small per-thread buffer (a predicated store), and
// a warp merges its buffers into the lists when any lane's buffer is full.
// After each shell a query is done when its K-th distance is below the
// distance to the boundary of the loaded block; the tile stops when all its
// queries are done.  Results are the exact K smallest (d2, particle index)
// keys, with d2 computed as distance() in src/kdtree.f90:1441-1465.
#pragma once

#include <cub/cub.cuh>

#include "knn_core.cuh"

namespace avism {

constexpr int TK_THREADS = 64;     // queries per round
constexpr int TK_BUF = 8;          // per-thread candidate buffer
constexpr int TK_CHUNK = 512;      // staged candidates per pass
constexpr int TK_MAXBINS = 512;    // bins per staging batch

using TkScan = cub::BlockScan<int, TK_THREADS>;

template <int KCAP>
struct TkSmem {
    typename TkScan::TempStorage scan;
    float4 cand[TK_CHUNK];
    unsigned long long list[KCAP][TK_THREADS];
    unsigned long long buf[TK_BUF][TK_THREADS];
    int32_t bin[TK_MAXBINS];
    int32_t pre[TK_MAXBINS + 1];
    int32_t qrow[65];              // particle tiles: prefix of query counts per bin row
    int64_t qbeg[64];              // particle tiles: first sorted particle of each row
};

// merge a thread's buffer into its sorted list (keeps the K smallest)
template <int KCAP>
__device__ __forceinline__ void tk_flush(TkSmem<KCAP> &S, int tid, int K, int &cnt, int &nb,
                                         unsigned long long &tau) {
    for (int b = 0; b < nb; b++) {
        const unsigned long long key = S.buf[b][tid];
        int i;
        if (cnt < K) {
            i = cnt++;
        } else {
            if (key >= S.list[K - 1][tid]) continue;
            i = K - 1;
        }
        while (i > 0) {
            const unsigned long long prev = S.list[i - 1][tid];
            if (prev <= key) break;
            S.list[i][tid] = prev;
            i--;
        }
        S.list[i][tid] = key;
    }
    nb = 0;
    tau = cnt == K ? S.list[K - 1][tid] : ~0ULL;
}

// block of bins [lo, hi] per axis (unwrapped); per axis "full" when it covers
// every bin of a periodic axis
struct BinBlock {
    int lo[3], hi[3];
};

__device__ __forceinline__ bool axis_full(const KnnGrid &G, const BinBlock &B, int a) {
    return G.periodic && (B.hi[a] - B.lo[a] + 1 >= G.nb);
}

// distance from q to the boundary of the loaded block (inf where nothing lies beyond)
__device__ __forceinline__ float block_radius(const KnnGrid &G, const BinBlock &B, const float q[3], bool *all) {
    float r = FLT_MAX;
    bool done = true;
    for (int a = 0; a < 3; a++) {
        if (G.periodic) {
            if (axis_full(G, B, a)) continue;
            r = fminf(r, fminf(q[a] - (G.origin + (float)B.lo[a] * G.bw), (G.origin + (float)(B.hi[a] + 1) * G.bw) - q[a]));
            done = false;
        } else {
            if (B.lo[a] > 0) { r = fminf(r, q[a] - (G.origin + (float)B.lo[a] * G.bw)); done = false; }
            if (B.hi[a] < G.nb - 1) { r = fminf(r, (G.origin + (float)(B.hi[a] + 1) * G.bw) - q[a]); done = false; }
        }
    }
    *all = done;
    return r - G.margin;
}

// Scan all bins of block `now` not in block `prev` (prev empty when prev.lo > prev.hi).
template <int KCAP>
__device__ void tk_scan_shell(const KnnGrid &G, TkSmem<KCAP> &S, const BinBlock &now, const BinBlock &prev,
                              bool has_prev, bool active, float qx, float qy, float qz, int K, int &cnt, int &nb,
                              unsigned long long &tau) {
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    // per-axis ranges of distinct bins (clip / wrap)
    int lo[3], hi[3];
    bool full[3];
    for (int a = 0; a < 3; a++) {
        full[a] = axis_full(G, now, a);
        if (full[a]) { lo[a] = 0; hi[a] = G.nb - 1; }
        else if (G.periodic) { lo[a] = now.lo[a]; hi[a] = now.hi[a]; }
        else { lo[a] = max(now.lo[a], 0); hi[a] = min(now.hi[a], G.nb - 1); }
    }
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    const int64_t nbins = (int64_t)nx * ny * nz;
    for (int64_t b0 = 0; b0 < nbins; b0 += TK_MAXBINS) {
        // collect the new bins of this batch with their particle counts
        const int nbatch = (int)min((int64_t)TK_MAXBINS, nbins - b0);
        // each thread handles TK_MAXBINS / TK_THREADS consecutive bins of the batch
        constexpr int PER = TK_MAXBINS / TK_THREADS;
        int cnts[PER];
        for (int k = 0; k < PER; k++) {
            const int t = tid * PER + k;
            int bin = -1, n = 0;
            if (t < nbatch) {
                const int64_t id = b0 + t;
                const int ux = (int)(id % nx), uy = (int)((id / nx) % ny), uz = (int)(id / ((int64_t)nx * ny));
                const int v[3] = {lo[0] + ux, lo[1] + uy, lo[2] + uz};
                // was this bin in the previous block?
                bool old = has_prev;
                for (int a = 0; a < 3 && old; a++) {
                    if (axis_full(G, prev, a)) continue;
                    const int span = prev.hi[a] - prev.lo[a];
                    if (full[a]) {
                        int d = (v[a] - prev.lo[a]) % G.nb;
                        if (d < 0) d += G.nb;
                        if (d > span) old = false;
                    } else if (v[a] < prev.lo[a] || v[a] > prev.hi[a]) {
                        old = false;
                    }
                }
                if (!old) {
                    const int bx = G.periodic ? wrap_bin(v[0], G.nb) : v[0];
                    const int by = G.periodic ? wrap_bin(v[1], G.nb) : v[1];
                    const int bz = G.periodic ? wrap_bin(v[2], G.nb) : v[2];
                    bin = bx + G.nb * (by + G.nb * bz);
                    n = (int)(G.start[bin + 1] - G.start[bin]);
                }
                S.bin[t] = bin;
            }
            cnts[k] = n;
        }
        int excl[PER];
        int agg;
        TkScan(S.scan).ExclusiveSum(cnts, excl, agg);
        for (int k = 0; k < PER; k++) {
            const int t = tid * PER + k;
            if (t < nbatch) S.pre[t] = excl[k];
        }
        if (tid == 0) S.pre[nbatch] = agg;
        __syncthreads();
        const int total = S.pre[nbatch];
        for (int c0 = 0; c0 < total; c0 += TK_CHUNK) {
            const int nchunk = min(TK_CHUNK, total - c0);
            // stage the chunk: candidate c0+u lives in the bin found by search
            for (int u = tid; u < nchunk; u += blockDim.x) {
                const int g = c0 + u;
                int l = 0, h = nbatch;          // largest t with pre[t] <= g
                while (h - l > 1) {
                    const int m = (l + h) >> 1;
                    if (S.pre[m] <= g) l = m; else h = m;
                }
                S.cand[u] = G.sp[G.start[S.bin[l]] + (g - S.pre[l])];
            }
            __syncthreads();
            for (int u = 0; u < nchunk; u++) {
                if (active) {
                    const float4 p = S.cand[u];
                    const float d2 = dist2_ref(p.x, p.y, p.z, qx, qy, qz, G.box, G.periodic);
                    const unsigned long long key = knn_key(d2, (uint32_t)__float_as_int(p.w));
                    if (key < tau) S.buf[nb++][tid] = key;
                }
                if (__any_sync(0xffffffffu, nb == TK_BUF)) tk_flush<KCAP>(S, tid, K, cnt, nb, tau);
            }
            __syncthreads();
        }
        (void)lane;
        __syncthreads();        // S.bin / S.pre / S.scan are reused by the next batch
    }
}

// Exact kNN of the thread's query inside a tile whose queries lie in the
// block of bins `start`.  Returns the count (K unless fewer particles exist);
// the sorted keys are S.list[0..cnt-1][tid].
template <int KCAP>
__device__ int tk_query_tile(const KnnGrid &G, TkSmem<KCAP> &S, const BinBlock &start, bool active, float qx,
                             float qy, float qz, int K) {
    const int tid = threadIdx.x;
    int cnt = 0, nb = 0;
    unsigned long long tau = ~0ULL;
    bool done = !active;
    BinBlock prev = start, now = start;
    bool has_prev = false;
    const float q[3] = {qx, qy, qz};
    for (int s = 0;; s++) {
        tk_scan_shell<KCAP>(G, S, now, prev, has_prev, active && !done, qx, qy, qz, K, cnt, nb, tau);
        if (active) tk_flush<KCAP>(S, tid, K, cnt, nb, tau);
        bool all;
        const float r = block_radius(G, now, q, &all);
        if (active && !done) {
            if (all) done = true;
            else if (cnt == K && r > 0.0f && key_d2(S.list[K - 1][tid]) < __fmul_rn(r, r)) done = true;
        }
        if (__syncthreads_and(done ? 1 : 0)) break;
        bool everything = true;
        for (int a = 0; a < 3; a++) {
            if (G.periodic) everything &= axis_full(G, now, a);
            else everything &= (now.lo[a] <= 0 && now.hi[a] >= G.nb - 1);
        }
        if (everything) break;
        prev = now;
        has_prev = true;
        for (int a = 0; a < 3; a++) {
            now.lo[a] -= 1;
            now.hi[a] += 1;
        }
    }
    return cnt;
}

}  // namespace avism
