// indexx.cu -- the exact permutation of INDEXX (src/num.f90:2-84) in parallel.
//
// INDEXX is the Numerical Recipes index quicksort: median-of-3 pivot (with the
// reference's compare order), Hoare partition, straight insertion below 7
// elements.  It is not stable, and the catalogue depends on how it orders equal
// keys (equal divergences of periodic ghost cells; equal cube volumes), so the
// GPU reproduces its permutation exactly rather than sorting stably.
//
// A Hoare partition of segment [l, ir] around pivot a = key(l) pairs the m-th
// position (from the left, starting at l+2) holding a key >= a with the m-th
// position (from the right, starting at ir-1) holding a key <= a, and swaps the
// pairs until they cross.  These lists come from two prefix sums, so one
// partition step of every large segment runs in parallel; disjoint segments
// evolve independently, so processing them level by level yields the same
// permutation as the reference's stack order.  Segments of at most
// SMALL_SEG elements finish with the sequential algorithm, one thread each.
#include <cub/cub.cuh>
#include <climits>

#include "common.cuh"

namespace avism {

static constexpr int SMALL_SEG = 48;

struct Seg {
    int32_t l, ir;      // 1-based, inclusive
    float a;            // pivot key
    int32_t cge, cle;   // list lengths
    int32_t mstar, i, j;
};

__device__ __forceinline__ void swp(float *K, int32_t *I, int32_t p, int32_t q) {   // 1-based
    const float tk = K[p - 1];
    K[p - 1] = K[q - 1];
    K[q - 1] = tk;
    const int32_t ti = I[p - 1];
    I[p - 1] = I[q - 1];
    I[q - 1] = ti;
}

// sequential INDEXX restricted to [l0, ir0] (all of it lies inside the segment)
__device__ void nr_sequential(float *K, int32_t *I, int32_t l0, int32_t ir0) {
    const int M = 7;
    int32_t stack[64];
    int js = 0;
    int32_t l = l0, ir = ir0;
    for (;;) {
        if (ir - l < M) {
            for (int32_t j = l + 1; j <= ir; j++) {
                const float a = K[j - 1];
                const int32_t ia = I[j - 1];
                int32_t i = j - 1;
                // the reference scans down to position 1; every key left of l
                // is <= a, so the scan always stops by l-1
                for (; i >= l; i--) {
                    if (K[i - 1] <= a) break;
                    K[i] = K[i - 1];
                    I[i] = I[i - 1];
                }
                K[i] = a;
                I[i] = ia;
            }
            if (js == 0) return;
            ir = stack[--js];
            l = stack[--js];
        } else {
            const int32_t k = (l + ir) / 2;
            swp(K, I, k, l + 1);
            if (K[l] > K[ir - 1]) swp(K, I, l + 1, ir);
            if (K[l - 1] > K[ir - 1]) swp(K, I, l, ir);
            if (K[l] > K[l - 1]) swp(K, I, l + 1, l);
            int32_t i = l + 1, j = ir;
            const float a = K[l - 1];
            const int32_t ia = I[l - 1];
            for (;;) {
                do i++; while (K[i - 1] < a);
                do j--; while (K[j - 1] > a);
                if (j < i) break;
                swp(K, I, i, j);
            }
            K[l - 1] = K[j - 1];
            I[l - 1] = I[j - 1];
            K[j - 1] = a;
            I[j - 1] = ia;
            if (ir - i + 1 >= j - l) {
                stack[js++] = i;
                stack[js++] = ir;
                ir = j - 1;
            } else {
                stack[js++] = l;
                stack[js++] = j - 1;
                l = i;
            }
        }
    }
}

__global__ void k_init_idx(int32_t n, const float *__restrict__ key_in, float *__restrict__ K, int32_t *__restrict__ I) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    K[i] = key_in[i];
    I[i] = i + 1;
}

__global__ void k_small(const Seg *__restrict__ segs, int32_t nseg, float *K, int32_t *I) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    nr_sequential(K, I, segs[s].l, segs[s].ir);
}

// median-of-3 exactly as src/num.f90:41-60
__global__ void k_med3(Seg *segs, int32_t nseg, float *K, int32_t *I) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int32_t l = segs[s].l, ir = segs[s].ir;
    const int32_t k = (l + ir) / 2;
    swp(K, I, k, l + 1);
    if (K[l] > K[ir - 1]) swp(K, I, l + 1, ir);
    if (K[l - 1] > K[ir - 1]) swp(K, I, l, ir);
    if (K[l] > K[l - 1]) swp(K, I, l + 1, l);
    segs[s].a = K[l - 1];
}

// owner segment of each position in a large segment (-1 elsewhere)
__global__ void k_seg_of(const Seg *__restrict__ segs, int32_t *__restrict__ seg_of) {
    const int32_t s = blockIdx.x;
    const int32_t l = segs[s].l, ir = segs[s].ir;
    for (int32_t p = l + threadIdx.x; p <= ir; p += blockDim.x) seg_of[p - 1] = s;
}

__global__ void k_flags_ge_le(int32_t n, const Seg *__restrict__ segs, const int32_t *__restrict__ seg_of,
                              const float *__restrict__ K, int32_t *__restrict__ ge, int32_t *__restrict__ le) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int32_t s = seg_of[x];
    int32_t g = 0, e = 0;
    if (s >= 0) {
        const int32_t p = x + 1, l = segs[s].l, ir = segs[s].ir;
        const float a = segs[s].a, v = K[x];
        g = (p >= l + 2 && v >= a) ? 1 : 0;
        e = (p >= l + 1 && p <= ir - 1 && v <= a) ? 1 : 0;
    }
    ge[x] = g;
    le[x] = e;
}

// prefix sums are exclusive over 0-based x: P[x] = flags at positions < x+1 (1-based)
__global__ void k_lists(int32_t n, Seg *segs, const int32_t *__restrict__ seg_of,
                        const int32_t *__restrict__ ge, const int32_t *__restrict__ le,
                        const int32_t *__restrict__ Pge, const int32_t *__restrict__ Ple,
                        int32_t *__restrict__ GE, int32_t *__restrict__ LE) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int32_t s = seg_of[x];
    if (s < 0) return;
    const int32_t l = segs[s].l, ir = segs[s].ir;
    const int32_t base = l - 1;
    // totals: P[ir] (exclusive at x = ir) counts flags at positions <= ir
    const int32_t tot_ge = (ir < n ? Pge[ir] : Pge[n - 1] + ge[n - 1]) - Pge[base];
    const int32_t tot_le = (ir < n ? Ple[ir] : Ple[n - 1] + le[n - 1]) - Ple[base];
    if (ge[x]) GE[base + (Pge[x] - Pge[base])] = x + 1;
    if (le[x]) LE[base + (tot_le - 1 - (Ple[x] - Ple[base]))] = x + 1;
    if (x == base) {
        segs[s].cge = tot_ge;
        segs[s].cle = tot_le;
    }
}

// crossing point of the Hoare scans and the final i, j of the partition
__global__ void k_cross(Seg *segs, int32_t nseg, const int32_t *__restrict__ GE, const int32_t *__restrict__ LE,
                        int32_t *err) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int32_t base = segs[s].l - 1, cge = segs[s].cge, cle = segs[s].cle;
    auto G = [&](int32_t k) -> int64_t { return k < 0 ? LLONG_MIN : (k < cge ? (int64_t)GE[base + k] : LLONG_MAX); };
    auto Lq = [&](int32_t k) -> int64_t { return k < 0 ? LLONG_MAX : (k < cle ? (int64_t)LE[base + k] : LLONG_MIN); };
    // m* = first k with !(GE[k] < LE[k]); predicate is monotone
    int32_t lo = 0, hi = min(cge, cle);
    while (lo < hi) {
        const int32_t mid = (lo + hi) / 2;
        if (G(mid) < Lq(mid)) lo = mid + 1; else hi = mid;
    }
    const int32_t m = lo;
    int64_t i, j;
    if (G(m) == Lq(m)) {             // the scans meet on a key equal to the pivot
        i = min(G(m + 1), Lq(m - 1));
        j = max(Lq(m + 1), G(m - 1));
    } else {
        i = min(G(m), Lq(m - 1));
        j = max(Lq(m), G(m - 1));
    }
    const int32_t l = segs[s].l, ir = segs[s].ir;
    if (i < l + 1 || i > ir + 1 || j < l || j > ir - 1 || i <= j) {
        // not a valid Hoare crossing: flag it and leave the segment untouched
        atomicOr(err, 1);
        segs[s].mstar = 0;
        segs[s].i = ir + 1;
        segs[s].j = l;
        return;
    }
    segs[s].mstar = m;
    segs[s].i = (int32_t)i;
    segs[s].j = (int32_t)j;
}

__global__ void k_swap_pairs(int32_t n, const Seg *__restrict__ segs, const int32_t *__restrict__ seg_of,
                             const int32_t *__restrict__ ge, const int32_t *__restrict__ Pge,
                             const int32_t *__restrict__ LE, float *K, int32_t *I) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int32_t s = seg_of[x];
    if (s < 0 || !ge[x]) return;
    const int32_t base = segs[s].l - 1;
    const int32_t k = Pge[x] - Pge[base];
    if (k >= segs[s].mstar) return;
    const int32_t q = LE[base + k];
    if (q <= x + 1 || q > segs[s].ir) return;
    swp(K, I, x + 1, q);
}

// pivot into place, children into the next level's lists
__global__ void k_finish(const Seg *__restrict__ segs, int32_t nseg, float *K, int32_t *I, Seg *next_large,
                         int32_t *n_large, Seg *next_small, int32_t *n_small) {
    const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int32_t l = segs[s].l, ir = segs[s].ir, i = segs[s].i, j = segs[s].j;
    if (j < l || j > ir) return;
    swp(K, I, l, j);
    const int32_t cl[2] = {l, i}, cr[2] = {j - 1, ir};
    for (int c = 0; c < 2; c++) {
        const int32_t sz = cr[c] - cl[c] + 1;
        if (sz <= 1) continue;
        Seg t;
        t.l = cl[c];
        t.ir = cr[c];
        if (sz <= SMALL_SEG) next_small[atomicAdd(n_small, 1)] = t;
        else next_large[atomicAdd(n_large, 1)] = t;
    }
}

__global__ void k_copy_out(int32_t n, const int32_t *__restrict__ I, int32_t *__restrict__ out) {
    const int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) out[x] = I[x];
}

void indexx_device(Ctx &c, int32_t n, const float *key_in, int32_t *indx_out) {
    if (n <= 0) return;
    float *K = c.get_t<float>(B_SORT_KEY, n);
    int32_t *I = c.get_t<int32_t>(B_SORT_IDX, n);
    ++c.launches, k_init_idx<<<grid_for(n, 256), 256, 0, c.stream>>>(n, key_in, K, I);
    // segment lists: two ping-pong large lists and one small list
    const int32_t segcap = n / 2 + 8;
    Seg *large[2] = {(Seg *)c.get(B_SEG_A, sizeof(Seg) * (size_t)segcap * 2), nullptr};
    large[1] = large[0] + segcap;
    Seg *small = (Seg *)c.get(B_SEG_B, sizeof(Seg) * (size_t)segcap);
    int32_t *cnt = c.get_t<int32_t>(B_COUNTERS, 4);     // [0] large next, [1] small, [2] error
    int32_t *seg_of = c.get_t<int32_t>(B_LIST_A, n);
    int32_t *ge = c.get_t<int32_t>(B_GE, n), *le = c.get_t<int32_t>(B_LE, n);
    int32_t *Pge = c.get_t<int32_t>(B_SCAN_A, n), *Ple = c.get_t<int32_t>(B_SCAN_B, n);
    int32_t *GE = c.get_t<int32_t>(B_LIST_B, n), *LE = c.get_t<int32_t>(B_UMIN, n);
    AV_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int32_t), c.stream));
    Seg root;
    root.l = 1;
    root.ir = n;
    int32_t nlarge = 0, nsmall = 0;
    if (n <= SMALL_SEG) {
        AV_CUDA(cudaMemcpyAsync(small, &root, sizeof(Seg), cudaMemcpyHostToDevice, c.stream));
        nsmall = 1;
    } else {
        AV_CUDA(cudaMemcpyAsync(large[0], &root, sizeof(Seg), cudaMemcpyHostToDevice, c.stream));
        nlarge = 1;
    }
    int cur = 0;
    size_t tmp = 0;
    AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, ge, Pge, n, c.stream));
    void *tbuf = c.get(B_CUB_TMP, tmp);
    int32_t hcnt[2] = {0, nsmall};
    AV_CUDA(cudaMemcpyAsync(cnt + 1, &nsmall, sizeof(int32_t), cudaMemcpyHostToDevice, c.stream));
    while (nlarge > 0) {
        Seg *S = large[cur], *N = large[cur ^ 1];
        AV_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t), c.stream));
        ++c.launches, k_med3<<<grid_for(nlarge, 128), 128, 0, c.stream>>>(S, nlarge, K, I);
        AV_CUDA(cudaMemsetAsync(seg_of, 0xff, sizeof(int32_t) * (size_t)n, c.stream));
        ++c.launches, k_seg_of<<<nlarge, 256, 0, c.stream>>>(S, seg_of);
        ++c.launches, k_flags_ge_le<<<grid_for(n, 256), 256, 0, c.stream>>>(n, S, seg_of, K, ge, le);
        AV_CUDA(cub::DeviceScan::ExclusiveSum(tbuf, tmp, ge, Pge, n, c.stream));
        AV_CUDA(cub::DeviceScan::ExclusiveSum(tbuf, tmp, le, Ple, n, c.stream));
        ++c.launches, k_lists<<<grid_for(n, 256), 256, 0, c.stream>>>(n, S, seg_of, ge, le, Pge, Ple, GE, LE);
        ++c.launches, k_cross<<<grid_for(nlarge, 128), 128, 0, c.stream>>>(S, nlarge, GE, LE, cnt + 2);
        ++c.launches, k_swap_pairs<<<grid_for(n, 256), 256, 0, c.stream>>>(n, S, seg_of, ge, Pge, LE, K, I);
        ++c.launches, k_finish<<<grid_for(nlarge, 128), 128, 0, c.stream>>>(S, nlarge, K, I, N, cnt, small, cnt + 1);
        AV_CUDA(cudaGetLastError());
        AV_CUDA(cudaMemcpyAsync(hcnt, cnt, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        nlarge = hcnt[0];
        cur ^= 1;
    }
    int32_t tail[2];
    AV_CUDA(cudaMemcpyAsync(tail, cnt + 1, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    nsmall = tail[0];
    AV_CHECK(tail[1] == 0, AVISM_ERR_INTERNAL, "indexx: inconsistent partition");
    if (nsmall > 0) ++c.launches, k_small<<<grid_for(nsmall, 64), 64, 0, c.stream>>>(small, nsmall, K, I);
    ++c.launches, k_copy_out<<<grid_for(n, 256), 256, 0, c.stream>>>(n, I, indx_out);
    AV_CUDA(cudaGetLastError());
}

}  // namespace avism
