// voidfind.cu -- VOIDFIND on the device (src/voidfinding.f90:59-713).
//
// 1. candidates: cells with FLAGV (MARK_ALL) compacted in K,J,I order of the
//    ext grid, their divergence ordered by the exact INDEXX, reversed;
// 2. growth: one warp per candidate grows its cube shell by shell (the six
//    faces are checked together, lanes over face cells), with the boundary and
//    single-cell rules of src/voidfinding.f90:640-679;
// 3. acceptance: a candidate is accepted iff no earlier accepted cube covers its
//    centre.  Candidates are taken in windows of the divergence order: those
//    covered by cubes of earlier windows are dropped without growing; the rest
//    are resolved in rounds -- every still-open cube paints its rank into a
//    min-grid, a candidate whose own centre holds its own rank has no open
//    predecessor covering it and is accepted, accepted cubes paint the
//    coverage grid, covered candidates are dropped.
// Cube ids are the ranks of accepted candidates, as NVOID in the reference.
#include <cub/cub.cuh>

#include "common.cuh"
#include "knn_core.cuh"

namespace avism {

enum : uint8_t { ST_OPEN = 0, ST_ACCEPT = 1, ST_COVERED = 2, ST_EDGE = 3, ST_REJECT = 4 };

struct VfArgs {
    int low1, low2, ne, nx, ext;
    const uint8_t *flags;
    const int32_t *marcap;      // ext or null (-1 everywhere)
    const float *reqp;
    int32_t nreqp;
    float rmin_sub;
    const int32_t *cand_pos;    // ext linear index per candidate
    const int32_t *indx;        // INDEXX of the candidate keys (1-based, ascending)
    int32_t ncand;
    uint8_t *st;                // per rank
    int32_t *wv;                // half-width per rank
    uint8_t *cover;             // ext grid: covered by a cube accepted in an earlier window
    unsigned long long *umin;   // ext grid: (epoch, rank) min of open cubes
    unsigned long long *amin;   // ext grid: (window, rank) min of this window's accepted cubes
    // learned proposal of the half-width (per particle bin), or null
    const float *w0;
    int nb, periodic_bins;
    float rx1, dx, bin_origin, inv_bw, box;
    float wfac;                 // fraction of the proposed half-width swept at once
};

__device__ __forceinline__ int32_t rank_pos(const VfArgs &A, int32_t r) {
    return A.cand_pos[A.indx[A.ncand - 1 - r] - 1];
}

__device__ __forceinline__ void pos_coords(const VfArgs &A, int64_t e, int c[3]) {
    c[0] = (int)(e % A.ne) + A.low1;
    c[1] = (int)((e / A.ne) % A.ne) + A.low1;
    c[2] = (int)(e / ((int64_t)A.ne * A.ne)) + A.low1;
}

__device__ __forceinline__ int64_t eidx(const VfArgs &A, int i, int j, int k) {
    return (int64_t)(i - A.low1) + (int64_t)A.ne * ((int64_t)(j - A.low1) + (int64_t)A.ne * (k - A.low1));
}

// all six faces of the cube of half-width w pass (src/voidfinding.f90:500-619)
__device__ bool faces_pass_warp(const VfArgs &A, const int c[3], int w, int32_t indv, int lane) {
    const int side = 2 * w + 1;
    const int face = side * side;
    const int total = 6 * face;
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        bool ok = true;
        if (t < total) {
            const int f = t / face, rem = t - f * face;
            const int axis = f >> 1, s = (f & 1) ? -1 : 1;
            const int u = axis == 0 ? 1 : 0, v = axis == 2 ? 1 : 2;
            int cell[3], nb[3];
            cell[axis] = c[axis] + s * w;
            cell[u] = c[u] - w + rem % side;
            cell[v] = c[v] - w + rem / side;
            nb[0] = cell[0]; nb[1] = cell[1]; nb[2] = cell[2];
            nb[axis] += s;
            const int64_t en = eidx(A, nb[0], nb[1], nb[2]);
            const uint8_t fn = A.flags[en];
            const int bit = 1 + 2 * axis + (s > 0 ? 1 : 0);
            const int32_t mp = A.marcap ? A.marcap[en] : -1;
            ok = (fn & 0x80) && mp == indv && !(A.flags[eidx(A, cell[0], cell[1], cell[2])] & (1u << bit));
        }
        if (__any_sync(0xffffffffu, !ok)) return false;
    }
    return true;
}

// First shell in 0..cap whose faces fail, or cap + 1: every face cell of the
// cube of half-width cap checked at once.  A cell at Chebyshev distance d lies
// on the face of shell d along each axis where its offset is +-d (all six
// directions for the centre), and is checked there exactly as faces_pass_warp
// checks it; the first failing shell is the smallest failing d.
__device__ int first_failing_shell(const VfArgs &A, const int c[3], int cap, int32_t indv, int lane) {
    const int side = 2 * cap + 1;
    const int64_t total = (int64_t)side * side * side;
    int fail = cap + 1;
    for (int64_t t = lane; t < total; t += 32) {
        const int o[3] = {(int)(t % side) - cap, (int)((t / side) % side) - cap, (int)(t / ((int64_t)side * side)) - cap};
        const int d = max(abs(o[0]), max(abs(o[1]), abs(o[2])));
        if (d >= fail) continue;
        const int cell[3] = {c[0] + o[0], c[1] + o[1], c[2] + o[2]};
        const uint8_t fc = A.flags[eidx(A, cell[0], cell[1], cell[2])];
        bool ok = true;
        for (int a = 0; a < 3 && ok; a++) {
            for (int s = -1; s <= 1 && ok; s += 2) {
                if (d > 0 ? o[a] != s * d : false) continue;
                int nb[3] = {cell[0], cell[1], cell[2]};
                nb[a] += s;
                const int64_t en = eidx(A, nb[0], nb[1], nb[2]);
                const int bit = 1 + 2 * a + (s > 0 ? 1 : 0);
                const int32_t mp = A.marcap ? A.marcap[en] : -1;
                ok = (A.flags[en] & 0x80) && mp == indv && !(fc & (1u << bit));
            }
        }
        if (!ok) fail = d;
    }
    return __reduce_min_sync(0xffffffffu, fail);
}

// proposed half-width for the centre cell c: the bin of its position
__device__ __forceinline__ int proposed_width(const VfArgs &A, const int c[3]) {
    if (!A.w0) return 0;
    int b[3];
    for (int a = 0; a < 3; a++) {
        float x = A.rx1 + (float)(c[a] - 1) * A.dx;
        if (A.periodic_bins) {
            if (x < A.bin_origin) x += A.box;
            else if (x >= A.bin_origin + A.box) x -= A.box;
        }
        b[a] = bin_coord(x, A.bin_origin, A.inv_bw, A.nb);
    }
    const float w = A.w0[b[0] + (int64_t)A.nb * (b[1] + (int64_t)A.nb * b[2])] * A.wfac;
    return w > 0.0f ? min((int)w, 64) : 0;
}

// Phase 1: drop edge / covered candidates of the window, grow the others.
__global__ void k_phase1(VfArgs A, int32_t r0, int32_t r1, int32_t *open_list, int32_t *n_open) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int32_t r = r0 + (int32_t)warp;
    if (r >= r1) return;
    const int32_t e = rank_pos(A, r);
    int c[3];
    pos_coords(A, e, c);
    uint8_t st;
    int w = 0;
    if (c[0] <= A.low1 + 1 || c[1] <= A.low1 + 1 || c[2] <= A.low1 + 1 || c[0] >= A.low2 - 1 ||
        c[1] >= A.low2 - 1 || c[2] >= A.low2 - 1) {
        st = ST_EDGE;
    } else if (A.cover[e]) {
        st = ST_COVERED;
    } else {
        const int32_t indv = A.marcap ? A.marcap[e] : -1;
        bool flag1 = false;
        if (indv > 0 && A.reqp && indv <= A.nreqp && A.reqp[indv - 1] < A.rmin_sub) flag1 = true;
        bool f2 = false;
        if (!flag1) {
            // with a proposed half-width, shells 0..cap are checked in one sweep
            // (cap stops short of the first shell that touches the edge region)
            int cap = proposed_width(A, c);
            for (int a = 0; a < 3; a++)
                cap = min(cap, min(c[a] - (A.low1 + 1), (A.low2 - 1) - c[a]) - 1);
            if (cap > 0) {
                const int f = first_failing_shell(A, c, cap, indv, lane);
                w = min(f, cap);           // shells below w pass; the loop resumes at w
            }
            for (;;) {
                if (!faces_pass_warp(A, c, w, indv, lane)) break;
                w++;
                bool any = false, all = true, one_side = false;
                for (int a = 0; a < 3; a++) {
                    const bool lo = c[a] - w <= A.low1 + 1, hi = c[a] + w >= A.low2 - 1;
                    any |= lo || hi;
                    all &= lo && hi;
                    one_side |= (lo || hi) && !(lo && hi);
                }
                if (any) {
                    if (!all && one_side) f2 = true;
                    break;
                }
            }
        }
        if (w == 0) f2 = true;
        for (int a = 0; a < 3; a++)
            if (c[a] - w == A.low1 || c[a] + w == A.low2) f2 = true;
        st = f2 ? ST_REJECT : ST_OPEN;
    }
    if (lane == 0) {
        A.st[r] = st;
        A.wv[r] = w;
        if (st == ST_OPEN) open_list[atomicAdd(n_open, 1)] = r;
    }
}

__device__ __forceinline__ unsigned long long umin_key(uint32_t epoch, int32_t r) {
    return ((unsigned long long)(0xffffffffu - epoch) << 32) | (unsigned long long)(uint32_t)r;
}

// Every open cube paints (epoch, rank) into the min-grid.
__global__ void k_paint_umin(VfArgs A, const int32_t *open_list, int32_t n_open, uint32_t epoch) {
    const int lane = threadIdx.x & 31;
    const int64_t wi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wi >= n_open) return;
    const int32_t r = open_list[wi];
    const int w = A.wv[r];
    int c[3];
    pos_coords(A, rank_pos(A, r), c);
    const int side = 2 * w + 1;
    const int64_t vol = (int64_t)side * side * side;
    const unsigned long long key = umin_key(epoch, r);
    for (int64_t t = lane; t < vol; t += 32) {
        const int a = (int)(t % side), b = (int)((t / side) % side), d = (int)(t / ((int64_t)side * side));
        atomicMin(&A.umin[eidx(A, c[0] - w + a, c[1] - w + b, c[2] - w + d)], key);
    }
}

__global__ void k_decide(VfArgs A, const int32_t *open_list, int32_t n_open, uint32_t epoch, uint32_t window,
                         int32_t *next_open, int32_t *n_next, int32_t *acc_list, int32_t *n_acc) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_open) return;
    const int32_t r = open_list[t];
    const int32_t e = rank_pos(A, r);
    const unsigned long long am = A.amin[e];
    // a cube accepted in this window covers the centre only if its rank is smaller
    const bool acc_before = (uint32_t)(am >> 32) == 0xffffffffu - window && (int32_t)(uint32_t)am < r;
    if (A.cover[e] || acc_before) {
        A.st[r] = ST_COVERED;
    } else if (A.umin[e] == umin_key(epoch, r)) {
        A.st[r] = ST_ACCEPT;
        acc_list[atomicAdd(n_acc, 1)] = r;
    } else {
        next_open[atomicAdd(n_next, 1)] = r;
    }
}

// this window's accepted cubes paint (window, rank) into the accepted min-grid
__global__ void k_paint_amin(VfArgs A, const int32_t *acc_list, int32_t n_acc, uint32_t window) {
    const int lane = threadIdx.x & 31;
    const int64_t wi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wi >= n_acc) return;
    const int32_t r = acc_list[wi];
    const int w = A.wv[r];
    int c[3];
    pos_coords(A, rank_pos(A, r), c);
    const int side = 2 * w + 1;
    const int64_t vol = (int64_t)side * side * side;
    const unsigned long long key = umin_key(window, r);
    for (int64_t t = lane; t < vol; t += 32) {
        const int a = (int)(t % side), b = (int)((t / side) % side), d = (int)(t / ((int64_t)side * side));
        atomicMin(&A.amin[eidx(A, c[0] - w + a, c[1] - w + b, c[2] - w + d)], key);
    }
}

__global__ void k_paint_cover(VfArgs A, const int32_t *acc_list, int32_t n_acc) {
    const int lane = threadIdx.x & 31;
    const int64_t wi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wi >= n_acc) return;
    const int32_t r = acc_list[wi];
    const int w = A.wv[r];
    int c[3];
    pos_coords(A, rank_pos(A, r), c);
    const int side = 2 * w + 1;
    const int64_t vol = (int64_t)side * side * side;
    for (int64_t t = lane; t < vol; t += 32) {
        const int a = (int)(t % side), b = (int)((t / side) % side), d = (int)(t / ((int64_t)side * side));
        A.cover[eidx(A, c[0] - w + a, c[1] - w + b, c[2] - w + d)] = 1;
    }
}

// ---- candidate compaction --------------------------------------------------
struct IsCand {
    const uint8_t *flags;
    __host__ __device__ bool operator()(const int32_t &e) const { return flags[e] & 1; }
};

__global__ void k_cand_keys(VfArgs A, const float *dv, const int32_t *pos, int32_t n, float *key) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t e = pos[t];
    if (A.ext) {
        key[t] = dv[e];
    } else {
        int c[3];
        pos_coords(A, e, c);
        const int nx = A.nx;
        for (int a = 0; a < 3; a++) {
            if (c[a] < 1) c[a] += nx;
            else if (c[a] > nx) c[a] -= nx;
        }
        key[t] = dv[(int64_t)(c[0] - 1) + (int64_t)nx * ((int64_t)(c[1] - 1) + (int64_t)nx * (c[2] - 1))];
    }
}

struct IsAccepted {
    const uint8_t *st;
    __host__ __device__ int32_t operator()(const int32_t &r) const { return st[r] == ST_ACCEPT ? 1 : 0; }
};

__global__ void k_write_cubes(VfArgs A, const int32_t *ids, int32_t nrank, float dx, float rx1,
                              int32_t *ci, float *cf, int32_t cap) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrank || A.st[r] != ST_ACCEPT) return;
    const int32_t id = ids[r];
    if (id >= cap) return;
    const int32_t e = rank_pos(A, r);
    int c[3];
    pos_coords(A, e, c);
    const int w = A.wv[r];
    int32_t *I = ci;
    I[0 * cap + id] = c[0] - w; I[1 * cap + id] = c[0] + w;
    I[2 * cap + id] = c[1] - w; I[3 * cap + id] = c[1] + w;
    I[4 * cap + id] = c[2] - w; I[5 * cap + id] = c[2] + w;
    I[6 * cap + id] = c[0]; I[7 * cap + id] = c[1]; I[8 * cap + id] = c[2];
    I[9 * cap + id] = A.marcap ? A.marcap[e] : -1;
    const float side = __fmul_rn((float)(2 * w + 1), dx);
    cf[0 * cap + id] = __fmul_rn(__fmul_rn(side, side), side);
    const float half = __fmul_rn(0.5f, dx);
    for (int a = 0; a < 3; a++) {
        cf[(1 + 2 * a) * cap + id] = __fsub_rn(__fadd_rn(rx1, __fmul_rn((float)(c[a] - w - 1), dx)), half);
        cf[(2 + 2 * a) * cap + id] = __fadd_rn(__fadd_rn(rx1, __fmul_rn((float)(c[a] + w - 1), dx)), half);
    }
}

// last attempted rank (accepted or rejected by growth) and its accepted count
__global__ void k_nvoid_check(const uint8_t *st, const int32_t *ids, int32_t nrank, int32_t nvoid_max, int *err) {
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrank) return;
    if ((st[r] == ST_ACCEPT || st[r] == ST_REJECT) && ids[r] >= nvoid_max) atomicOr(err, 1);
}

int32_t voidfind_device(Ctx &c, const avism_params *p, const Level &L, const float *u1, const float *dv,
                        int fields_are_ext, const int8_t *smask_ext, const int32_t *marcap_ext,
                        const float *reqp, int32_t nreqp, CubesDev &cubes, const WidthProposal *wp) {
    const int ne = L.g.ne;
    const int64_t ne3 = (int64_t)ne * ne * ne;
    AV_CHECK(ne3 < (int64_t)INT32_MAX, AVISM_ERR_ARG, "ext grid larger than 2^31 cells");
    uint8_t *flags = c.get_t<uint8_t>(B_FLAGS, ne3);
    make_flags(c, p, L, u1, dv, fields_are_ext, smask_ext, marcap_ext, flags);
    c.mark("flags");

    VfArgs A;
    A.low1 = L.g.low1; A.low2 = L.g.low2; A.ne = ne; A.nx = L.g.nx; A.ext = fields_are_ext;
    A.flags = flags; A.marcap = marcap_ext; A.reqp = reqp; A.nreqp = nreqp; A.rmin_sub = p->rmin_sub;
    A.w0 = nullptr;
    if (wp && wp->w0) {
        A.w0 = wp->w0; A.nb = wp->nb; A.periodic_bins = wp->periodic; A.bin_origin = wp->origin;
        A.inv_bw = wp->inv_bw; A.box = wp->box; A.rx1 = L.rad_at(1); A.dx = L.g.dx;
        // the part of the proposed half-width swept at once (AVISM_TUNE_WFAC):
        // sweeping all of it cost 0.4 ms more at 512^3 than half of it
        const char *wf = getenv("AVISM_TUNE_WFAC");
        A.wfac = wf ? (float)atof(wf) : 0.5f;
    }

    // candidates in K,J,I order
    int32_t *pos = c.get_t<int32_t>(B_CAND_POS, ne3);
    int32_t *nsel_d = c.get_t<int32_t>(B_COUNTERS, 8);
    {
        cub::CountingInputIterator<int32_t> it(0);
        size_t tmp = 0;
        IsCand pred{flags};
        AV_CUDA(cub::DeviceSelect::If(nullptr, tmp, it, pos, nsel_d, (int)ne3, pred, c.stream));
        void *t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceSelect::If(t, tmp, it, pos, nsel_d, (int)ne3, pred, c.stream));
    }
    int32_t ncand = 0;
    AV_CUDA(cudaMemcpyAsync(&ncand, nsel_d, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    A.ncand = ncand;
    A.cand_pos = pos;
    if (ncand == 0) return 0;
    float *keys = c.get_t<float>(B_CAND_KEY, ncand);
    ++c.launches, k_cand_keys<<<grid_for(ncand, 256), 256, 0, c.stream>>>(A, dv, pos, ncand, keys);
    int32_t *indx = c.get_t<int32_t>(B_QUERY, ncand);
    c.mark("candidates");
    indexx_device(c, ncand, keys, indx);
    A.indx = indx;
    c.mark("indexx_div");

    uint8_t *st = c.get_t<uint8_t>(B_CUBE_ST, ncand);
    int32_t *wv = c.get_t<int32_t>(B_CUBE_W, ncand);
    uint8_t *cover = c.get_t<uint8_t>(B_COVER, ne3);
    unsigned long long *umin = c.get_t<unsigned long long>(B_PAINT, ne3);
    unsigned long long *amin = c.get_t<unsigned long long>(B_UMIN, ne3);
    AV_CUDA(cudaMemsetAsync(cover, 0, (size_t)ne3, c.stream));
    AV_CUDA(cudaMemsetAsync(umin, 0xff, (size_t)ne3 * 8, c.stream));
    AV_CUDA(cudaMemsetAsync(amin, 0xff, (size_t)ne3 * 8, c.stream));
    A.st = st; A.wv = wv; A.cover = cover; A.umin = umin; A.amin = amin;
    int32_t *open_a = c.get_t<int32_t>(B_LIST_A, ncand);
    int32_t *open_b = c.get_t<int32_t>(B_LIST_B, ncand);
    int32_t *acc = c.get_t<int32_t>(B_GE, ncand);
    int32_t *cnt = nsel_d;       // [0] open, [1] next open, [2] accepted
    uint32_t epoch = 0, window = 0;
    int32_t B = 1024;
    for (int32_t r0 = 0; r0 < ncand;) {
        const int32_t r1 = (int32_t)std::min<int64_t>((int64_t)r0 + B, ncand);
        window++;
        AV_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int32_t), c.stream));
        const int64_t nthr = (int64_t)(r1 - r0) * 32;
        ++c.launches, k_phase1<<<grid_for(nthr, 256), 256, 0, c.stream>>>(A, r0, r1, open_a, cnt);
        AV_CUDA(cudaGetLastError());
        int32_t h[4];
        AV_CUDA(cudaMemcpyAsync(h, cnt, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        int32_t nopen = h[0];
        const int32_t survivors = nopen;
        int32_t *cur = open_a, *nxt = open_b;
        int32_t nacc_window = 0;            // accepted of this window, kept in acc[0..)
        while (nopen > 0) {
            epoch++;
            AV_CUDA(cudaMemsetAsync(cnt + 1, 0, sizeof(int32_t), c.stream));
            AV_CUDA(cudaMemcpyAsync(cnt + 2, &nacc_window, sizeof(int32_t), cudaMemcpyHostToDevice, c.stream));
            ++c.launches, k_paint_umin<<<grid_for((int64_t)nopen * 32, 256), 256, 0, c.stream>>>(A, cur, nopen, epoch);
            ++c.launches, k_decide<<<grid_for(nopen, 256), 256, 0, c.stream>>>(A, cur, nopen, epoch, window, nxt, cnt + 1, acc, cnt + 2);
            AV_CUDA(cudaMemcpyAsync(h, cnt, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            const int32_t newly = h[2] - nacc_window;
            if (newly > 0)
                ++c.launches, k_paint_amin<<<grid_for((int64_t)newly * 32, 256), 256, 0, c.stream>>>(A, acc + nacc_window, newly, window);
            AV_CUDA(cudaGetLastError());
            nacc_window = h[2];
            nopen = h[1];
            std::swap(cur, nxt);
        }
        if (nacc_window > 0)
            ++c.launches, k_paint_cover<<<grid_for((int64_t)nacc_window * 32, 256), 256, 0, c.stream>>>(A, acc, nacc_window);
        r0 = r1;
        if (survivors * 4 < B) B = std::min(B * 2, 1 << 22);
        else if (survivors * 2 > B) B = std::max(B / 2, 256);
    }
    c.mark("grow_accept");
    // cube ids in rank order
    int32_t *ids = c.get_t<int32_t>(B_LE, ncand + 1);
    {
        cub::CountingInputIterator<int32_t> it(0);
        cub::TransformInputIterator<int32_t, IsAccepted, cub::CountingInputIterator<int32_t>> acc_it(it, IsAccepted{st});
        size_t tmp = 0;
        AV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, acc_it, ids, ncand + 1, c.stream));
        void *t = c.get(B_CUB_TMP, tmp);
        AV_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, acc_it, ids, ncand + 1, c.stream));
    }
    int32_t nvoid = 0;
    AV_CUDA(cudaMemcpyAsync(&nvoid, ids + ncand, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    int *err = (int *)(cnt + 4);
    AV_CUDA(cudaMemsetAsync(err, 0, sizeof(int), c.stream));
    ++c.launches, k_nvoid_check<<<grid_for(ncand, 256), 256, 0, c.stream>>>(st, ids, ncand, p->nvoid_max, err);
    int herr = 0;
    AV_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    AV_CHECK(herr == 0, AVISM_ERR_NVOID_MAX, "NVOID > NVOID_MAX!! Increase NVOID_MAX");
    const int32_t cap = std::max(nvoid, 1);
    cubes.cap = cap;
    cubes.i32 = (int32_t *)c.get(B_CUBES, (size_t)cap * 17 * 4);
    cubes.f32 = (float *)(cubes.i32 + (size_t)cap * 10);
    ++c.launches, k_write_cubes<<<grid_for(ncand, 256), 256, 0, c.stream>>>(A, ids, ncand, L.g.dx, L.rad_at(1), cubes.i32, cubes.f32, cap);
    AV_CUDA(cudaGetLastError());
    c.mark("cube_arrays");
    return nvoid;
}

}  // namespace avism
