// common.cuh -- shared definitions of the AVISM B200 library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/avism_gpu.h"

namespace avism {

// ---- status plumbing ------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define AV_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            throw ::avism::Error{AVISM_ERR_CUDA, std::string(#call) + ": " +           \
                                                     cudaGetErrorString(e_)};           \
    } while (0)

#define AV_CHECK(cond, code, text)                                                      \
    do {                                                                                \
        if (!(cond)) throw ::avism::Error{(code), (text)};                              \
    } while (0)

// ---- device buffer pool: named, grow-only --------------------------------
enum BufId : int {
    B_SP = 0,        // float4 binned particles (x, y, z, orig index)
    B_BIN_START,     // int64 bin offsets
    B_KEYS_A, B_KEYS_B, B_VALS_A, B_VALS_B,
    B_CUB_TMP,
    B_PX, B_PY, B_PZ, B_PVX, B_PVY, B_PVZ, B_PM,   // particle inputs (device copies)
    B_HPART, B_PDENS, B_NORM,
    B_UMASS, B_U2, B_U3, B_U4,                     // inner grids
    B_FIX0, B_FIX1, B_FIX2, B_FIX3,                // exact-sum limb counters (u64)
    B_U1CO, B_DIVER,                               // inner normalised density / divergence
    B_U1EXT, B_DVEXT,                              // ext grids (ABI outputs)
    B_FLAGS, B_SMASK, B_MARCAP,                    // ext byte flags, ext mask, ext parent ids
    B_REQP,
    B_CAND_POS, B_CAND_KEY, B_SORT_KEY, B_SORT_IDX, B_SEG_A, B_SEG_B, B_GE, B_LE, B_SCAN_A, B_SCAN_B,
    B_CUBE_W, B_CUBE_ST, B_COVER, B_UMIN, B_LIST_A, B_LIST_B, B_COUNTERS,
    B_CUBES,                                       // packed cube arrays
    B_MARCA, B_PAINT, B_LABMAP, B_LABEL_AUX, B_CCL,
    B_RED0, B_RED1, B_RED2,
    B_QUERY, B_RAD, B_BALL, B_SCAL, B_KNN_R0,
    B_SV, B_PDENS_S, B_HPART_S,                    // per-particle attributes in binned order
    B_SVW,                                         // (vx, vy, vz, m / PPART_DENS) in binned order
    B_PR_PARAMS, B_PR_PACKED, B_PR_PACKED_TMP,     // learned proposal: parameters, packed weights
    B_PR_TRAIN, B_PR_IDX, B_PR_GRAD, B_PR_ERR,     // training scratch
    B_PR_PYR0, B_PR_PYR1, B_PR_PYR2, B_PR_PYR3,    // feature pyramid
    B_PR_R0, B_PR_W0, B_PR_FEAT,                   // per-bin radius / half-width, feature rows
    B_KNN_STATS,                                   // warp kNN counters
    B_FLAGS_IN,                                    // flag bytes of the periodic inner grid
    B_PR_CNT, B_PR_BOX1, B_PR_BOX2, B_PR_BOX4,     // centred box counts of the bins
    B_PR_TMPA, B_PR_TMPB, B_PR_TMPC,
    B_PX4, B_PV4,                                  // packed (x, y, z, m), (vx, vy, vz, 0) in input order
    B_FSTART,                                      // int32 offsets of quarter-bin x cells
    B_PER_CELL, B_PER_LAB, B_PER_PAIRS,            // VOID_PERIODIC: centre cells, their labels, label-map updates
    B_LL_CELL, B_LL_CELL2, B_LL_KEY, B_LL_KEY2,    // cells of every void in K, J, I order (sorted by label)
    B_LL_CNT, B_LL_OFF, B_LL_SUM,                  // their counts, offsets and per-void REAL*4 sums
    B_U1RAND, B_SMASK_IN,                          // survey: the randoms' grid, the inner mask
    B_GRID_IN,                                     // grid input: the four input grids
    B_GAS1, B_GAS2, B_GAS3, B_GAS4, B_DIVER2,      // MASCLET input: the level's gas grids, the DM divergence
    B_AMR1, B_AMR2, B_AMR3, B_AMR4,                // MASCLET level 1: the patches' cells
    B_NUM
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    void *buf[B_NUM] = {};
    size_t cap[B_NUM] = {};
    std::string last_error;
    std::vector<double> stage_ms;
    int num_sms = 148;
    // host->device copies of the particle attributes (m, then vx, vy, vz) run on
    // a second stream after the positions' copies, so that binning's keys and
    // sort overlap them; ev_mass marks the end of the masses, ev_attr the end of
    // all; mass_ready() / attrs_ready() order the main stream after them
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_pos = nullptr, ev_mass = nullptr, ev_attr = nullptr;
    bool mass_pending = false, attr_pending = false;
    // binned velocities still to be gathered into sv (bin_particles leaves them
    // for sv_velocities() while their copy is in flight)
    struct SvPending {
        bool on = false;
        int64_t n = 0;
        const float4 *sp = nullptr;
        float4 *sv = nullptr;
        const float *vx = nullptr, *vy = nullptr, *vz = nullptr;
    } svp;
    // scratch pinned host memory for small readbacks
    void *hpin = nullptr;
    size_t hpin_cap = 0;
    // number of this library's kernels launched since the context was created
    int64_t launches = 0;
    // learned-proposal weights loaded (B_PR_PARAMS / B_PR_PACKED hold them)
    bool prop_loaded = false;
    // collect warp-kNN counters in particles_to_grid
    bool knn_stats = false;
    // branch counters of the last particles_to_grid with counters on: cells on
    // the ball fallback, FILL_H_ZEROS orphans, DDENS particles with NORM = 0
    int64_t path_counts[3] = {0, 0, 0};
    // named stage marks: events recorded on the stream, resolved by stage_close()
    std::vector<cudaEvent_t> marks;
    std::vector<std::string> mark_names;
    std::vector<std::string> stage_names;

    void stage_open() {
        for (cudaEvent_t e : marks) cudaEventDestroy(e);
        marks.clear();
        mark_names.clear();
        stage_ms.clear();
        stage_names.clear();
        mark("start");
    }
    void mark(const char *name) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        cudaEventRecord(e, stream);
        marks.push_back(e);
        mark_names.push_back(name);
    }
    void stage_close() {
        if (marks.empty()) return;
        cudaEventSynchronize(marks.back());
        for (size_t i = 1; i < marks.size(); i++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, marks[i - 1], marks[i]);
            stage_ms.push_back(ms);
            stage_names.push_back(mark_names[i]);
        }
        for (cudaEvent_t e : marks) cudaEventDestroy(e);
        marks.clear();
        mark_names.clear();
    }

    void *get(BufId id, size_t bytes) {
        if (bytes == 0) bytes = 16;
        if (cap[id] < bytes) {
            if (buf[id]) AV_CUDA(cudaFree(buf[id]));
            buf[id] = nullptr;
            cap[id] = 0;
            size_t want = bytes + bytes / 8;
            cudaError_t e = cudaMalloc(&buf[id], want);
            if (e != cudaSuccess) {
                cudaGetLastError();
                e = cudaMalloc(&buf[id], bytes);
                want = bytes;
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Error{AVISM_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed"};
            }
            cap[id] = want;
        }
        return buf[id];
    }
    template <class T> T *get_t(BufId id, size_t n) { return (T *)get(id, n * sizeof(T)); }

    void *host_pinned(size_t bytes) {
        if (hpin_cap < bytes) {
            if (hpin) cudaFreeHost(hpin);
            hpin = nullptr;
            AV_CUDA(cudaMallocHost(&hpin, bytes));
            hpin_cap = bytes;
        }
        return hpin;
    }
    void sync() { AV_CUDA(cudaStreamSynchronize(stream)); }
    void mass_ready() {
        if (!mass_pending) return;
        mass_pending = false;
        AV_CUDA(cudaStreamWaitEvent(stream, ev_mass, 0));
    }
    void attrs_ready() {
        mass_pending = false;
        if (!attr_pending) return;
        attr_pending = false;
        AV_CUDA(cudaStreamWaitEvent(stream, ev_attr, 0));
    }
    // the caller's host arrays must not be read after a failed call returns:
    // both streams are drained (their copies may still be queued)
    void drop_pending_copies() {
        mass_pending = attr_pending = false;
        svp = SvPending{};
        cudaStreamSynchronize(copy_stream);
        cudaStreamSynchronize(stream);
    }
};

// pointer classification: true if p is device (or managed) memory
bool is_device_ptr(const void *p);

// copies a caller array into a device buffer (no copy if it is already device memory)
const void *to_device(Ctx &c, BufId id, const void *src, size_t bytes);
// as to_device, the copy issued on stream st
const void *to_device_on(Ctx &c, cudaStream_t st, BufId id, const void *src, size_t bytes);
// copies a device result to the caller's array (device-to-device if it is device memory)
void from_device(Ctx &c, void *dst, const void *src_dev, size_t bytes);

// ---- level geometry (host) -------------------------------------------------
struct Level {
    avism_grid g;
    std::vector<float> rad;          // RADX(rad_lo..rad_hi)
    float rad_at(int i) const { return rad[(size_t)(i - g.rad_lo)]; }
};
int grid_setup_host(const avism_params *p, avism_grid *g, float *radx);
Level make_level(const avism_params *p);

// ---- launch helpers ----------------------------------------------------------
inline unsigned grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 0x7fffffffLL) g = 0x7fffffffLL;
    return (unsigned)g;
}

// ---- stage entry points (implemented across the .cu files) -----------------
struct BinnedParticles {
    int64_t n = 0;
    int nb = 1;                      // bins per axis
    float box = 0.f, bw = 0.f, inv_bw = 0.f, origin = 0.f;
    int periodic = 0;
    const float4 *sp = nullptr;      // binned particles (x, y, z, orig idx bits)
    const int64_t *start = nullptr;  // nb^3 + 1 offsets
    // offsets of quarter-bin cells along x (4 nb^3 + 1), or null: the kNN then
    // trims each row of bins to the query's reach at a quarter of a bin
    const int32_t *fstart = nullptr;
};

// sv (nullable): receives (vx, vy, vz, m) in binned order
// the velocities of bin_particles' split form gathered into sv (a no-op when
// none are pending); every reader of sv's velocities calls it first
void sv_velocities(Ctx &c);
BinnedParticles bin_particles(Ctx &c, int64_t n, const float *x, const float *y, const float *z,
                              float box, int periodic, float occupancy, const float *vx = nullptr,
                              const float *vy = nullptr, const float *vz = nullptr, const float *m = nullptr,
                              float4 *sv = nullptr, bool fine = false);

void knn_batch(Ctx &c, const BinnedParticles &bp, int64_t nq, const float *qx, const float *qy,
               const float *qz, int k, int64_t *idx_out, float *dist_out);

// per-bin proposed cube half-widths of the learned proposal, with the binning
struct WidthProposal {
    const float *w0 = nullptr;
    int nb = 0, periodic = 0;
    float origin = 0.f, inv_bw = 0.f, box = 0.f;
};

// particles -> grid (SPH/TSC).  All pointers are device pointers.
struct P2G {
    int64_t n;
    const float *x, *y, *z, *vx, *vy, *vz, *m;
    float *u_mass, *u2, *u3, *u4;    // inner NX^3
    float *hpart, *part_dens;        // per particle, input order; null when not wanted
    const int8_t *smask;             // inner NX^3 or null
    WidthProposal *wprop = nullptr;  // receives the half-width proposal (learned = 1), nullable
};
void particles_to_grid(Ctx &c, const avism_params *p, const Level &L, const P2G &a);

// normalisation + divergence (inner grids) and ext copies.
struct FieldsOut {
    float meandens;
};
FieldsOut fields_inner(Ctx &c, const avism_params *p, const Level &L, const float *u_mass,
                       const float *u2, const float *u3, const float *u4, float *u1co_in,
                       float *diver_in);
void ext_copy(Ctx &c, const Level &L, const float *inner, float *ext);
// the pieces of fields_inner: U1CO = U1DMCO*ROTE on the inner grid, the divergence
// (velocities or the linear theory), and survey mode's D/(alpha R) contrast
void rho_inner(Ctx &c, const Level &L, const float *u_mass, float *u1co_in);
void divergence_inner(Ctx &c, const avism_params *p, const Level &L, const float *u1co_in, const float *u2,
                      const float *u3, const float *u4, float *diver_in);
float survey_contrast(Ctx &c, const Level &L, const int8_t *smask, const float *u1rand, float *u1co_in);
// grid input: U1CO, DIVER and MEANDENS of the level from the input grids (NHY^3)
float grid_fields_inner(Ctx &c, const avism_params *p, const Level &L, int nhy, const float *u1g, const float *u2g,
                        const float *u3g, const float *u4g, float *u1co_in, float *diver_in);
// input grids given at NHY^3 on this level (copied, or SMOOTH_2-averaged below level 0)
void level_grids(Ctx &c, const Level &L, const avism_params *p, int nhy, int ngrids, const float *const *g,
                 float *const *co);
// MASCLET level-1 patches: geometry on the host, cells on the device
struct AmrPatches {
    int32_t npatch = 0;
    std::vector<int32_t> nx, ny, nz, ix, iy, iz;
    std::vector<float> rx, ry, rz;
    std::vector<int64_t> offset;
    const float *u11g = nullptr, *u12g = nullptr, *u13g = nullptr, *u14g = nullptr;
};
// MASCLET input at levels <= 1: U1CO and DIVERCO (inner) from the gas grids (at
// level 1 the patches amr) and the DM grids of particles_to_grid (u_mass and
// du* may be null when the flags do not use them); returns MEANDENS
float masclet_fields_inner(Ctx &c, const avism_params *p, const Level &L, int nhy, const float *const *gas,
                           const AmrPatches *amr, const float *u_mass, const float *du2, const float *du3,
                           const float *du4, float *u1co_in, float *diver_in);

// flags on the ext grid from inner (wrapped) fields, or from given ext fields.
void make_flags(Ctx &c, const avism_params *p, const Level &L, const float *u1, const float *dv,
                int fields_are_ext, const int8_t *smask_ext, const int32_t *marcap_ext,
                uint8_t *flags);

// learned proposal (proposal.cu)
void proposal_load(Ctx &c, const float *params_dev);
void proposal_features(Ctx &c, const avism_params *p, const P2G &a, float *feat_dev, int *nb_out, float *bw_out);
void proposal_infer(Ctx &c, int64_t ns, const float *feat, const float *prm_dev, float *out);
void proposal_grad(Ctx &c, int64_t ns, const float *feat, const float *tgt, const float *msk, const float *prm,
                   float *grad, float *loss);
void proposal_train(Ctx &c, int64_t ns, const float *feat, const float *tgt, const float *msk, int steps, int batch,
                    float lr, uint32_t seed, float *prm, float *loss_curve);
constexpr int PROPOSAL_NPARAM = 9308;

// exact Numerical Recipes INDEXX on device arrays (key f32, idx i32 1-based out)
void indexx_device(Ctx &c, int32_t n, const float *key_in, int32_t *indx_out);

// candidates + growth + acceptance; fills device cube arrays (packed), returns nvoid
struct CubesDev {
    int32_t *i32;   // 10 arrays of cap entries: inicio_x..final_z, icx, icy, icz, father
    float *f32;     // 7 arrays: vol, rini_x..rfin_z
    int32_t cap;
};
int32_t voidfind_device(Ctx &c, const avism_params *p, const Level &L, const float *u1,
                        const float *dv, int fields_are_ext, const int8_t *smask_ext,
                        const int32_t *marcap_ext, const float *reqp, int32_t nreqp,
                        CubesDev &cubes, const WidthProposal *wp = nullptr);

// merge + post-processing; cubes in host memory (copied), outputs host arrays
void merge_post(Ctx &c, const avism_params *p, const Level &L, int32_t nvoid,
                const avism_cubes *cubes_host, const float *u1co_inner_dev, float meandens,
                avism_voids *out, int32_t *marca_ext_out);

}  // namespace avism
