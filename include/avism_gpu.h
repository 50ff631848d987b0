/*
 * avism_gpu.h -- C-ABI of the B200 (sm_100a) AVISM void-finding library.
 *
 * The Fortran driver of AVISM (src/avism.f90) keeps reading config/voids.dat and
 * the particle files and keeps writing the catalogue; it calls these entry points
 * through an ISO_C_BINDING interface module in place of the Fortran routines named
 * in each comment.  All functions return an int status (AVISM_OK == 0) and never
 * exit or throw.  avism_gpu_last_error() returns the message of the last failure.
 *
 * Conventions (match the reference's arrays one to one):
 *   - 3D grids are Fortran column-major, x fastest.  "inner" grids are NX^3
 *     (indices 1..NX); "ext" grids cover LOW1..LOW2 per axis (periodic ghost
 *     shell of NPLUS cells, src/avism.f90:780-812), NE = LOW2-LOW1+1 per side.
 *   - index outputs keep the reference's values: 1-based particle/cube ids,
 *     grid indices in LOW1..LOW2.
 *   - every array argument may be a host pointer or a CUDA device pointer of the
 *     context's device; the library detects which and copies host arrays.
 *   - a context is bound to one GPU, is not re-entrant, and retains no caller
 *     pointer after a call returns.
 */
#ifndef AVISM_GPU_H
#define AVISM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
    AVISM_OK = 0,
    AVISM_ERR_ARG = 1,          /* invalid argument (size, null, range)          */
    AVISM_ERR_CUDA = 2,         /* CUDA runtime error                            */
    AVISM_ERR_OOM = 3,          /* device or host allocation failed             */
    AVISM_ERR_NVOID_MAX = 4,    /* 'NVOID > NVOID_MAX!! Increase NVOID_MAX'      */
    AVISM_ERR_OUT_OF_BOX = 5,   /* 'Particles outside the bounding box! Check L0!' */
    AVISM_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up            */
    AVISM_ERR_NO_DEVICE = 7,    /* no CUDA device / wrong architecture           */
    AVISM_ERR_UNSUPPORTED = 8,  /* option not implemented by this library        */
    AVISM_ERR_INTERNAL = 9,     /* internal consistency check failed             */
    AVISM_ERR_IO = 10           /* a file could not be opened, read or written,  */
                                /* or its records are not the expected ones      */
};

/* ---- parameters: POD mirror of config/voids.dat (src/avism.f90:173-254) -- */
typedef struct avism_params {
    int32_t nx;                 /* NCOX=NCOY=NCOZ: cells per side of this level   */
    int32_t periodic;           /* FLAG_PERIOD (0/1)                              */
    float   lado0;              /* LADO0, box side [cMpc]                         */
    float   ache;               /* h                                              */
    float   omega0;             /* Omega_m                                        */
    float   zeta;               /* redshift of the snapshot (ZETA)                */
    int32_t nvoid_max;          /* NVOID_MAX                                      */
    float   dens_thre;          /* DENS_THRE  (centres)                           */
    float   dens_thre2;         /* DENS_THRE2 (edges)                             */
    float   grad_thre;          /* GRAD_THRE                                      */
    float   div_thre;           /* DIV_THRE                                       */
    float   rmin;               /* RMIN [cMpc]                                    */
    float   rmin_sub;           /* RMIN_SUB [cMpc]                                */
    int32_t kneighbours;        /* KNEIGHBOURS                                    */
    int32_t flag_vel_interp;    /* 0 TSC, 1 SPH                                   */
    int32_t flag_dens_interp;   /* 0 TSC, 1 SPH                                   */
    int32_t level;              /* IR                                             */
    int32_t levmin;             /* LEVMIN                                         */
    int32_t learned;            /* 0: plain search, 1: learned proposal, 2: density estimate */
    int32_t kernel_mode;        /* KERNEL_MODE (src/particles.f90:9): 1 (or 0) M4 cubic
                                   spline, 2 Gaussian exp(-q^2)                    */
    int32_t no_velocities;      /* 1: FLAG_VEL_AVAILABLE = 0, the divergence is the
                                   linear-theory -Omega_m^0.6 a H (rho/rho_mean - 1)
                                   (src/avism.f90:1259-1306, 1647-1650); the
                                   velocity arrays may then be NULL               */
    int32_t flag_dens;          /* MASCLET input (FLAG_DATA = 0): FLAG_DENS, the density
                                   components: 0 DM + gas, 1 DM, 2 gas            */
    int32_t flag_div;           /* MASCLET input: FLAG_DIV, the divergence: 0 the
                                   minimum of gas and DM, 1 DM, 2 gas, -1 linear
                                   theory of the density (src/avism.f90:1633-1650) */
    int32_t reserved[3];
} avism_params;

/* ---- level geometry (MALLA + PBC extension, src/avism.f90:780-865) ------ */
typedef struct avism_grid {
    int32_t nx, nplus, low1, low2, ne;   /* ne = low2-low1+1                       */
    int32_t rad_lo, rad_hi;              /* index range held by the RADX array     */
    float   dx;                          /* DX = RADX(2)-RADX(1)                   */
    float   rx1;                         /* RADX(1)                                */
    float   lado;                        /* LADO = LADO0-LADO0/NX                  */
    float   lado0plus;                   /* LADO0PLUS (periodic extended box)      */
    float   rete, rote, hte;             /* scale factor, background density, H(z) */
} avism_grid;

/* ---- VOIDFIND outputs: the cube arrays of module COMMONDATA ------------- */
/* Each array holds at least nvoid_max entries; entry i is cube i+1.         */
typedef struct avism_cubes {
    int32_t *inicio_x, *final_x, *inicio_y, *final_y, *inicio_z, *final_z;
    int32_t *icx, *icy, *icz;
    int32_t *father;
    float   *vol;
    float   *rini_x, *rfin_x, *rini_y, *rfin_y, *rini_z, *rfin_z;
} avism_cubes;

/* ---- MERGE_VOID + post-processing outputs (src/avism.f90:1738-1973) ------ */
/* Arrays hold nvoid entries (one per cube, entry i is cube id i+1); marca is  */
/* the ext grid (NE^3 int32) and may be NULL.                                 */
typedef struct avism_voids {
    int32_t *indice;            /* cube ids by volume, largest first (INDICE)    */
    int32_t *uvoid;             /* -1 main void, 0 removed, >0 owner id          */
    int32_t *ncellv;            /* cells of each main void (inner grid)          */
    float   *volnew, *req;      /* volume [cMpc^3], equivalent radius            */
    float   *xc, *yc, *zc;      /* centre = cell of max divergence               */
    float   *gxc, *gyc, *gzc;   /* volume-weighted geometrical centre            */
    float   *eps, *ip;          /* ellipticity, inverse porosity                 */
    float   *umean, *mtot;      /* mean rho/rho_mean, mass [Msun]                */
    int32_t *marca;             /* ext grid of void ids (nullable)               */
    int32_t nvoid2;             /* voids after merging                           */
    int32_t nvoidt;             /* voids after post-processing (NVOIDT)          */
    double  volt_clean;         /* total comoving volume in voids                */
} avism_voids;

typedef struct avism_gpu_ctx avism_gpu_ctx;

/* ---- context ------------------------------------------------------------- */
int avism_gpu_create(avism_gpu_ctx **out, int device);
int avism_gpu_destroy(avism_gpu_ctx *ctx);
const char *avism_gpu_last_error(const avism_gpu_ctx *ctx);
/* Device-side time of the last call's stages (ms); returns the stage count and
 * writes at most n entries.  avism_gpu_stage_name(i) names stage i.            */
int avism_gpu_stage_times(const avism_gpu_ctx *ctx, double *ms, int n);
const char *avism_gpu_stage_name(const avism_gpu_ctx *ctx, int i);
/* Number of this library's kernels launched on the context so far.           */
int64_t avism_gpu_launches(const avism_gpu_ctx *ctx);

/* ---- a1: level grid, replaces MALLA (src/grid.f90:3-76) and the PBC block
 *      src/avism.f90:780-865.  radx receives RADX(rad_lo..rad_hi); pass NULL
 *      to query the geometry only.  Host only, no GPU needed.                 */
int avism_gpu_grid_setup(const avism_params *p, avism_grid *g, float *radx);

/* ---- a3/a4: k nearest neighbours, replaces knn_search (src/kdtree.f90:504-540)
 *      Neighbours of each query sorted by (squared distance, particle index);
 *      idx is 1-based, dist = sqrt(squared distance).  box_l > 0 selects the
 *      periodic minimum-image distance of src/kdtree.f90:1441-1465.           */
int avism_gpu_knn(avism_gpu_ctx *ctx, int64_t n, const float *x, const float *y,
                  const float *z, float box_l, int64_t nq, const float *qx,
                  const float *qy, const float *qz, int32_t k, int64_t *idx,
                  float *dist);

/* ---- a5-a10: particles to grid.  Replaces PPART_DENS, VVEL_INTERP_SPH_VW,
 *      FILL_H_ZEROS, H_DISTANCE, DDENS_INTERP_SPH (src/particles.f90:276-929)
 *      and DENS_INTERP_TSC / VEL_INTERP_TSC (src/particles.f90:16-271), called
 *      at src/avism.f90:1159-1245.  Inputs in the units READ_BINARY_PART_1
 *      leaves (src/reader.f90:441-457).  u_mass: mass per inner cell (the
 *      U1DMCO of DDENS/TSC before normalisation); u2..u4: velocity grids;
 *      hpart / part_dens: per particle, nullable.  smask: inner NX^3, nullable
 *      (all ones).                                                              */
int avism_gpu_particles_to_grid(avism_gpu_ctx *ctx, const avism_params *p, int64_t n,
                                const float *x, const float *y, const float *z,
                                const float *vx, const float *vy, const float *vz,
                                const float *m, const int8_t *smask,
                                float *u_mass, float *u2, float *u3, float *u4,
                                float *hpart, float *part_dens);

/* ---- a11-a13: density normalisation (src/avism.f90:1249-1250, 1384-1411),
 *      DIVER_UNIFORM (src/divergence.f90:2-50) and REAL_MAKE_PERIODIC
 *      (src/num.f90:89-133).  Outputs the ext grids U1CO and DIVERCO and the
 *      mean density MEANDENS [Msun/Mpc^3].                                      */
int avism_gpu_fields(avism_gpu_ctx *ctx, const avism_params *p, const float *u_mass,
                     const float *u2, const float *u3, const float *u4,
                     float *u1co_ext, float *diverco_ext, float *meandens);

/* ---- a14-a17: MARK_ALL + VOIDFIND (src/voidfinding.f90:13-713).  Inputs are
 *      the ext grids; smask_ext / marcap_ext are nullable (all ones / all -1,
 *      i.e. the first level of a particle run); reqp has one entry per parent
 *      void (nullable when marcap_ext is NULL).  Fills cubes[0..nvoid-1].       */
int avism_gpu_voidfind(avism_gpu_ctx *ctx, const avism_params *p, const float *u1co_ext,
                       const float *diverco_ext, const int8_t *smask_ext,
                       const int32_t *marcap_ext, const float *reqp,
                       avism_cubes *cubes, int32_t *nvoid);

/* ---- a14/a16: MARK_ALL (src/voidfinding.f90:13-55) and the six directional
 *      flag grids of VOIDFIND (src/voidfinding.f90:256-432) as one byte per ext
 *      cell: bit0 FLAGV, bit1 X1, bit2 X2, bit3 Y1, bit4 Y2, bit5 Z1, bit6 Z2,
 *      bit7 FLAG_SUB.  Inputs as avism_gpu_voidfind.                             */
int avism_gpu_flags(avism_gpu_ctx *ctx, const avism_params *p, const float *u1co_ext,
                    const float *diverco_ext, const int8_t *smask_ext,
                    const int32_t *marcap_ext, uint8_t *flags_ext);

/* ---- a18: INDEXX (src/num.f90:2-84): the Numerical Recipes index sort,
 *      reproducing its exact permutation of equal keys.  indx is 1-based.      */
int avism_gpu_indexx(avism_gpu_ctx *ctx, int32_t n, const float *arr, int32_t *indx);

/* ---- a18-a24: volume ordering, MERGE_VOID (src/voidfinding.f90:718-999) and
 *      the post-processing of src/avism.f90:1797-1973 (NCELL_MIN and RMIN
 *      filters, VOID_SHAPE, SIMPLE_CONNECTION_FAST, VOID_PERIODIC, global
 *      properties).  u1co_ext: the U1CO grid; meandens from avism_gpu_fields.   */
int avism_gpu_merge_post(avism_gpu_ctx *ctx, const avism_params *p, int32_t nvoid,
                         const avism_cubes *cubes, const float *u1co_ext,
                         float meandens, avism_voids *out);

/* ---- whole level on the device: particles in, catalogue out (a5-a24).
 *      Intermediate grids stay in HBM; only the catalogue arrays come back.    */
int avism_gpu_run_level(avism_gpu_ctx *ctx, const avism_params *p, int64_t n,
                        const float *x, const float *y, const float *z,
                        const float *vx, const float *vy, const float *vz,
                        const float *m, avism_cubes *cubes, int32_t *nvoid,
                        avism_voids *voids, float *meandens);

/* Counters of the warp kNN in the last particles_to_grid / run_level call,
 * collected while enabled (enable = 1 turns collection on for later calls, 0
 * off): out[0] queries, [1] radius attempts, [2] candidates scanned, [3]
 * candidates kept inside the radius, [4] queries that fell back to the shell
 * search, [5] queries (K <= 32) ranked by the exact counting select after the
 * bitonic order failed its check; and which of the reference's rare branches
 * the call took: [6] cells whose K-th distance is <= DX and that took the
 * ball_search fallback (src/particles.f90:868-878), [7] particles left with
 * h = 0 for FILL_H_ZEROS (src/particles.f90:398-430), [8] particles whose
 * DDENS NORM is 0 and whose mass goes to their own cell
 * (src/particles.f90:549-557).  No reference counterpart (instrumentation of
 * this library).                                                              */
int avism_gpu_knn_counters(avism_gpu_ctx *ctx, int enable, int64_t *out, int n);

/* ---- learned proposal.  No reference counterpart: AVISM has no learned part.
 *      A 12 -> 64 -> 64 -> 64 -> 2 ReLU MLP (BF16 weights, FP32 accumulation)
 *      predicts, per particle bin, the K-th neighbour distance of a query in the
 *      bin and the half-width of a cube grown from a centre in it, from 12
 *      multi-scale features of the binned particles (density, velocity
 *      divergence and density-gradient magnitude at 1, 2, 4 and 8 bins).  With
 *      params.learned = 1 the kNN starts from the predicted radius; the search
 *      grows or shrinks it until the neighbour list is verified, so results are
 *      identical to learned = 0 (learned = 2 starts from a radius estimated from
 *      the 27 surrounding bins' counts instead).
 *      Parameter vector: AVISM_PROPOSAL_NPARAM floats, mu[12], sigma[12],
 *      W1[64][12], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[2][64],
 *      b4[2], slack[2] (radius factor, half-width offset).                    */
#define AVISM_PROPOSAL_NPARAM 9308
/* weights used by learned = 1 calls on this context */
int avism_gpu_proposal_load(avism_gpu_ctx *ctx, const float *params, int32_t nparam);
/* features of every bin of the binning particles_to_grid uses (nb^3 rows of
 * 12, bin index x fastest); feat may be NULL to query nb and the bin width bw */
int avism_gpu_proposal_features(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x,
                                const float *y, const float *z, const float *vx, const float *vy,
                                const float *vz, const float *m, int64_t cap_rows, float *feat,
                                int32_t *nb, float *bw);
/* raw network outputs (nrows x 2) for explicit feature rows, on the tensor cores */
int avism_gpu_proposal_infer(avism_gpu_ctx *ctx, int64_t nrows, const float *feat, const float *params,
                             float *out);
/* loss and gradient of one batch (all ns samples; target / mask ns x 2) */
int avism_gpu_proposal_grad(avism_gpu_ctx *ctx, int64_t ns, const float *feat, const float *target,
                            const float *mask, const float *params, float *grad, float *loss);
/* Adam training on the GPU over random mini-batches; params in: initial, out:
 * trained; loss_curve (nullable) receives one loss per step                   */
int avism_gpu_proposal_train(avism_gpu_ctx *ctx, int64_t ns, const float *feat, const float *target,
                             const float *mask, int32_t steps, int32_t batch, float lr, uint32_t seed,
                             float *params, float *loss_curve);

/* ---- a26: voids-in-voids.  The next level's parent map: MARCAP(2NX)^3 =
 *      MARCA of the coarse cell and REQP = REQ of the main voids (replaces
 *      src/avism.f90:2123-2157), extended over the next level's ghost shell as
 *      MARCAP2 (src/avism.f90:1670-1674, INT_MAKE_PERIODIC src/num.f90:137-181).
 *      p describes the current level; marca_ext is its final MARCA (ext grid),
 *      uvoid / req its catalogue columns (nvoid entries).  marcap_next_ext
 *      receives the ext grid of the level with 2*nx cells per side, reqp_next
 *      nvoid radii (0 for voids that are not main voids).                      */
int avism_gpu_next_level(avism_gpu_ctx *ctx, const avism_params *p, int32_t nvoid, const int32_t *marca_ext,
                         const int32_t *uvoid, const float *req, int32_t *marcap_next_ext, float *reqp_next);
/* A level below the first, particles in and catalogue out (as run_level), with
 * the parent map and radii of avism_gpu_next_level: growth stays inside the
 * parent voids (src/voidfinding.f90:34-36, 487-529).  In the reference only
 * AMR input reaches this path (particle arrays are freed inside the level
 * loop, src/avism.f90:1613-1629); here the particles are passed again.       */
int avism_gpu_run_sublevel(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                           const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                           const int32_t *marcap_ext, const float *reqp, int32_t nreqp, avism_cubes *cubes,
                           int32_t *nvoid, avism_voids *voids, float *meandens);

/* ---- grid input (FLAG_DATA = 2): replaces src/avism.f90:1316-1362 for the
 *      grids of READ_BINARY_GRID (src/reader.f90:523-552).  u1g..u4g: the input
 *      grid, nhy^3 cells, column-major, as the reference holds it after
 *      reading: U1G = delta + 1 (rho / rho_B) and the velocities / UV.  The
 *      level's grid is params.nx = nhy * 2^level; level 0 takes the grids as
 *      they are, a level below 0 smooths them onto the coarser grid
 *      (SMOOTH_2, src/amr2uniform.f90:65-120), a level above 0 is the
 *      reference's 'LEVEL > 0 FOR BIN_GRID NOT IMPLEMENTED YET' stop
 *      (AVISM_ERR_UNSUPPORTED).  U1CO = U1GCO (no mean normalisation),
 *      DIVERCO = DIVER_UNIFORM of the velocities, MEANDENS the background
 *      density ROTE*UM/UL^3.  avism_gpu_grid_fields returns the ext grids (as
 *      avism_gpu_fields), avism_gpu_run_level_grid the level's catalogue.      */
int avism_gpu_grid_fields(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g, const float *u2g,
                          const float *u3g, const float *u4g, float *u1co_ext, float *diverco_ext, float *meandens);
int avism_gpu_run_level_grid(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                             const float *u2g, const float *u3g, const float *u4g, avism_cubes *cubes,
                             int32_t *nvoid, avism_voids *voids, float *meandens);

/* ---- MASCLET input (FLAG_DATA = 0) at levels <= 1: replaces the MASCLET branch
 *      of the level loop (src/avism.f90:980-1156) with the density and
 *      divergence choices of 1366-1405 and 1633-1650.  The dark-matter particles
 *      (every level's particles as READ_MASCLET fills them, src/reader.f90:86-405:
 *      positions [cMpc], velocities and masses in MASCLET units) go to the grid
 *      as in the particle path (SPH or TSC by flag_vel_interp / flag_dens_interp),
 *      U1DMCO = mass / (DX^3 a^3) / ROTE.  The gas grids u1g = 1 + delta and the
 *      velocities u2g..u4g (nhy^3, level 0) are copied at level 0 and averaged by
 *      SMOOTH_2 (src/amr2uniform.f90:65-120) below it.  U1CO = (U1DMCO + U1GCO,
 *      U1DMCO or U1GCO by flag_dens) * ROTE / its REAL*8 mean; DIVERCO by
 *      flag_div: the minimum of the DIVER_UNIFORM of the gas and of the DM
 *      velocities (0), DM (1), gas (2), or the linear theory of U1CO (-1).  The
 *      particle arrays may be NULL (n = 0) when neither flag uses the dark
 *      matter (flag_dens = 2 and flag_div = 2 or -1); u2g..u4g may be NULL when
 *      flag_div is 1 or -1.  At level 1 the gas fields come from the level-1
 *      patches amr (DIVER_FINA_GAS, src/divergence.f90:55-340, and VMESH,
 *      src/amr2uniform.f90:127-248, as the reference computes them: a cell
 *      under k patch cells takes their sum over k + 1, the children of a
 *      refined base cell that no patch covers take 0, the others their base
 *      cell's values) and the DM divergence is 0 (the reference computes
 *      DIVER_UNIFORM of the DM only at levels <= 0).  amr is ignored below
 *      level 1.  A patch whose 2-cell rim needs base-cell differences outside
 *      2..nhy-1, or whose cells fall outside the level grid, returns
 *      AVISM_ERR_ARG (the reference reads or writes outside its arrays there);
 *      so do sizes that disagree with the offsets.  Levels above 1 return AVISM_ERR_UNSUPPORTED: the reference's
 *      VMESH indexes its base-size refinement flags with coordinates beyond
 *      them there.
 *      avism_gpu_masclet_fields returns the ext grids (as avism_gpu_fields),
 *      avism_gpu_run_level_masclet the level's catalogue.                       */
/* the level-1 refinement patches of a MASCLET snapshot (host or device arrays):
 * sizes PATCHNX..Z, first base cells PATCHX..Z (1-based), corners PATCHRX..Z,
 * the start of each patch's cells in the cell arrays (offset[npatch] = total),
 * and the cells (x fastest): U11G = 1 + delta, U12G..U14G the velocities      */
typedef struct avism_patches {
    int32_t npatch;
    const int32_t *nx, *ny, *nz, *ix, *iy, *iz;
    const float *rx, *ry, *rz;
    const int64_t *offset;
    const float *u11g, *u12g, *u13g, *u14g;
} avism_patches;
int avism_gpu_masclet_fields(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                             const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                             int64_t n, const float *x, const float *y, const float *z, const float *vx,
                             const float *vy, const float *vz, const float *m, float *u1co_ext,
                             float *diverco_ext, float *meandens);
int avism_gpu_run_level_masclet(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                                const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                                int64_t n, const float *x, const float *y, const float *z, const float *vx,
                                const float *vy, const float *vz, const float *m, avism_cubes *cubes,
                                int32_t *nvoid, avism_voids *voids, float *meandens);
/* A MASCLET level below LEVMIN (voids-in-voids, src/avism.f90:1159-1973 at IR >
 * LEVMIN): the fields as avism_gpu_run_level_masclet, the void stage as
 * avism_gpu_run_sublevel with the parent map MARCAP2 (marcap_ext, the ext grid
 * of this level) and the parent radii REQP of avism_gpu_next_level.         */
int avism_gpu_run_sublevel_masclet(avism_gpu_ctx *ctx, const avism_params *p, int32_t nhy, const float *u1g,
                                   const float *u2g, const float *u3g, const float *u4g, const avism_patches *amr,
                                   int64_t n, const float *x, const float *y, const float *z, const float *vx,
                                   const float *vy, const float *vz, const float *m, const int32_t *marcap_ext,
                                   const float *reqp, int32_t nreqp, avism_cubes *cubes, int32_t *nvoid,
                                   avism_voids *voids, float *meandens);

/* ---- survey mode (FLAG_SURVEY = 1): replaces src/avism.f90:1420-1596.  The
 *      tracers (x..m, masses as weights; velocities nullable with
 *      no_velocities = 1) and the randoms (rx, ry, rz, weights rw, in the units
 *      READ_BINARY_PART_1 leaves: weights / UM) go to the grid with the survey
 *      mask smask (inner NX^3 int8: 0 unobserved; avism_io_read_mask).  The
 *      randoms use the same interpolation, SPH with their own kNN of
 *      KNEIGHBOURS2 = MIN(8*KNEIGHBOURS, 256) neighbours (H_DISTANCE,
 *      FILL_H_ZEROS, DDENS_INTERP_SPH) or TSC.  The contrast is D/(alpha R):
 *      alpha = DSUM/RSUM over the observed cells, the ratio floored at 1e-4 and
 *      clamped at 1000, divided by its mean over SMASK > 0; MEANDENS is the
 *      background density.  Without velocities the divergence is the linear
 *      theory one.  DSUM, RSUM and the mean ratio are REAL*8 sums per x-row,
 *      rows in j order, planes in k order (the reference's OpenMP reduction
 *      leaves the order open).
 *      avism_gpu_survey_fields returns the ext grids U1CO and DIVERCO (as
 *      avism_gpu_fields) and the randoms' mass grid u1rand (inner, nullable);
 *      avism_gpu_run_level_survey runs the whole level with the mask on the ext
 *      grid (0 on the ghost shell) for MARK_ALL and the growth.                  */
int avism_gpu_survey_fields(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                            const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                            int64_t nrand, const float *rx, const float *ry, const float *rz, const float *rw,
                            const int8_t *smask, float *u1co_ext, float *diverco_ext, float *meandens,
                            float *u1rand);
int avism_gpu_run_level_survey(avism_gpu_ctx *ctx, const avism_params *p, int64_t n, const float *x, const float *y,
                               const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                               int64_t nrand, const float *rx, const float *ry, const float *rz, const float *rw,
                               const int8_t *smask, avism_cubes *cubes, int32_t *nvoid, avism_voids *voids,
                               float *meandens);

/* ---- kNN without allocation.  No reference counterpart: an extra form of
 *      avism_gpu_knn (same neighbours, same distances, bit for bit) for callers
 *      that cannot allocate device memory -- a host whose device memory is
 *      wholly reserved by another allocator (a framework's caching allocator
 *      that has claimed the card), or one that cannot take the device-wide
 *      synchronisation cudaMalloc/cudaFree imply while its other streams run.
 *      It needs no context and allocates nothing: its scratch is one static
 *      device array of this library (under 40 MiB per device, present from
 *      module load), so n <= AVISM_KNN_NOALLOC_MAX_N; a larger n is rejected
 *      with AVISM_ERR_ARG and its message.
 *        - x..dist must be device pointers on `device` (AVISM_ERR_ARG otherwise).
 *        - stream is a cudaStream_t (NULL: the legacy default stream).  The work
 *          is queued on it and the call returns without waiting, except that
 *          box_l <= 0 waits once on the stream for the points' bounding cube.
 *        - the scratch is shared by every call on a device in this process:
 *          calls whose work overlaps in time (two streams, two host threads)
 *          race on it and corrupt each other's results.  Serialise them, e.g.
 *          on one stream.
 *        - nothing in the scratch needs to start at zero: each call writes
 *          every scratch word before reading it.
 *        - the first call on a device sets the device context up and looks the
 *          scratch address up (cudaGetSymbolAddress), which may load the module
 *          and allocate inside the CUDA runtime; make that first call before any
 *          stream capture.
 *        - the address is kept for the life of the process: do not call this
 *          entry point again after cudaDeviceReset() (or any teardown of the
 *          device's primary context), which invalidates it.
 *      errbuf (nullable, errlen bytes) receives the failure message, "" on
 *      success.                                                                 */
#define AVISM_KNN_NOALLOC_MAX_N 1048576
int avism_gpu_knn_noalloc(int device, void *stream, int64_t n, const float *x,
                          const float *y, const float *z, float box_l, int64_t nq,
                          const float *qx, const float *qy, const float *qz,
                          int32_t k, int64_t *idx, float *dist, char *errbuf,
                          int32_t errlen);

/* ---- on-disk formats at the boundary (host only: no context, no GPU) ------
 * Particle files of READ_BINARY_PART_1 (src/reader.f90:410-460): Fortran
 * sequential unformatted records with 4-byte length markers -- [int64 NPARTT,
 * REAL*4 ZETA], then x, y, z [cMpc], vx, vy, vz [km/s] and m [Msun], NPARTT
 * REAL*4 values each.  The values come back as stored; the reference divides
 * masses by UM and velocities by UV right after reading (src/reader.f90:455-458).
 * avism_io_read_particles fails with AVISM_ERR_ARG when NPARTT > capacity
 * (the reference's 'NPARTT > PARTIRED' stop) and AVISM_ERR_IO on any record
 * whose markers do not frame the expected length.                            */
int avism_io_particle_header(const char *path, int64_t *n, float *zeta);
int avism_io_read_particles(const char *path, int64_t capacity, float *x, float *y, float *z,
                            float *vx, float *vy, float *vz, float *m);
/* READ_BINARY_PART_2 (src/reader.f90:465-519): the same file without the three
 * velocity records (x, y, z, m); the driver then takes the no-velocity path
 * (avism_params.no_velocities = 1).  Header via avism_io_particle_header.
 * Records longer than a gfortran subrecord (2147483639 bytes) are read as the
 * chain of subrecords gfortran writes for them, in every reader here.        */
int avism_io_read_particles_novel(const char *path, int64_t capacity, float *x, float *y, float *z,
                                  float *m);
/* READ_BINARY_GRID (src/reader.f90:523-552): [REAL*4 ZETA], then U1G (density
 * contrast delta), U2G, U3G, U4G (velocities in km/s), nx^3 REAL*4 each,
 * column-major, as stored.  The reference then takes U1G + 1 and divides the
 * velocities by UV (src/reader.f90:546-550); avism_gpu_run_level_grid expects
 * those converted values.                                                     */
int avism_io_read_grid(const char *path, int32_t nx, float *zeta, float *u1, float *u2, float *u3, float *u4);
/* MASCLET snapshot (READ_MASCLET, src/reader.f90:86-405): the grid file (text:
 * IRR T NL MAP / ZETA / IR NDXYZ0 NST0, then per level IRR NPATCH NPART NPARTST,
 * a skipped line and four lines per patch), the gas file and the dark-matter
 * file (sequential unformatted).  avism_io_masclet_header gives the number of
 * levels, the level-0 particle count, NPARTT (all levels), ZETA and MAP (the
 * level-0 particle mass).  avism_io_read_masclet reads the level-0 gas grids
 * u1g..u4g (nhy^3; u1g = the stored delta + 1, as src/reader.f90:389-394) and
 * every level's DM particles into x..m (level 0 first, masses MAP; then each
 * level's particles with their stored masses); the AMR patches' grids are
 * skipped.  AVISM_ERR_ARG when NPARTT > capacity, AVISM_ERR_IO on a record
 * that is missing or of the wrong length.                                     */
int avism_io_masclet_header(const char *grid_path, int32_t *nl, int32_t *ndxyz0, int64_t *npartt, float *zeta,
                            float *map);
int avism_io_read_masclet(const char *grid_path, const char *gas_path, const char *dm_path, int32_t nhy,
                          float *u1g, float *u2g, float *u3g, float *u4g, int64_t capacity, float *x, float *y,
                          float *z, float *vx, float *vy, float *vz, float *m, int64_t *npartt);
/* The level-1 patches of a MASCLET snapshot, for avism_gpu_*_masclet at level
 * 1 (an avism_patches over these arrays).  avism_io_masclet_patches_size gives
 * NPATCH(1) and the patches' cells in total.  avism_io_read_masclet_patches
 * reads their geometry from the grid file (PATCHNX..NZ, PATCHX..Z, PATCHRX..RZ;
 * src/reader.f90:168-174), offset[npatch + 1] (the first cell of each patch in
 * the cell arrays, offset[0] = 0) and, from the gas file, U11G (the stored
 * delta + 1, src/reader.f90:393), U12G, U13G, U14G of each patch, column-major
 * at its own size (src/reader.f90:285-312).  AVISM_ERR_ARG when the patches or
 * cells exceed the capacities.                                                */
int avism_io_masclet_patches_size(const char *grid_path, int32_t *npatch, int64_t *ncells);
int avism_io_read_masclet_patches(const char *grid_path, const char *gas_path, int32_t nhy, int32_t capacity,
                                  int64_t capacity_cells, int32_t *nx, int32_t *ny, int32_t *nz, int32_t *ix,
                                  int32_t *iy, int32_t *iz, float *rx, float *ry, float *rz, int64_t *offset,
                                  float *u11g, float *u12g, float *u13g, float *u14g);
/* Survey mask (src/avism.f90:403-418): a stream file [int32 NMASK, REAL*4
 * MASKLOW, MASKUPPER, MASKSIDE, INTEGER*1 SMASK2(NMASK^3)].  NMASK must equal
 * ncox (the coarse grid, else AVISM_ERR_ARG as the reference's stop); the mask
 * is mapped onto the level's nx^3 cells by integer refinement NDOWN = nx/NMASK
 * (even, src/avism.f90:873-892), and positive values become 1
 * (src/avism.f90:898).  smask: inner nx^3 (int8); lims (nullable, 3 floats)
 * receives MASKLOW, MASKUPPER, MASKSIDE.                                      */
int avism_io_read_mask(const char *path, int32_t ncox, int32_t nx, int8_t *smask, float *lims);
/* Survey randoms (src/avism.f90:1425-1444): sequential unformatted [INTEGER*4
 * NRAND], then RANDX, RANDY, RANDZ [cMpc] and the weights MASSRAND [Msun], as
 * stored (the reference divides the weights by UM).                          */
int avism_io_randoms_header(const char *path, int32_t *nrand);
int avism_io_read_randoms(const char *path, int32_t capacity, float *x, float *y, float *z, float *w);
/* vel_cube.dat (src/avism.f90:1198-1202): the SPH velocity grids U2, U3, U4
 * (inner nx^3 each, column-major) written raw, STREAM access.                 */
int avism_io_write_vel_cube(const char *path, int32_t nx, const float *u2, const float *u3, const float *u4);

/* The voids / cubes catalogues and the map file of one iteration
 * (src/avism.f90:710-722 and 2026-2085), as tools/read_voids.py reads them.
 * avism_io_write_headers creates the voids file (and the cubes file when
 * cubes_path is not NULL) with their first lines: NLEV LEVMIN LEVMAX NCOX NCOY
 * NCOZ LADO0, and NLEV LEVMIN LEVMAX.
 * avism_io_append_level appends one level, as run_level / run_sublevel left it:
 *  - voids: IR NVOID NVOIDT NVOIDP VOLT_CLEAN/LADO0^3 MEANDENS, then for every
 *    main void in INDICE order: IND XC YC ZC GXC GYC GZC VOLM REQ UMEAN EPS IP
 *    INDP REQPP MTOT, with INDP = FATHER(IND) and REQPP its parent's REQ above
 *    LEVMIN (req_parent: the parent level's REQ by parent id), 0 at LEVMIN.
 *    The reference reads REQPP from its shared REQ array, which this level's
 *    loop may already have overwritten at that index; the parent's own value
 *    is written here;
 *  - cubes (cubes_path not NULL): IR NVOID NVOIDT, then every cube in INDICE
 *    order: IND UVOID INICIOX FINALX INICIOY FINALY INICIOZ FINALZ RINIXCO
 *    RFINXCO RINIYCO RFINYCO RINIZCO RFINZCO;
 *  - map (map_path not NULL): MARCA, U1CO - 1 and DIVERCO on the inner NX^3
 *    cells, column-major, raw (STREAM access), from voids->marca and the ext
 *    grids of avism_gpu_fields.
 * Reals are written with 9 (REAL*8: 17) significant digits.                   */
int avism_io_write_headers(const char *voids_path, const char *cubes_path, int32_t nlev, int32_t levmin,
                           int32_t levmax, int32_t ncox, int32_t ncoy, int32_t ncoz, float lado0);
int avism_io_append_level(const char *voids_path, const char *cubes_path, const char *map_path,
                          const avism_params *p, int32_t nvoid, int32_t nvoidp, float meandens,
                          const avism_cubes *cubes, const avism_voids *voids, const float *req_parent,
                          const float *u1co_ext, const float *diverco_ext);

#ifdef __cplusplus
}
#endif

#endif /* AVISM_GPU_H */
