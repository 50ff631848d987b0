/*
 * avism_oracle.h -- CPU oracle for the AVISM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * Fortran routines (oscarmonllor99/AVISM, the src/ directory), used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product (avism_b200/, libavism_gpu.so) never links, loads or calls it.
 *
 * Parity status: parity unpinned by the reference.  The reference ships no
 * golden vectors and cannot be compiled here (no Fortran compiler), so this
 * oracle is pinned by analytic known-answer cases (tests/test_oracle_pins.py),
 * brute-force kNN and an independent INDEXX restatement rather than by
 * reference outputs.
 *
 * Floating point: compiled with -ffp-contract=off; every f32/f64 operation and
 * promotion point follows the Fortran expression it restates (cited per function).
 * Where the reference's result depends on thread timing or traversal order the
 * oracle fixes a rule, stated at the function:
 *   - kNN / ball results are ordered by (squared distance, particle index);
 *   - FP64 scatter sums are accumulated in particle order.
 */
#ifndef AVISM_ORACLE_H
#define AVISM_ORACLE_H

#include <stdint.h>
#include "../include/avism_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* a1: grid geometry (src/grid.f90:3-76, src/avism.f90:780-865) and the
 * cosmology at ZETA (src/avism.f90:476-488, 609-616). */
int orc_grid_setup(const avism_params *p, avism_grid *g, float *radx);

/* a2-a4: k-d tree kNN and ball search (src/kdtree.f90). */
typedef struct orc_kdtree orc_kdtree;
orc_kdtree *orc_kd_build(int64_t n, const float *x, const float *y, const float *z, float box_l);
void orc_kd_free(orc_kdtree *t);
/* k nearest of one query: idx 0-based, d2 squared distances, ascending (d2, idx) */
void orc_kd_knn(const orc_kdtree *t, float qx, float qy, float qz, int k, int64_t *idx, float *d2);
/* all points with d2 <= r*r; returns the count; outputs sorted by (d2, idx).
 * *cap / *idx / *d2 are a growable buffer owned by the caller (realloc'd). */
int64_t orc_kd_ball(const orc_kdtree *t, float qx, float qy, float qz, float r,
                    int64_t **idx, float **d2, int64_t *cap);
/* batch kNN for tests: idx 1-based, dist = sqrt(d2) */
int orc_knn(int64_t n, const float *x, const float *y, const float *z, float box_l,
            int64_t nq, const float *qx, const float *qy, const float *qz, int k,
            int64_t *idx, float *dist);

/* a5-a10: particles to grid (src/particles.f90).  Grids inner NX^3. */
int orc_ppart_dens(const orc_kdtree *t, int64_t n, const float *x, const float *y,
                   const float *z, const float *m, int k, float *part_dens);
int orc_vvel_interp_sph_vw(const orc_kdtree *t, const avism_grid *g, const float *radx,
                           int k, int64_t n, const float *m, const float *vx,
                           const float *vy, const float *vz, const float *part_dens,
                           const int8_t *smask, int gauss, float *hpart, float *u2, float *u3,
                           float *u4);
int orc_h_distance(const orc_kdtree *t, const avism_grid *g, const float *radx, int k,
                   int64_t n, const int8_t *smask, float *hpart);
int orc_fill_h_zeros(const orc_kdtree *t, int64_t n, const float *x, const float *y,
                     const float *z, int k, float *hpart);
int orc_ddens_interp_sph(const avism_grid *g, const float *radx, int64_t n,
                         const float *x, const float *y, const float *z,
                         const float *hpart, const float *m, int gauss, float *u);
int orc_dens_interp_tsc(const avism_grid *g, const float *radx, int periodic, int64_t n,
                        const float *x, const float *y, const float *z, const float *m,
                        float *u);
int orc_vel_interp_tsc(const avism_grid *g, const float *radx, int periodic, int64_t n,
                       const float *x, const float *y, const float *z, const float *vx,
                       const float *vy, const float *vz, float *u2, float *u3, float *u4);
/* whole particle->grid block of src/avism.f90:1159-1245 */
int orc_particles_to_grid(const avism_params *p, int64_t n, const float *x, const float *y,
                          const float *z, const float *vx, const float *vy, const float *vz,
                          const float *m, const int8_t *smask, float *u_mass, float *u2,
                          float *u3, float *u4, float *hpart, float *part_dens);

/* a11-a13: normalisation, DIVER_UNIFORM, periodic ghost fill. */
int orc_diver_uniform(int nx, float dx, const float *v2, const float *v3, const float *v4,
                      int periodic, float *diver);
int orc_fields(const avism_params *p, const float *u_mass, const float *u2, const float *u3,
               const float *u4, float *u1co_ext, float *diverco_ext, float *meandens);

/* a14-a17: MARK_ALL + VOIDFIND.  flags_ext (nullable) receives the packed
 * per-cell byte: bit0 FLAGV, bit1 X1, bit2 X2, bit3 Y1, bit4 Y2, bit5 Z1,
 * bit6 Z2, bit7 FLAG_SUB. */
int orc_voidfind(const avism_params *p, const float *u1co_ext, const float *diverco_ext,
                 const int8_t *smask_ext, const int32_t *marcap_ext, const float *reqp,
                 avism_cubes *cubes, int32_t *nvoid, uint8_t *flags_ext,
                 int32_t *ncand, int32_t *cand_order /* nullable: ext linear idx, desc div */);

/* a18: Numerical Recipes indexx as in src/num.f90:2-84 (indx 1-based). */
int orc_indexx(int32_t n, const float *arr, int32_t *indx);

/* a18-a24: INDEXX by volume, MERGE_VOID and the post-processing. */
int orc_merge_post(const avism_params *p, int32_t nvoid, const avism_cubes *cubes,
                   const float *u1co_ext, float meandens, avism_voids *out);

/* the full level: particles -> catalogue (a5-a24) */
int orc_run_level(const avism_params *p, int64_t n, const float *x, const float *y,
                  const float *z, const float *vx, const float *vy, const float *vz,
                  const float *m, avism_cubes *cubes, int32_t *nvoid, avism_voids *voids,
                  float *meandens, float *u1co_ext, float *diverco_ext);

/* survey mode (src/avism.f90:1420-1596): the D/(alpha R) contrast of the
 * inner U1CO (rho/rho_B * ROTE on entry) from the randoms' grid u1rand, and
 * the whole fields stage with tracers, randoms and the mask */
int orc_survey_contrast(const avism_params *p, const avism_grid *g, const int8_t *smask, const float *u1rand,
                        float *u1, float *meandens);
int orc_survey_fields(const avism_params *p, int64_t n, const float *x, const float *y, const float *z,
                      const float *vx, const float *vy, const float *vz, const float *m, int64_t nrand,
                      const float *rx, const float *ry, const float *rz, const float *rw, const int8_t *smask,
                      float *u1co_ext, float *diverco_ext, float *meandens, float *u1rand_out);

/* grid input (FLAG_DATA = 2, src/avism.f90:1316-1362; SMOOTH_2 below level 0) */
int orc_grid_fields(const avism_params *p, int32_t nhy, const float *u1g, const float *u2g, const float *u3g,
                    const float *u4g, float *u1co_ext, float *diverco_ext, float *meandens);
/* the level's copies (level 0) or SMOOTH_2 averages (below it) of NHY^3 grids;
 * co[q] must hold zeros */
void orc_level_grids(const avism_params *p, int32_t nhy, int ngrids, const float *const *in, float *const *co);

/* MASCLET input (FLAG_DATA = 0) at levels <= 0 (src/avism.f90:980-1156,
 * 1366-1405, 1633-1650): DM particles and gas grids, combined by FLAG_DENS /
 * FLAG_DIV; the particle arrays may be NULL when the flags do not use them;
 * level 1 takes the gas fields from the level-1 patches (VMESH, DIVER_FINA_GAS) */
int orc_masclet_fields(const avism_params *p, int32_t nhy, const float *u1g, const float *u2g, const float *u3g,
                       const float *u4g, const avism_patches *amr, int64_t n, const float *x, const float *y,
                       const float *z, const float *vx, const float *vy, const float *vz, const float *m,
                       float *u1co_ext, float *diverco_ext, float *meandens);

#ifdef __cplusplus
}
#endif
/* cells on the ball fallback, FILL_H_ZEROS orphans and DDENS NORM = 0
 * particles of the last orc_particles_to_grid call */
void orc_path_counts(int64_t *out);

#endif
