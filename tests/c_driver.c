/* c_driver.c -- a caller of the C-ABI shaped like the Fortran driver: it reads
 * the level parameters and the particles from a file, runs one level through
 * avism_gpu_run_level with host arrays it owns (the COMMONDATA cube arrays and
 * the catalogue columns), and writes what the catalogue writer would read.
 * Used by tests/test_c_driver.py; built there with gcc -std=c99.
 *
 * input:  avism_params (raw struct), int64 n, then x y z vx vy vz m (n f32 each)
 * output: int32 nvoid, f32 meandens, int32 nvoid2, int32 nvoidt, f64 volt_clean,
 *         the 17 cube columns and the 15 catalogue columns, nvoid entries each,
 *         in the order of avism_cubes and avism_voids                          */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "avism_gpu.h"

static int rd(void *dst, size_t size, size_t count, FILE *f) { return fread(dst, size, count, f) == count; }

int main(int argc, char **argv) {
    avism_params p;
    int64_t n = 0;
    float *part[7];
    int32_t *ci[13];
    float *cf[19];
    avism_cubes cb;
    avism_voids vo;
    avism_gpu_ctx *ctx = NULL;
    int32_t nvoid = 0;
    float meandens = 0.0f;
    size_t cap, i;
    int st;
    FILE *f, *o;
    if (argc != 3) return 64;
    f = fopen(argv[1], "rb");
    if (!f || !rd(&p, sizeof p, 1, f) || !rd(&n, sizeof n, 1, f)) return 65;
    for (i = 0; i < 7; i++) {
        part[i] = (float *)malloc((size_t)n * sizeof(float));
        if (!part[i] || !rd(part[i], sizeof(float), (size_t)n, f)) return 65;
    }
    fclose(f);
    cap = (size_t)(p.nvoid_max > 0 ? p.nvoid_max : 1);
    for (i = 0; i < 13; i++) ci[i] = (int32_t *)calloc(cap, sizeof(int32_t));
    for (i = 0; i < 19; i++) cf[i] = (float *)calloc(cap, sizeof(float));
    cb.inicio_x = ci[0]; cb.final_x = ci[1]; cb.inicio_y = ci[2]; cb.final_y = ci[3];
    cb.inicio_z = ci[4]; cb.final_z = ci[5]; cb.icx = ci[6]; cb.icy = ci[7]; cb.icz = ci[8];
    cb.father = ci[9];
    cb.vol = cf[0]; cb.rini_x = cf[1]; cb.rfin_x = cf[2]; cb.rini_y = cf[3]; cb.rfin_y = cf[4];
    cb.rini_z = cf[5]; cb.rfin_z = cf[6];
    memset(&vo, 0, sizeof vo);
    vo.indice = ci[10]; vo.uvoid = ci[11]; vo.ncellv = ci[12];
    vo.volnew = cf[7]; vo.req = cf[8]; vo.xc = cf[9]; vo.yc = cf[10]; vo.zc = cf[11];
    vo.gxc = cf[12]; vo.gyc = cf[13]; vo.gzc = cf[14]; vo.eps = cf[15]; vo.ip = cf[16];
    vo.umean = cf[17]; vo.mtot = cf[18];
    vo.marca = NULL;
    st = avism_gpu_create(&ctx, 0);
    if (st != AVISM_OK) { fprintf(stderr, "avism_gpu_create: %d\n", st); return 2; }
    st = avism_gpu_run_level(ctx, &p, n, part[0], part[1], part[2], part[3], part[4], part[5], part[6], &cb,
                             &nvoid, &vo, &meandens);
    if (st != AVISM_OK) { fprintf(stderr, "avism_gpu_run_level: %d %s\n", st, avism_gpu_last_error(ctx)); return 3; }
    o = fopen(argv[2], "wb");
    if (!o) return 66;
    fwrite(&nvoid, sizeof nvoid, 1, o);
    fwrite(&meandens, sizeof meandens, 1, o);
    fwrite(&vo.nvoid2, sizeof vo.nvoid2, 1, o);
    fwrite(&vo.nvoidt, sizeof vo.nvoidt, 1, o);
    fwrite(&vo.volt_clean, sizeof vo.volt_clean, 1, o);
    for (i = 0; i < 10; i++) fwrite(ci[i], sizeof(int32_t), (size_t)nvoid, o);
    for (i = 0; i < 7; i++) fwrite(cf[i], sizeof(float), (size_t)nvoid, o);
    for (i = 10; i < 13; i++) fwrite(ci[i], sizeof(int32_t), (size_t)nvoid, o);
    for (i = 7; i < 19; i++) fwrite(cf[i], sizeof(float), (size_t)nvoid, o);
    fclose(o);
    avism_gpu_destroy(ctx);
    for (i = 0; i < 7; i++) free(part[i]);
    for (i = 0; i < 13; i++) free(ci[i]);
    for (i = 0; i < 19; i++) free(cf[i]);
    return 0;
}
