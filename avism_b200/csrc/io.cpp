// io.cpp -- the on-disk formats at the library's boundary (host only).
//
//  * particle files of READ_BINARY_PART_1 (src/reader.f90:410-460): Fortran
//    sequential unformatted records, each framed by 4-byte length markers:
//    [int64 NPARTT, REAL*4 ZETA], then x, y, z, vx, vy, vz, m (NPARTT REAL*4
//    each), as written by the reference's input tools;
//  * the voids / cubes catalogues and the map of one iteration
//    (src/avism.f90:710-722 headers, 2026-2085 per level): whitespace-separated
//    text lines with the reference's columns, and the map as raw STREAM arrays
//    (MARCA int32, delta = U1CO - 1 and DIVERCO REAL*4, inner NX^3 each,
//    column-major).  Reals are printed with enough digits to read back the same
//    REAL*4 (or REAL*8) value; the reference's list-directed spacing is not kept,
//    readers split on whitespace.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/avism_gpu.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() { if (f) std::fclose(f); }
};

// one record: 4-byte marker, payload, the same marker
bool read_record(FILE *f, void *dst, uint32_t bytes) {
    uint32_t a = 0, b = 0;
    if (std::fread(&a, 4, 1, f) != 1 || a != bytes) return false;
    if (bytes && std::fread(dst, 1, bytes, f) != bytes) return false;
    return std::fread(&b, 4, 1, f) == 1 && b == bytes;
}

// 9 significant digits read back as the same REAL*4
void put_f(FILE *f, float v) { std::fprintf(f, " %.9g", (double)v); }

}  // namespace

extern "C" {

int avism_io_particle_header(const char *path, int64_t *n, float *zeta) {
    if (!path || !n || !zeta) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    unsigned char rec[12];
    if (!read_record(in.f, rec, 12)) return AVISM_ERR_IO;
    std::memcpy(n, rec, 8);
    std::memcpy(zeta, rec + 8, 4);
    return *n >= 0 ? AVISM_OK : AVISM_ERR_IO;
}

int avism_io_read_particles(const char *path, int64_t capacity, float *x, float *y, float *z, float *vx,
                            float *vy, float *vz, float *m) {
    float *dst[7] = {x, y, z, vx, vy, vz, m};
    for (float *d : dst)
        if (!d) return AVISM_ERR_ARG;
    if (!path) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    unsigned char rec[12];
    if (!read_record(in.f, rec, 12)) return AVISM_ERR_IO;
    int64_t n;
    std::memcpy(&n, rec, 8);
    if (n < 0) return AVISM_ERR_IO;
    if (n > capacity) return AVISM_ERR_ARG;                              // 'ERROR: NPARTT > PARTIRED'
    if ((uint64_t)n * 4 > 0xffffffffull) return AVISM_ERR_UNSUPPORTED;   // would need a split record
    for (float *d : dst)
        if (!read_record(in.f, d, (uint32_t)(n * 4))) return AVISM_ERR_IO;
    return AVISM_OK;
}

int avism_io_write_headers(const char *voids_path, const char *cubes_path, int32_t nlev, int32_t levmin,
                           int32_t levmax, int32_t ncox, int32_t ncoy, int32_t ncoz, float lado0) {
    if (!voids_path) return AVISM_ERR_ARG;
    {
        File v(voids_path, "w");
        if (!v.f) return AVISM_ERR_IO;
        std::fprintf(v.f, " %d %d %d %d %d %d", nlev, levmin, levmax, ncox, ncoy, ncoz);
        put_f(v.f, lado0);
        std::fputc('\n', v.f);
        if (std::ferror(v.f)) return AVISM_ERR_IO;
    }
    if (cubes_path) {
        File c(cubes_path, "w");
        if (!c.f) return AVISM_ERR_IO;
        std::fprintf(c.f, " %d %d %d\n", nlev, levmin, levmax);
        if (std::ferror(c.f)) return AVISM_ERR_IO;
    }
    return AVISM_OK;
}

int avism_io_append_level(const char *voids_path, const char *cubes_path, const char *map_path,
                          const avism_params *p, int32_t nvoid, int32_t nvoidp, float meandens,
                          const avism_cubes *cubes, const avism_voids *voids, const float *req_parent,
                          const float *u1co_ext, const float *diverco_ext) {
    if (!voids_path || !p || !voids || nvoid < 0) return AVISM_ERR_ARG;
    if (nvoid > 0 && (!voids->indice || !voids->uvoid || !voids->xc || !voids->yc || !voids->zc || !voids->gxc ||
                      !voids->gyc || !voids->gzc || !voids->volnew || !voids->req || !voids->umean ||
                      !voids->eps || !voids->ip || !voids->mtot))
        return AVISM_ERR_ARG;
    for (int32_t iv = 0; iv < nvoid; iv++)
        if (voids->indice[iv] < 1 || voids->indice[iv] > nvoid) return AVISM_ERR_ARG;
    const bool sub = p->level > p->levmin;
    if (sub && nvoid > 0 && (!cubes || !cubes->father)) return AVISM_ERR_ARG;
    if (cubes_path && nvoid > 0 &&
        (!cubes || !cubes->inicio_x || !cubes->final_x || !cubes->inicio_y || !cubes->final_y || !cubes->inicio_z ||
         !cubes->final_z || !cubes->rini_x || !cubes->rfin_x || !cubes->rini_y || !cubes->rfin_y || !cubes->rini_z ||
         !cubes->rfin_z))
        return AVISM_ERR_ARG;
    if (map_path && (!voids->marca || !u1co_ext || !diverco_ext)) return AVISM_ERR_ARG;
    {
        File v(voids_path, "a");
        if (!v.f) return AVISM_ERR_IO;
        // IR, NVOID, NVOIDT, NVOIDP, VOLT_CLEAN/(LADO0**3), MEANDENS
        const float l3 = (p->lado0 * p->lado0) * p->lado0;
        std::fprintf(v.f, " %d %d %d %d %.17g", p->level, nvoid, voids->nvoidt, nvoidp,
                     voids->volt_clean / (double)l3);
        put_f(v.f, meandens);
        std::fputc('\n', v.f);
        for (int32_t iv = 0; iv < nvoid; iv++) {
            const int32_t i = voids->indice[iv] - 1;
            if (voids->uvoid[i] != -1) continue;              // main voids only
            int32_t indp = 0;
            float reqpp = 0.0f;
            if (sub) {
                indp = cubes->father[i];
                if (req_parent && indp > 0) reqpp = req_parent[indp - 1];
            }
            std::fprintf(v.f, " %d", i + 1);
            const float cols[] = {voids->xc[i], voids->yc[i], voids->zc[i], voids->gxc[i], voids->gyc[i],
                                  voids->gzc[i], voids->volnew[i], voids->req[i], voids->umean[i], voids->eps[i],
                                  voids->ip[i]};
            for (float c : cols) put_f(v.f, c);
            std::fprintf(v.f, " %d", indp);
            put_f(v.f, reqpp);
            put_f(v.f, voids->mtot[i]);
            std::fputc('\n', v.f);
        }
        if (std::ferror(v.f)) return AVISM_ERR_IO;
    }
    if (cubes_path) {
        File c(cubes_path, "a");
        if (!c.f) return AVISM_ERR_IO;
        std::fprintf(c.f, " %d %d %d\n", p->level, nvoid, voids->nvoidt);
        for (int32_t iv = 0; iv < nvoid; iv++) {
            const int32_t i = voids->indice[iv] - 1;
            std::fprintf(c.f, " %d %d %d %d %d %d %d %d", i + 1, voids->uvoid[i], cubes->inicio_x[i],
                         cubes->final_x[i], cubes->inicio_y[i], cubes->final_y[i], cubes->inicio_z[i],
                         cubes->final_z[i]);
            const float cols[] = {cubes->rini_x[i], cubes->rfin_x[i], cubes->rini_y[i], cubes->rfin_y[i],
                                  cubes->rini_z[i], cubes->rfin_z[i]};
            for (float col : cols) put_f(c.f, col);
            std::fputc('\n', c.f);
        }
        if (std::ferror(c.f)) return AVISM_ERR_IO;
    }
    if (map_path) {
        avism_grid g;
        const int st = avism_gpu_grid_setup(p, &g, nullptr);
        if (st != AVISM_OK) return st;
        const size_t nx = (size_t)g.nx, ne = (size_t)g.ne, o = (size_t)(1 - g.low1);  // inner i -> ext i-1+o
        File mf(map_path, "ab");
        if (!mf.f) return AVISM_ERR_IO;
        std::vector<int32_t> mi(nx);
        std::vector<float> row(nx);
        for (int pass = 0; pass < 3; pass++)
            for (size_t k = 0; k < nx; k++)
                for (size_t j = 0; j < nx; j++) {
                    const size_t base = o + ne * ((o + j) + ne * (o + k));
                    if (pass == 0) {
                        for (size_t i = 0; i < nx; i++) mi[i] = voids->marca[base + i];
                        if (std::fwrite(mi.data(), 4, nx, mf.f) != nx) return AVISM_ERR_IO;
                    } else {
                        for (size_t i = 0; i < nx; i++)
                            row[i] = pass == 1 ? -1.0f + u1co_ext[base + i] : diverco_ext[base + i];
                        if (std::fwrite(row.data(), 4, nx, mf.f) != nx) return AVISM_ERR_IO;
                    }
                }
    }
    return AVISM_OK;
}

}  // extern "C"
