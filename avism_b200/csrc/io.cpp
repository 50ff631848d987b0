// io.cpp -- the on-disk formats at the library's boundary (host only).
//
//  * particle files of READ_BINARY_PART_1 (src/reader.f90:410-460): Fortran
//    sequential unformatted records, each framed by 4-byte length markers:
//    [int64 NPARTT, REAL*4 ZETA], then x, y, z, vx, vy, vz, m (NPARTT REAL*4
//    each), as written by the reference's input tools; READ_BINARY_PART_2
//    (src/reader.f90:465-519) without the three velocity records;
//  * grid files of READ_BINARY_GRID (src/reader.f90:523-552): [REAL*4 ZETA],
//    then the density contrast and the three velocity grids;
//  * survey inputs: the stream mask file (src/avism.f90:403-418, mapped onto
//    the level's grid as src/avism.f90:873-901) and the randoms file
//    (src/avism.f90:1425-1444);
//  * MASCLET snapshots (READ_MASCLET, src/reader.f90:86-405): the grid file
//    (text), the gas file and the dark-matter file (sequential unformatted);
//    the level-0 gas grids and every level's particles are read;
//  * the vel_cube.dat side dump of the SPH velocity grids
//    (src/avism.f90:1198-1202, STREAM access);
//  * the voids / cubes catalogues and the map of one iteration
//    (src/avism.f90:710-722 headers, 2026-2085 per level): whitespace-separated
//    text lines with the reference's columns, and the map as raw STREAM arrays
//    (MARCA int32, delta = U1CO - 1 and DIVERCO REAL*4, inner NX^3 each,
//    column-major).  Reals are printed with enough digits to read back the same
//    REAL*4 (or REAL*8) value; the reference's list-directed spacing is not kept,
//    readers split on whitespace.
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/avism_gpu.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(path ? std::fopen(path, mode) : nullptr) {}
    ~File() { if (f) std::fclose(f); }
};

// Largest payload of one gfortran subrecord with 4-byte markers.  A longer
// record is written as a chain of subrecords: each carries its own leading and
// trailing length markers, and a negative leading marker says that another
// subrecord of the same record follows (the trailing marker of a continuation
// is negative too; only its magnitude is checked here).
constexpr uint64_t MAX_SUBRECORD = 2147483639ull;

// one logical record of exactly `bytes` payload bytes, as one record or a chain
// of subrecords
bool read_record(FILE *f, void *dst, uint64_t bytes) {
    unsigned char *out = static_cast<unsigned char *>(dst);
    uint64_t got = 0;
    for (;;) {
        int32_t head = 0, tail = 0;
        if (std::fread(&head, 4, 1, f) != 1 || head == INT32_MIN) return false;
        const uint64_t len = (uint64_t)(head < 0 ? -(int64_t)head : head);
        if (got + len > bytes) return false;
        if (len && std::fread(out + got, 1, len, f) != len) return false;
        if (std::fread(&tail, 4, 1, f) != 1 || tail == INT32_MIN) return false;
        if ((uint64_t)(tail < 0 ? -(int64_t)tail : tail) != len) return false;
        got += len;
        if (head >= 0) break;
    }
    return got == bytes;
}

// the leading record [int64 NPARTT, REAL*4 ZETA] of the particle files
bool read_particle_head(FILE *f, int64_t *n, float *zeta) {
    unsigned char rec[12];
    if (!read_record(f, rec, 12)) return false;
    std::memcpy(n, rec, 8);
    std::memcpy(zeta, rec + 8, 4);
    return *n >= 0;
}

// 9 significant digits read back as the same REAL*4
void put_f(FILE *f, float v) { std::fprintf(f, " %.9g", (double)v); }

// one record of any length (or chain of subrecords), skipped; its payload
// length in *total when given
bool skip_record(FILE *f, uint64_t *total = nullptr) {
    uint64_t sum = 0;
    for (;;) {
        int32_t head = 0, tail = 0;
        if (std::fread(&head, 4, 1, f) != 1 || head == INT32_MIN) return false;
        const int64_t len = head < 0 ? -(int64_t)head : head;
        if (std::fseek(f, (long)len, SEEK_CUR) != 0) return false;
        if (std::fread(&tail, 4, 1, f) != 1 || tail == INT32_MIN) return false;
        if ((tail < 0 ? -(int64_t)tail : tail) != len) return false;
        sum += (uint64_t)len;
        if (head >= 0) {
            if (total) *total = sum;
            return true;
        }
    }
}

// list-directed input of a text file: the next `count` numbers (blank- or
// comma-separated), starting on a new line and going on over the following
// lines if one holds fewer (a READ(u,*) statement); count 0 skips one line
bool read_values(FILE *f, int count, double *out) {
    char line[4096];
    int got = 0;
    do {
        if (!std::fgets(line, sizeof line, f)) return false;
        char *s = line;
        while (got < count) {
            while (*s == ' ' || *s == '\t' || *s == ',' || *s == '\r' || *s == '\n') s++;
            if (!*s) break;
            char *e = nullptr;
            const double v = std::strtod(s, &e);
            if (e == s) return false;
            out[got++] = v;
            s = e;
        }
    } while (got < count);
    return true;
}

// the MASCLET grid file (src/reader.f90:153-175): IRR, T, NL, MAP / ZETA /
// IR, NDXYZ0, NST0, then per level IRR, NPATCH, NPART, NPARTST, a skipped line
// and four lines per patch (sizes, cell offsets, corner, parent)
struct MascletGrid {
    int nl = 0, ndxyz0 = 0;
    float t = 0.0f, map = 0.0f, zeta = 0.0f;
    std::vector<int64_t> npatch, npart;           // levels 1..NL at [1..NL]
    // every patch, levels in order: PATCHNX..NZ, PATCHX..Z, PATCHRX..RZ
    std::vector<int32_t> pn[3], pl[3];
    std::vector<float> pr[3];
};
bool read_masclet_grid(const char *path, MascletGrid &g) {
    File in(path, "r");
    if (!in.f) return false;
    double v[4];
    if (!read_values(in.f, 4, v)) return false;
    g.t = (float)v[1];
    g.nl = (int)v[2];
    g.map = (float)v[3];
    if (!read_values(in.f, 1, v)) return false;
    g.zeta = (float)v[0];
    if (!read_values(in.f, 3, v)) return false;
    g.ndxyz0 = (int)v[1];
    if (g.nl < 0 || g.ndxyz0 < 0) return false;
    g.npatch.assign(g.nl + 1, 0);
    g.npart.assign(g.nl + 1, 0);
    for (int ir = 1; ir <= g.nl; ir++) {
        if (!read_values(in.f, 4, v)) return false;
        g.npatch[ir] = (int64_t)v[1];
        g.npart[ir] = (int64_t)v[2];
        if (g.npatch[ir] < 0 || g.npart[ir] < 0) return false;
        if (!read_values(in.f, 0, v)) return false;
        for (int64_t i = 0; i < g.npatch[ir]; i++) {
            if (!read_values(in.f, 3, v)) return false;
            for (int a = 0; a < 3; a++) g.pn[a].push_back((int32_t)v[a]);
            if (!read_values(in.f, 3, v)) return false;
            for (int a = 0; a < 3; a++) g.pl[a].push_back((int32_t)v[a]);
            if (!read_values(in.f, 3, v)) return false;
            for (int a = 0; a < 3; a++) g.pr[a].push_back((float)v[a]);       // READ(33,*) AAA,BBB,CCC
            if (!read_values(in.f, 1, v)) return false;
        }
    }
    return true;
}

}  // namespace

extern "C" {

int avism_io_particle_header(const char *path, int64_t *n, float *zeta) {
    if (!path || !n || !zeta) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    return read_particle_head(in.f, n, zeta) ? AVISM_OK : AVISM_ERR_IO;
}

namespace {

// READ_BINARY_PART_1 / _2: the header, then one record of NPARTT REAL*4 per
// destination array, in order
int read_particle_columns(const char *path, int64_t capacity, float *const *dst, int ncol) {
    for (int i = 0; i < ncol; i++)
        if (!dst[i]) return AVISM_ERR_ARG;
    if (!path) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    int64_t n;
    float zeta;
    if (!read_particle_head(in.f, &n, &zeta)) return AVISM_ERR_IO;
    if (n > capacity) return AVISM_ERR_ARG;                              // 'ERROR: NPARTT > PARTIRED'
    for (int i = 0; i < ncol; i++)
        if (!read_record(in.f, dst[i], (uint64_t)n * 4)) return AVISM_ERR_IO;
    return AVISM_OK;
}

}  // namespace

int avism_io_read_particles(const char *path, int64_t capacity, float *x, float *y, float *z, float *vx,
                            float *vy, float *vz, float *m) {
    float *const dst[7] = {x, y, z, vx, vy, vz, m};
    return read_particle_columns(path, capacity, dst, 7);
}

int avism_io_read_particles_novel(const char *path, int64_t capacity, float *x, float *y, float *z, float *m) {
    float *const dst[4] = {x, y, z, m};
    return read_particle_columns(path, capacity, dst, 4);
}

int avism_io_read_grid(const char *path, int32_t nx, float *zeta, float *u1, float *u2, float *u3, float *u4) {
    float *const dst[4] = {u1, u2, u3, u4};
    if (!path || !zeta || nx < 1) return AVISM_ERR_ARG;
    for (float *d : dst)
        if (!d) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    if (!read_record(in.f, zeta, 4)) return AVISM_ERR_IO;
    const uint64_t bytes = (uint64_t)nx * (uint64_t)nx * (uint64_t)nx * 4;
    for (float *d : dst)
        if (!read_record(in.f, d, bytes)) return AVISM_ERR_IO;
    return AVISM_OK;
}

int avism_io_masclet_header(const char *grid_path, int32_t *nl, int32_t *ndxyz0, int64_t *npartt, float *zeta,
                            float *map) {
    if (!grid_path) return AVISM_ERR_ARG;
    MascletGrid g;
    if (!read_masclet_grid(grid_path, g)) return AVISM_ERR_IO;
    int64_t n = g.ndxyz0;
    for (int ir = 1; ir <= g.nl; ir++) n += g.npart[ir];
    if (nl) *nl = g.nl;
    if (ndxyz0) *ndxyz0 = g.ndxyz0;
    if (npartt) *npartt = n;
    if (zeta) *zeta = g.zeta;
    if (map) *map = g.map;
    return AVISM_OK;
}

int avism_io_read_masclet(const char *grid_path, const char *gas_path, const char *dm_path, int32_t nhy,
                          float *u1g, float *u2g, float *u3g, float *u4g, int64_t capacity, float *x, float *y,
                          float *z, float *vx, float *vy, float *vz, float *m, int64_t *npartt) {
    if (!grid_path || !gas_path || !dm_path || nhy < 1) return AVISM_ERR_ARG;
    float *const gas[4] = {u1g, u2g, u3g, u4g};
    float *const part[7] = {x, y, z, vx, vy, vz, m};
    for (float *d : gas)
        if (!d) return AVISM_ERR_ARG;
    for (float *d : part)
        if (!d) return AVISM_ERR_ARG;
    MascletGrid g;
    if (!read_masclet_grid(grid_path, g)) return AVISM_ERR_IO;
    int64_t n = g.ndxyz0;
    for (int ir = 1; ir <= g.nl; ir++) n += g.npart[ir];
    if (n > capacity) return AVISM_ERR_ARG;                              // 'ERROR: NPARTT > PARTIRED'
    const uint64_t cells = (uint64_t)nhy * (uint64_t)nhy * (uint64_t)nhy * 4;
    // gas (src/reader.f90:259-273): a header record, then U1G, U2G, U3G, U4G at level 0
    {
        File in(gas_path, "rb");
        if (!in.f || !skip_record(in.f)) return AVISM_ERR_IO;
        for (float *d : gas)
            if (!read_record(in.f, d, cells)) return AVISM_ERR_IO;
    }
    // dark matter (src/reader.f90:315-385): a header record, U1DM, the level-0
    // particles' x, y, z, vx, vy, vz (mass MAP) and one more record; then per
    // level one record per patch (U11DM) and the particles' seven columns with
    // their masses, and one more record
    {
        File in(dm_path, "rb");
        if (!in.f || !skip_record(in.f) || !skip_record(in.f)) return AVISM_ERR_IO;
        int64_t conta = g.ndxyz0;
        for (int q = 0; q < 6; q++)
            if (!read_record(in.f, part[q], (uint64_t)g.ndxyz0 * 4)) return AVISM_ERR_IO;
        if (!skip_record(in.f)) return AVISM_ERR_IO;
        for (int64_t i = 0; i < g.ndxyz0; i++) m[i] = g.map;
        for (int ir = 1; ir <= g.nl; ir++) {
            for (int64_t i = 0; i < g.npatch[ir]; i++)
                if (!skip_record(in.f)) return AVISM_ERR_IO;
            for (int q = 0; q < 7; q++)
                if (!read_record(in.f, part[q] + conta, (uint64_t)g.npart[ir] * 4)) return AVISM_ERR_IO;
            if (!skip_record(in.f)) return AVISM_ERR_IO;
            conta += g.npart[ir];
        }
    }
    // delta to density (src/reader.f90:389-394)
    const uint64_t nc = (uint64_t)nhy * (uint64_t)nhy * (uint64_t)nhy;
    for (uint64_t c = 0; c < nc; c++) u1g[c] = u1g[c] + 1.0f;
    if (npartt) *npartt = n;
    return AVISM_OK;
}

int avism_io_masclet_patches_size(const char *grid_path, int32_t *npatch, int64_t *ncells) {
    if (!grid_path) return AVISM_ERR_ARG;
    MascletGrid g;
    if (!read_masclet_grid(grid_path, g)) return AVISM_ERR_IO;
    const int64_t np = g.nl >= 1 ? g.npatch[1] : 0;
    int64_t cells = 0;
    for (int64_t i = 0; i < np; i++) {
        for (int a = 0; a < 3; a++)
            if (g.pn[a][i] < 1 || g.pn[a][i] > (1 << 20)) return AVISM_ERR_IO;   // a patch edge of 2^20 cells at most
        cells += (int64_t)g.pn[0][i] * g.pn[1][i] * g.pn[2][i];
    }
    if (npatch) *npatch = (int32_t)np;
    if (ncells) *ncells = cells;
    return AVISM_OK;
}

int avism_io_read_masclet_patches(const char *grid_path, const char *gas_path, int32_t nhy, int32_t capacity,
                                  int64_t capacity_cells, int32_t *nx, int32_t *ny, int32_t *nz, int32_t *ix,
                                  int32_t *iy, int32_t *iz, float *rx, float *ry, float *rz, int64_t *offset,
                                  float *u11g, float *u12g, float *u13g, float *u14g) {
    int32_t *const geom[6] = {nx, ny, nz, ix, iy, iz};
    float *const corner[3] = {rx, ry, rz};
    float *const cells_out[4] = {u11g, u12g, u13g, u14g};
    if (!grid_path || !gas_path || nhy < 1 || !offset) return AVISM_ERR_ARG;
    for (int32_t *d : geom)
        if (!d) return AVISM_ERR_ARG;
    for (float *d : corner)
        if (!d) return AVISM_ERR_ARG;
    for (float *d : cells_out)
        if (!d) return AVISM_ERR_ARG;
    int32_t np = 0;
    int64_t ncells = 0;
    const int st = avism_io_masclet_patches_size(grid_path, &np, &ncells);
    if (st) return st;
    if (np > capacity || ncells > capacity_cells) return AVISM_ERR_ARG;
    MascletGrid g;
    if (!read_masclet_grid(grid_path, g)) return AVISM_ERR_IO;
    offset[0] = 0;
    for (int32_t i = 0; i < np; i++) {
        for (int a = 0; a < 3; a++) {
            geom[a][i] = g.pn[a][i];
            geom[3 + a][i] = g.pl[a][i];
            corner[a][i] = g.pr[a][i];
        }
        offset[i + 1] = offset[i] + (int64_t)g.pn[0][i] * g.pn[1][i] * g.pn[2][i];
    }
    // gas (src/reader.f90:259-312): the header, the four level-0 grids and six
    // more records; then per level-1 patch U11G, U12G, U13G, U14G and seven
    // more records
    File in(gas_path, "rb");
    if (!in.f || !skip_record(in.f)) return AVISM_ERR_IO;
    const uint64_t base = (uint64_t)nhy * (uint64_t)nhy * (uint64_t)nhy * 4;
    for (int q = 0; q < 4; q++) {
        uint64_t len = 0;
        if (!skip_record(in.f, &len) || len != base) return AVISM_ERR_IO;
    }
    for (int q = 0; q < 6; q++)
        if (!skip_record(in.f)) return AVISM_ERR_IO;
    for (int32_t i = 0; i < np; i++) {
        const uint64_t bytes = (uint64_t)(offset[i + 1] - offset[i]) * 4;
        for (float *d : cells_out)
            if (!read_record(in.f, d + offset[i], bytes)) return AVISM_ERR_IO;
        for (int q = 0; q < 7; q++)
            if (!skip_record(in.f)) return AVISM_ERR_IO;
    }
    // delta to density (src/reader.f90:393)
    for (int64_t c = 0; c < ncells; c++) u11g[c] = u11g[c] + 1.0f;
    return AVISM_OK;
}

int avism_io_read_mask(const char *path, int32_t ncox, int32_t nx, int8_t *smask, float *lims) {
    if (!path || !smask || ncox < 1 || nx < 1) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    int32_t nmask = 0;
    float hdr[3];
    if (std::fread(&nmask, 4, 1, in.f) != 1) return AVISM_ERR_IO;
    if (nmask != ncox) return AVISM_ERR_ARG;       // 'MASK grid does not coincide with AVISM coarse grid'
    if (std::fread(hdr, 4, 3, in.f) != 3) return AVISM_ERR_IO;
    if (lims) std::memcpy(lims, hdr, sizeof hdr);
    const size_t nm = (size_t)nmask;
    std::vector<int8_t> m2(nm * nm * nm);
    if (std::fread(m2.data(), 1, m2.size(), in.f) != m2.size()) return AVISM_ERR_IO;
    int ndown = 1;
    if (nx > nmask) {
        ndown = nx / nmask;
        if (ndown % 2 != 0) return AVISM_ERR_ARG;  // 'STH WRONG IN MASK INTERPOLATION'
    } else if (nx != nmask) {
        return AVISM_ERR_ARG;
    }
    const size_t n = (size_t)nx;
    for (size_t k = 0; k < n; k++)
        for (size_t j = 0; j < n; j++)
            for (size_t i = 0; i < n; i++) {
                const size_t i2 = i / ndown, j2 = j / ndown, k2 = k / ndown;
                int8_t v = m2[i2 + nm * (j2 + nm * k2)];
                if (v > 0) v = 1;                  // WHERE (SMASK > 0) SMASK = 1
                smask[i + n * (j + n * k)] = v;
            }
    return AVISM_OK;
}

int avism_io_randoms_header(const char *path, int32_t *nrand) {
    if (!path || !nrand) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    if (!read_record(in.f, nrand, 4)) return AVISM_ERR_IO;
    return *nrand >= 0 ? AVISM_OK : AVISM_ERR_IO;
}

int avism_io_read_randoms(const char *path, int32_t capacity, float *x, float *y, float *z, float *w) {
    float *const dst[4] = {x, y, z, w};
    if (!path) return AVISM_ERR_ARG;
    for (float *d : dst)
        if (!d) return AVISM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return AVISM_ERR_IO;
    int32_t n = 0;
    if (!read_record(in.f, &n, 4) || n < 0) return AVISM_ERR_IO;
    if (n > capacity) return AVISM_ERR_ARG;
    for (float *d : dst)
        if (!read_record(in.f, d, (uint64_t)n * 4)) return AVISM_ERR_IO;
    return AVISM_OK;
}

int avism_io_write_vel_cube(const char *path, int32_t nx, const float *u2, const float *u3, const float *u4) {
    if (!path || nx < 1 || !u2 || !u3 || !u4) return AVISM_ERR_ARG;
    File out(path, "wb");
    if (!out.f) return AVISM_ERR_IO;
    const size_t nc = (size_t)nx * (size_t)nx * (size_t)nx;
    for (const float *u : {u2, u3, u4})
        if (std::fwrite(u, 4, nc, out.f) != nc) return AVISM_ERR_IO;
    return std::fflush(out.f) == 0 ? AVISM_OK : AVISM_ERR_IO;
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
