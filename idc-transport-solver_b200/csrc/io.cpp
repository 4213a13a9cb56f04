// Binary files of the reference's serial 2-D build: scalar flux (.sd2) and angular flux (.af2).
//
//   .sd2: [nx:i64, ax:f64, bx:f64] [ny:i64, ay:f64, by:f64]          SpatialDomain::WriteToDisk
//         dg_degree:i64, size_bytes:i64, count:i64, density:f64[count]  DensityFunction::WriteToDisk
//   .af2: the same domain block, then the ordinate type name (null-terminated, "#R" appended when the
//         set is symmetric-reduced) and ang_order:i64 (OrdinateFlux::WriteToDisk), then dg_degree,
//         size_bytes, count and the density.
// (objects/SpatialDomain.cpp:385-411, objects/RKDG/DensityFunction.cpp:2228-2400,
//  objects/RKDG/OrdinateFlux.cpp:2553-2620, 2720-2930, utils/global.cpp:162-185.)  The density is the
// halo layout the ABI uses everywhere, so files map to and from the sweep's arrays without re-layout.
// Little-endian host byte order, as the reference writes it.
#include "idcsweep.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct File {
    std::FILE *f = nullptr;
    explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

template <typename T>
bool put(std::FILE *f, const T &v) {
    return std::fwrite(&v, sizeof(T), 1, f) == 1;
}
template <typename T>
bool get(std::FILE *f, T *v) {
    return std::fread(v, sizeof(T), 1, f) == 1;
}

bool put_domain(std::FILE *f, int64_t nx, int64_t ny, double ax, double bx, double ay, double by) {
    return put(f, nx) && put(f, ax) && put(f, bx) && put(f, ny) && put(f, ay) && put(f, by);
}
bool get_domain(std::FILE *f, int64_t *nx, int64_t *ny, double *ax, double *bx, double *ay, double *by) {
    return get(f, nx) && get(f, ax) && get(f, bx) && get(f, ny) && get(f, ay) && get(f, by);
}

bool put_density(std::FILE *f, int64_t p, int64_t count, const double *d) {
    const int64_t bytes = count * (int64_t)sizeof(double);
    return put(f, p) && put(f, bytes) && put(f, count) &&
           std::fwrite(d, sizeof(double), (size_t)count, f) == (size_t)count;
}

bool get_string(std::FILE *f, std::string *s) {
    s->clear();
    for (int n = 0; n < 4096; ++n) {
        const int c = std::fgetc(f);
        if (c == EOF) return false;
        if (c == 0) return true;
        s->push_back((char)c);
    }
    return false;
}

}  // namespace

extern "C" {

int idc_write_sd2(const char *path, int64_t nx, int64_t ny, double ax, double bx, double ay, double by,
                  int64_t dg_degree, const double *density) {
    if (!path || !density || nx <= 0 || ny <= 0 || dg_degree < 0) return IDC_ERR_ARG;
    File fl(path, "wb");
    if (!fl.f) return IDC_ERR_ARG;
    const int64_t count = (nx + 2) * (ny + 2) * (dg_degree + 1) * (dg_degree + 1);
    if (!put_domain(fl.f, nx, ny, ax, bx, ay, by) || !put_density(fl.f, dg_degree, count, density)) return IDC_ERR_ARG;
    return IDC_OK;
}

int idc_read_sd2(const char *path, int64_t *nx, int64_t *ny, double *ax, double *bx, double *ay, double *by,
                 int64_t *dg_degree, double *density, int64_t capacity, int64_t *count) {
    if (!path || !nx || !ny || !ax || !bx || !ay || !by || !dg_degree || !count) return IDC_ERR_ARG;
    File fl(path, "rb");
    if (!fl.f) return IDC_ERR_ARG;
    int64_t bytes = 0;
    if (!get_domain(fl.f, nx, ny, ax, bx, ay, by) || !get(fl.f, dg_degree) || !get(fl.f, &bytes) || !get(fl.f, count))
        return IDC_ERR_ARG;
    if (*count != (*nx + 2) * (*ny + 2) * (*dg_degree + 1) * (*dg_degree + 1) || bytes != *count * 8) return IDC_ERR_ARG;
    if (!density) return IDC_OK;   // header only
    if (capacity < *count) return IDC_ERR_ARG;
    if (std::fread(density, sizeof(double), (size_t)*count, fl.f) != (size_t)*count) return IDC_ERR_ARG;
    return IDC_OK;
}

int idc_write_af2(const char *path, int64_t nx, int64_t ny, double ax, double bx, double ay, double by,
                  const char *ordinate_type, int64_t ang_order, int64_t dg_degree, int64_t nq, const double *density) {
    if (!path || !density || !ordinate_type || nx <= 0 || ny <= 0 || dg_degree < 0 || nq <= 0) return IDC_ERR_ARG;
    File fl(path, "wb");
    if (!fl.f) return IDC_ERR_ARG;
    const int64_t count = (nx + 2) * (ny + 2) * nq * (dg_degree + 1) * (dg_degree + 1);
    const size_t len = std::strlen(ordinate_type) + 1;   // with the null byte
    if (!put_domain(fl.f, nx, ny, ax, bx, ay, by) || std::fwrite(ordinate_type, 1, len, fl.f) != len ||
        !put(fl.f, ang_order) || !put_density(fl.f, dg_degree, count, density))
        return IDC_ERR_ARG;
    return IDC_OK;
}

int idc_read_af2(const char *path, int64_t *nx, int64_t *ny, double *ax, double *bx, double *ay, double *by,
                 char *ordinate_type, int64_t type_capacity, int64_t *ang_order, int64_t *dg_degree, double *density,
                 int64_t capacity, int64_t *count) {
    if (!path || !nx || !ny || !ax || !bx || !ay || !by || !ang_order || !dg_degree || !count) return IDC_ERR_ARG;
    File fl(path, "rb");
    if (!fl.f) return IDC_ERR_ARG;
    std::string type;
    int64_t bytes = 0;
    if (!get_domain(fl.f, nx, ny, ax, bx, ay, by) || !get_string(fl.f, &type) || !get(fl.f, ang_order) ||
        !get(fl.f, dg_degree) || !get(fl.f, &bytes) || !get(fl.f, count))
        return IDC_ERR_ARG;
    const int64_t per_q = (*nx + 2) * (*ny + 2) * (*dg_degree + 1) * (*dg_degree + 1);
    if (per_q <= 0 || *count % per_q != 0 || bytes != *count * 8) return IDC_ERR_ARG;
    if (ordinate_type) {
        if ((int64_t)type.size() + 1 > type_capacity) return IDC_ERR_ARG;
        std::memcpy(ordinate_type, type.c_str(), type.size() + 1);
    }
    if (!density) return IDC_OK;
    if (capacity < *count) return IDC_ERR_ARG;
    if (std::fread(density, sizeof(double), (size_t)*count, fl.f) != (size_t)*count) return IDC_ERR_ARG;
    return IDC_OK;
}

}  // extern "C"
