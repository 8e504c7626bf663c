// Field files: RVF and legacy VTK (STRUCTURED_POINTS), host code.
//
// Formats as written by the reference C library:
// * RVF (src/rvf_io.c:11-50): a text line "nx ny nz", a text line
//   "dx dy dz" (printf %f), then 3 doubles per voxel in native byte order,
//   voxels x fastest, the three components of a voxel together.
// * VTK (src/vtk_io.c:74-133): the legacy header (version line, a comment
//   line, BINARY, DATASET STRUCTURED_POINTS, DIMENSIONS nx ny nz, ORIGIN
//   0 0 0, SPACING dx dy dz (%f), POINT_DATA n, SCALARS <name> double nd,
//   LOOKUP_TABLE default), then nd big-endian doubles per voxel, x fastest.
//
// Arrays at this ABI are component-major, [nd][nz][ny][nx], like every other
// array of the library.
//
// Readers:
// * Header values are parsed as the reference's readers parse them; the
//   spacing goes through a float (src/rvf_io.c:75-90, src/vtk_io.c:152-160).
// * The RVF binary data starts right after the second header line, and a
//   VTK file's right after the line that begins with 'L'.  The reference's
//   RVF reader ends its second fscanf with "\n", which also swallows
//   whitespace bytes at the start of the binary data; this reader does not.
// * Short files and unsupported element types (VTK float data, which the
//   reference rejects too) are errors.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "disptools_b200.h"

namespace {

void report(int line, const char *function, const std::string &message) {
    disptools_error_state *e = disptools_get_error();
    e->error = true;
    e->line = line;
    std::snprintf(e->file, sizeof e->file, "%s", __FILE__);
    std::snprintf(e->function, sizeof e->function, "%s", function);
    std::snprintf(e->message, sizeof e->message, "%s", message.c_str());
    e->trace[0] = '\0';
}

#define IO_FAIL(msg)                         \
    do {                                     \
        report(__LINE__, __func__, (msg));   \
        return DTB_ERR_IO;                   \
    } while (0)
#define ARG_FAIL(msg)                        \
    do {                                     \
        report(__LINE__, __func__, (msg));   \
        return DTB_ERR_ARGUMENT;             \
    } while (0)

struct File {
    FILE *fp = nullptr;
    ~File() {
        if (fp) std::fclose(fp);
    }
};

bool host_is_big_endian() {
    const uint16_t v = 0x0100;
    unsigned char b;
    std::memcpy(&b, &v, 1);
    return b == 0x01;
}

double swap_double(double v) {
    unsigned char in[8], out[8];
    std::memcpy(in, &v, 8);
    for (int i = 0; i < 8; ++i) out[i] = in[7 - i];
    double r;
    std::memcpy(&r, out, 8);
    return r;
}

// Reads one line (without the newline) into `out`; false at end of file.
bool read_line(FILE *fp, std::string *out) {
    out->clear();
    int c;
    while ((c = std::fgetc(fp)) != EOF) {
        if (c == '\n') return true;
        out->push_back((char) c);
    }
    return !out->empty();
}

bool dims_ok(size_t nx, size_t ny, size_t nz) { return nx > 0 && ny > 0 && nz > 0; }

struct RvfHeader {
    size_t nx = 0, ny = 0, nz = 0;
    double dx = 0, dy = 0, dz = 0;
};

int rvf_header(FILE *fp, RvfHeader *h) {
    std::string l1, l2;
    if (!read_line(fp, &l1) || std::sscanf(l1.c_str(), "%zu %zu %zu", &h->nx, &h->ny, &h->nz) != 3)
        IO_FAIL("read_rvf: expected size (3 integers)");
    float fx, fy, fz;
    if (!read_line(fp, &l2) || std::sscanf(l2.c_str(), "%f %f %f", &fx, &fy, &fz) != 3)
        IO_FAIL("read_rvf: expected spacing (3 floats)");
    h->dx = fx;
    h->dy = fy;
    h->dz = fz;
    if (!dims_ok(h->nx, h->ny, h->nz)) IO_FAIL("read_rvf: empty volume");
    return DTB_OK;
}

struct VtkHeader {
    int nd = 0;
    size_t nx = 0, ny = 0, nz = 0;
    double dx = 1, dy = 1, dz = 1;
};

int vtk_header(FILE *fp, VtkHeader *h) {
    std::string l;
    bool dims = false, scalars = false;
    float fx = 1.f, fy = 1.f, fz = 1.f;
    while (read_line(fp, &l)) {
        if (!l.empty() && l[0] == 'L') break;  // LOOKUP_TABLE: the data follows
        size_t a, b, c;
        if (std::sscanf(l.c_str(), "DIMENSIONS %zu %zu %zu", &a, &b, &c) == 3) {
            h->nx = a, h->ny = b, h->nz = c;
            dims = true;
        }
        std::sscanf(l.c_str(), "SPACING %f %f %f", &fx, &fy, &fz);
        size_t nd = 0;
        char name[256];
        char type[64];
        if (std::sscanf(l.c_str(), "SCALARS %255s %63s %zu", name, type, &nd) == 3) {
            if (std::strcmp(type, "double") != 0) IO_FAIL("read_vtk: only double data is supported");
            h->nd = (int) nd;
            scalars = true;
        }
    }
    if (!dims || !scalars || h->nd < 1 || !dims_ok(h->nx, h->ny, h->nz))
        IO_FAIL("read_vtk: missing DIMENSIONS or SCALARS ... double <components>");
    h->dx = fx;
    h->dy = fy;
    h->dz = fz;
    return DTB_OK;
}

}  // namespace

extern "C" int dtb_write_rvf(const char *filename, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                             const double *field) {
    disptools_clear_error();
    if (!filename || !field || !dims_ok(nx, ny, nz)) ARG_FAIL("write_rvf: invalid arguments");
    const size_t n = nx * ny * nz;
    std::vector<double> buf(3 * n);
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) buf[3 * i + c] = field[c * n + i];
    File f;
    f.fp = std::fopen(filename, "wb");
    if (!f.fp) IO_FAIL(std::string("write_rvf: ") + std::strerror(errno));
    std::fprintf(f.fp, "%zu %zu %zu\n%f %f %f\n", nx, ny, nz, dx, dy, dz);
    if (std::fwrite(buf.data(), sizeof(double), buf.size(), f.fp) != buf.size()) IO_FAIL("write_rvf: short write");
    return DTB_OK;
}

extern "C" int dtb_read_rvf_header(const char *filename, size_t *nx, size_t *ny, size_t *nz, double *dx, double *dy,
                                   double *dz) {
    disptools_clear_error();
    if (!filename || !nx || !ny || !nz || !dx || !dy || !dz) ARG_FAIL("read_rvf: null argument");
    File f;
    f.fp = std::fopen(filename, "rb");
    if (!f.fp) IO_FAIL(std::string("read_rvf: ") + std::strerror(errno));
    RvfHeader h;
    const int rc = rvf_header(f.fp, &h);
    if (rc != DTB_OK) return rc;
    *nx = h.nx, *ny = h.ny, *nz = h.nz, *dx = h.dx, *dy = h.dy, *dz = h.dz;
    return DTB_OK;
}

extern "C" int dtb_read_rvf(const char *filename, double *field, size_t capacity) {
    disptools_clear_error();
    if (!filename || !field) ARG_FAIL("read_rvf: null argument");
    File f;
    f.fp = std::fopen(filename, "rb");
    if (!f.fp) IO_FAIL(std::string("read_rvf: ") + std::strerror(errno));
    RvfHeader h;
    const int rc = rvf_header(f.fp, &h);
    if (rc != DTB_OK) return rc;
    const size_t n = h.nx * h.ny * h.nz;
    if (capacity < 3 * n) ARG_FAIL("read_rvf: output array too small");
    std::vector<double> buf(3 * n);
    if (std::fread(buf.data(), sizeof(double), buf.size(), f.fp) != buf.size()) IO_FAIL("read_rvf: file too short");
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) field[c * n + i] = buf[3 * i + c];
    return DTB_OK;
}

extern "C" int dtb_write_vtk(const char *filename, int nd, size_t nx, size_t ny, size_t nz, double dx, double dy,
                             double dz, const double *data) {
    disptools_clear_error();
    if (!filename || !data || nd < 1 || !dims_ok(nx, ny, nz)) ARG_FAIL("write_vtk: invalid arguments");
    const size_t n = nx * ny * nz;
    const bool swap = !host_is_big_endian();
    std::vector<double> buf((size_t) nd * n);
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < nd; ++c) {
            const double v = data[(size_t) c * n + i];
            buf[(size_t) nd * i + c] = swap ? swap_double(v) : v;
        }
    File f;
    f.fp = std::fopen(filename, "wb");
    if (!f.fp) IO_FAIL(std::string("write_vtk: ") + std::strerror(errno));
    std::fprintf(f.fp,
                 "# vtk DataFile Version 3.0\n"
                 "Generated by disptools_b200\n"
                 "BINARY\n"
                 "DATASET STRUCTURED_POINTS\n"
                 "DIMENSIONS %zu %zu %zu\n"
                 "ORIGIN 0 0 0\n"
                 "SPACING %f %f %f\n"
                 "POINT_DATA %zu\n"
                 "SCALARS image_data double %d\n"
                 "LOOKUP_TABLE default\n",
                 nx, ny, nz, dx, dy, dz, n, nd);
    if (std::fwrite(buf.data(), sizeof(double), buf.size(), f.fp) != buf.size()) IO_FAIL("write_vtk: short write");
    return DTB_OK;
}

extern "C" int dtb_read_vtk_header(const char *filename, int *nd, size_t *nx, size_t *ny, size_t *nz, double *dx,
                                   double *dy, double *dz) {
    disptools_clear_error();
    if (!filename || !nd || !nx || !ny || !nz || !dx || !dy || !dz) ARG_FAIL("read_vtk: null argument");
    File f;
    f.fp = std::fopen(filename, "rb");
    if (!f.fp) IO_FAIL(std::string("read_vtk: ") + std::strerror(errno));
    VtkHeader h;
    const int rc = vtk_header(f.fp, &h);
    if (rc != DTB_OK) return rc;
    *nd = h.nd, *nx = h.nx, *ny = h.ny, *nz = h.nz, *dx = h.dx, *dy = h.dy, *dz = h.dz;
    return DTB_OK;
}

extern "C" int dtb_read_vtk(const char *filename, double *data, size_t capacity) {
    disptools_clear_error();
    if (!filename || !data) ARG_FAIL("read_vtk: null argument");
    File f;
    f.fp = std::fopen(filename, "rb");
    if (!f.fp) IO_FAIL(std::string("read_vtk: ") + std::strerror(errno));
    VtkHeader h;
    const int rc = vtk_header(f.fp, &h);
    if (rc != DTB_OK) return rc;
    const size_t n = h.nx * h.ny * h.nz;
    if (capacity < (size_t) h.nd * n) ARG_FAIL("read_vtk: output array too small");
    std::vector<double> buf((size_t) h.nd * n);
    if (std::fread(buf.data(), sizeof(double), buf.size(), f.fp) != buf.size()) IO_FAIL("read_vtk: file too short");
    const bool swap = !host_is_big_endian();
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < h.nd; ++c) {
            const double v = buf[(size_t) h.nd * i + c];
            data[(size_t) c * n + i] = swap ? swap_double(v) : v;
        }
    return DTB_OK;
}
