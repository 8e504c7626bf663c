// Jacobian determinant on device pointers without any allocation.
//
// Some callers cannot let a library allocate device memory when they need a
// Jacobian map:
// * hosts that fix their device-memory budget at start-up (real-time and
//   embedded systems), where a later cudaMalloc may fail or, because
//   cudaMalloc and cudaFree can synchronise the device, stall a loop that
//   has a deadline;
// * processes whose device memory is already handed out by another
//   allocator (a framework's caching allocator that reserved it), so an
//   allocation of the library's own fails;
// * runtimes without an allocator of their own, which pass the library
//   pointers into memory they manage.
// dtb_jacobian_device() draws its launch descriptor and tile table from the
// library's growing device workspace and may call cudaMalloc; this entry
// point keeps them in a fixed array in device memory that is part of the
// library image instead.
//
// The array is `g_noalloc_scratch` below: NOALLOC_SCRATCH_BYTES (65 KiB)
// that every GPU which loads this library holds until the process exits.  It
// is shared by every call on a device and keeps the contents of the last
// call, so two calls whose work overlaps on the GPU (for instance on two
// streams without ordering between them) race on it.  The descriptor is
// written into the array by a one-thread kernel that receives it as a
// launch argument, and the tile table is cleared by a memset, so nothing is
// copied from host memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "dt_internal.h"

using namespace dtb;

namespace {

// Launch descriptor (VolumeDesc<float> or VolumeDesc<double>) in the first
// kilobyte, then one tile-to-volume entry per tile.
constexpr size_t NOALLOC_DESC_BYTES = 1024;
constexpr int NOALLOC_MAX_TILES = 16384;
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_DESC_BYTES + NOALLOC_MAX_TILES * sizeof(int);
static_assert(sizeof(VolumeDesc<double>) <= NOALLOC_DESC_BYTES, "descriptor does not fit");
static_assert(sizeof(VolumeDesc<float>) <= NOALLOC_DESC_BYTES, "descriptor does not fit");

// Host code may only use this name to look up the device address (see
// scratch_address); passed to a kernel directly it would not be one.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

void report(int line, const char *function, const char *message) {
    disptools_error_state *e = disptools_get_error();
    e->error = true;
    e->line = line;
    std::snprintf(e->file, sizeof e->file, "%s", __FILE__);
    std::snprintf(e->function, sizeof e->function, "%s", function);
    std::snprintf(e->message, sizeof e->message, "%s", message);
    e->trace[0] = '\0';
}

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this set-up).
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        report(__LINE__, __func__, cudaGetErrorString(e));
        return DTB_ERR_CUDA;
    }
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        report(__LINE__, __func__, "device ordinal beyond the supported range");
        return DTB_ERR_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            report(__LINE__, __func__, "cudaGetSymbolAddress of the scratch array failed");
            return DTB_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
    return DTB_OK;
}

// Writes the launch descriptor into the fixed array.
template <typename T>
__global__ void k_store_desc(const VolumeDesc<T> d, VolumeDesc<T> *out) {
    *out = d;
}

template <typename T>
int jacobian_noalloc(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz, int order, const T *field,
                     T *J, cudaStream_t s) {
    const int bz = nz < 32 ? (int) nz : 32;
    const long long tiles = (long long) ((nx + BX - 1) / BX) * (long long) ((ny + BY - 1) / BY) *
                            (long long) ((nz + bz - 1) / bz);
    if (tiles > NOALLOC_MAX_TILES) {
        char m[256];
        std::snprintf(m, sizeof m,
                      "volume too large for dtb_jacobian_device_noalloc: %lld tiles of %dx%dx%d voxels, "
                      "the fixed scratch holds %d (use dtb_jacobian_device)",
                      tiles, BX, BY, bz, NOALLOC_MAX_TILES);
        report(__LINE__, __func__, m);
        return DTB_ERR_ARGUMENT;
    }
    unsigned char *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != DTB_OK) return rc;

    VolumeDesc<T> d;
    std::memset(&d, 0, sizeof d);
    d.g.nx = (int) nx;
    d.g.ny = (int) ny;
    d.g.nz = (int) nz;
    d.g.order = order;
    d.g.ys = (long long) nx;
    d.g.zs = (long long) nx * ny;
    d.g.cs = (long long) nx * ny * nz;
    d.g.ih[0] = 1.0 / dx;
    d.g.ih[1] = 1.0 / dy;
    d.g.ih[2] = 1.0 / dz;
    d.g.sp[0] = dx;
    d.g.sp[1] = dy;
    d.g.sp[2] = dz;
    d.field[0] = const_cast<T *>(field);
    d.jout = J;
    d.tiles_x = (int) ((nx + BX - 1) / BX);
    d.tiles_y = (int) ((ny + BY - 1) / BY);
    d.tiles_z = (int) ((nz + bz - 1) / bz);
    d.ntiles = (int) tiles;
    d.bz = bz;
    VolumeDesc<T> *d_desc = reinterpret_cast<VolumeDesc<T> *>(scratch);
    int *d_tile_vol = reinterpret_cast<int *>(scratch + NOALLOC_DESC_BYTES);
    // The descriptor travels as a kernel argument (the launch keeps its own
    // copy), so `d` may go out of scope as soon as the launch is enqueued.
    k_store_desc<T><<<1, 1, 0, s>>>(d, d_desc);
    count_launch();
    cudaError_t e = cudaGetLastError();
    // Every tile belongs to volume 0: the table must be zero, whatever the
    // previous call left there.
    if (e == cudaSuccess) e = cudaMemsetAsync(d_tile_vol, 0, (size_t) tiles * sizeof(int), s);
    if (e == cudaSuccess) e = launch_jacobian<T>(d_desc, d_tile_vol, (int) tiles, (int) tiles, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        report(__LINE__, __func__, cudaGetErrorString(e));
        return DTB_ERR_CUDA;
    }
    return DTB_OK;
}

}  // namespace

extern "C" int dtb_jacobian_device_noalloc(int precision, int order, size_t nx, size_t ny, size_t nz, double dx,
                                           double dy, double dz, const void *field, void *J, void *stream) {
    disptools_clear_error();
    if (nx < 3 || ny < 3 || nz < 3 || nx >= (1u << 30) || ny >= (1u << 30) || nz >= (1u << 30)) {
        report(__LINE__, __func__, "every axis needs at least 3 voxels");
        return DTB_ERR_ARGUMENT;
    }
    if (!field || !J) {
        report(__LINE__, __func__, "null array");
        return DTB_ERR_ARGUMENT;
    }
    if (order != 4 && order != 2) {
        report(__LINE__, __func__, "order must be 4 or 2");
        return DTB_ERR_ARGUMENT;
    }
    if (!(dx > 0.0 && dy > 0.0 && dz > 0.0)) {
        report(__LINE__, __func__, "spacing must be positive");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == DTB_PRECISION_FP64)
        return jacobian_noalloc<double>(nx, ny, nz, dx, dy, dz, order, static_cast<const double *>(field),
                                        static_cast<double *>(J), s);
    if (precision == DTB_PRECISION_MIXED)
        return jacobian_noalloc<float>(nx, ny, nz, dx, dy, dz, order, static_cast<const float *>(field),
                                       static_cast<float *>(J), s);
    report(__LINE__, __func__, "invalid precision");
    return DTB_ERR_ARGUMENT;
}
