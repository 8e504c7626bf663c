// Smoothing and resampling of volumes for the multi-resolution pyramid.
//
// disptools' displacement() wrapper (disptools/displacements.py:443-472)
// builds each coarser level by scale_image (disptools/drawing.py:23-69):
// a Gaussian of 2.0 physical units, then a resampling onto a grid of the
// requested size that spans the same physical extent (output spacing
// s * n / n2, same origin).  The finer level's initial field is the coarser
// solution passed through the same function.  These kernels restate both
// steps on the device.
//
// * Smoothing: separable Gaussian, one pass per axis.  The weights are
//   exp(-k^2 / (2 sigma^2)) for |k| <= ceil(4 sigma), normalised to sum 1.
//   The border is zero-flux (indices clamped into the volume).  The sums are
//   formed in double in increasing k with explicitly rounded operations, so
//   the result is a fixed function of the input that a host restatement
//   reproduces bit for bit.  The reference uses ITK's recursive Gaussian,
//   an IIR approximation of the same filter, which is not available here.
// * Resampling: output voxel i of an axis samples the input at the
//   continuous index p = i * n / n2.  A point is inside the input when
//   -0.5 <= p < n - 0.5 on every axis (the half-voxel border of ITK's
//   images); outside points get 0, the resampler's default value.  Linear
//   mode interpolates along x, then y, then z, clamping the neighbour index
//   into the volume.  Nearest mode takes floor(p + 0.5).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "dt_internal.h"

using namespace dtb;

namespace {

constexpr int SMOOTH_MAX_RADIUS = 128;

struct SmoothWeights {
    int radius;
    double w[2 * SMOOTH_MAX_RADIUS + 1];
};

// One axis of the separable Gaussian over `comps` volumes of nx x ny x nz.
template <typename T>
__global__ void k_smooth_axis(const T *__restrict__ in, T *__restrict__ out, int nx, int ny, int nz, int comps,
                              int axis, SmoothWeights sw) {
    const long long n = (long long) nx * ny * nz * comps;
    const int len = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const long long stride = axis == 0 ? 1 : (axis == 1 ? (long long) nx : (long long) nx * ny);
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        const long long r = i / nx;
        const int pos = axis == 0 ? (int) (i % nx) : (axis == 1 ? (int) (r % ny) : (int) ((r / ny) % nz));
        const T *line = in + (i - (long long) pos * stride);
        double acc = 0.0;
        for (int k = -sw.radius; k <= sw.radius; ++k) {
            const int q = min(max(pos + k, 0), len - 1);
            acc = __dadd_rn(acc, __dmul_rn(sw.w[k + sw.radius], (double) line[(long long) q * stride]));
        }
        out[i] = (T) acc;
    }
}

__device__ __forceinline__ double lerp_rn(double a, double b, double f) {
    return __dadd_rn(a, __dmul_rn(__dsub_rn(b, a), f));
}

template <typename T>
__global__ void k_resample(const T *__restrict__ in, T *__restrict__ out, int nx, int ny, int nz, int nx2, int ny2,
                           int nz2, int comps, int mode) {
    const long long n2 = (long long) nx2 * ny2 * nz2 * comps;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n2;
         i += (long long) gridDim.x * blockDim.x) {
        const int x2 = (int) (i % nx2);
        long long r = i / nx2;
        const int y2 = (int) (r % ny2);
        r /= ny2;
        const int z2 = (int) (r % nz2);
        const int c = (int) (r / nz2);
        const double px = __ddiv_rn((double) x2 * (double) nx, (double) nx2);
        const double py = __ddiv_rn((double) y2 * (double) ny, (double) ny2);
        const double pz = __ddiv_rn((double) z2 * (double) nz, (double) nz2);
        const bool inside = px >= -0.5 && px < nx - 0.5 && py >= -0.5 && py < ny - 0.5 && pz >= -0.5 &&
                            pz < nz - 0.5;
        if (!inside) {
            out[i] = T(0);
            continue;
        }
        const T *vol = in + (long long) c * nx * ny * nz;
        auto at = [&](int x, int y, int z) -> double {
            return (double) vol[((long long) z * ny + y) * nx + x];
        };
        if (mode == 1) {  // nearest
            const int x = min((int) floor(px + 0.5), nx - 1);
            const int y = min((int) floor(py + 0.5), ny - 1);
            const int z = min((int) floor(pz + 0.5), nz - 1);
            out[i] = (T) at(x, y, z);
            continue;
        }
        const double fx0 = floor(px), fy0 = floor(py), fz0 = floor(pz);
        const double fx = __dsub_rn(px, fx0), fy = __dsub_rn(py, fy0), fz = __dsub_rn(pz, fz0);
        const int x0 = max((int) fx0, 0), y0 = max((int) fy0, 0), z0 = max((int) fz0, 0);
        const int x1 = min((int) fx0 + 1, nx - 1), y1 = min((int) fy0 + 1, ny - 1), z1 = min((int) fz0 + 1, nz - 1);
        const double c00 = lerp_rn(at(x0, y0, z0), at(x1, y0, z0), fx);
        const double c10 = lerp_rn(at(x0, y1, z0), at(x1, y1, z0), fx);
        const double c01 = lerp_rn(at(x0, y0, z1), at(x1, y0, z1), fx);
        const double c11 = lerp_rn(at(x0, y1, z1), at(x1, y1, z1), fx);
        const double c0 = lerp_rn(c00, c10, fy);
        const double c1 = lerp_rn(c01, c11, fy);
        out[i] = (T) lerp_rn(c0, c1, fz);
    }
}

void report(int line, const char *function, const char *message) {
    disptools_error_state *e = disptools_get_error();
    e->error = true;
    e->line = line;
    std::snprintf(e->file, sizeof e->file, "%s", __FILE__);
    std::snprintf(e->function, sizeof e->function, "%s", function);
    std::snprintf(e->message, sizeof e->message, "%s", message);
    e->trace[0] = '\0';
}

int grid_for(long long n) {
    const long long blocks = (n + 255) / 256;
    return (int) (blocks < 148 * 32 ? (blocks > 0 ? blocks : 1) : 148 * 32);
}

bool make_weights(double sigma, SmoothWeights *sw) {
    std::memset(sw, 0, sizeof *sw);
    if (!(sigma > 0.0)) {  // no smoothing along this axis
        sw->radius = 0;
        sw->w[0] = 1.0;
        return true;
    }
    const int r = (int) std::ceil(4.0 * sigma);
    if (r > SMOOTH_MAX_RADIUS) return false;
    sw->radius = r;
    double sum = 0.0;
    for (int k = -r; k <= r; ++k) {
        sw->w[k + r] = std::exp(-(double) k * k / (2.0 * sigma * sigma));
        sum += sw->w[k + r];
    }
    for (int k = 0; k <= 2 * r; ++k) sw->w[k] /= sum;
    return true;
}

template <typename T>
cudaError_t smooth(int comps, int nx, int ny, int nz, const SmoothWeights (&sw)[3], const T *in, T *out, T *scratch,
                   cudaStream_t s) {
    const long long n = (long long) nx * ny * nz * comps;
    const int grid = grid_for(n);
    k_smooth_axis<T><<<grid, 256, 0, s>>>(in, out, nx, ny, nz, comps, 0, sw[0]);
    count_launch();
    k_smooth_axis<T><<<grid, 256, 0, s>>>(out, scratch, nx, ny, nz, comps, 1, sw[1]);
    count_launch();
    k_smooth_axis<T><<<grid, 256, 0, s>>>(scratch, out, nx, ny, nz, comps, 2, sw[2]);
    count_launch();
    return cudaGetLastError();
}

bool dims_ok(size_t nx, size_t ny, size_t nz) {
    return nx >= 1 && ny >= 1 && nz >= 1 && nx < (1u << 30) && ny < (1u << 30) && nz < (1u << 30);
}

}  // namespace

extern "C" int dtb_smooth_device(int precision, int comps, size_t nx, size_t ny, size_t nz, double sigma_x,
                                 double sigma_y, double sigma_z, const void *in, void *out, void *scratch,
                                 void *stream) {
    disptools_clear_error();
    if (!dims_ok(nx, ny, nz) || comps < 1) {
        report(__LINE__, __func__, "invalid dimensions");
        return DTB_ERR_ARGUMENT;
    }
    if (!in || !out || !scratch) {
        report(__LINE__, __func__, "null array");
        return DTB_ERR_ARGUMENT;
    }
    SmoothWeights sw[3];
    if (!make_weights(sigma_x, &sw[0]) || !make_weights(sigma_y, &sw[1]) || !make_weights(sigma_z, &sw[2])) {
        report(__LINE__, __func__, "sigma too large (at most 32 voxels)");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (precision == DTB_PRECISION_FP64)
        e = smooth<double>(comps, (int) nx, (int) ny, (int) nz, sw, static_cast<const double *>(in),
                           static_cast<double *>(out), static_cast<double *>(scratch), s);
    else if (precision == DTB_PRECISION_MIXED)
        e = smooth<float>(comps, (int) nx, (int) ny, (int) nz, sw, static_cast<const float *>(in),
                          static_cast<float *>(out), static_cast<float *>(scratch), s);
    else {
        report(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        report(__LINE__, __func__, cudaGetErrorString(e));
        return DTB_ERR_CUDA;
    }
    return DTB_OK;
}

extern "C" int dtb_resample_device(int precision, int mode, int comps, size_t nx, size_t ny, size_t nz, size_t nx2,
                                   size_t ny2, size_t nz2, const void *in, void *out, void *stream) {
    disptools_clear_error();
    if (!dims_ok(nx, ny, nz) || !dims_ok(nx2, ny2, nz2) || comps < 1) {
        report(__LINE__, __func__, "invalid dimensions");
        return DTB_ERR_ARGUMENT;
    }
    if (!in || !out) {
        report(__LINE__, __func__, "null array");
        return DTB_ERR_ARGUMENT;
    }
    if (mode != DTB_RESAMPLE_LINEAR && mode != DTB_RESAMPLE_NEAREST) {
        report(__LINE__, __func__, "invalid mode");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n2 = (long long) nx2 * ny2 * nz2 * comps;
    const int grid = grid_for(n2);
    if (precision == DTB_PRECISION_FP64)
        k_resample<double><<<grid, 256, 0, s>>>(static_cast<const double *>(in), static_cast<double *>(out), (int) nx,
                                               (int) ny, (int) nz, (int) nx2, (int) ny2, (int) nz2, comps, mode);
    else if (precision == DTB_PRECISION_MIXED)
        k_resample<float><<<grid, 256, 0, s>>>(static_cast<const float *>(in), static_cast<float *>(out), (int) nx,
                                              (int) ny, (int) nz, (int) nx2, (int) ny2, (int) nz2, comps, mode);
    else {
        report(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        report(__LINE__, __func__, cudaGetErrorString(e));
        return DTB_ERR_CUDA;
    }
    return DTB_OK;
}
