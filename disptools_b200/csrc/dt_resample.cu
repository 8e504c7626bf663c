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
// * Smoothing (dtb_smooth_recursive_device, the pyramid's default): the
//   recursive Gaussian that ITK's SmoothingRecursiveGaussian is built on,
//   written from R. Deriche, "Recursively implementing the Gaussian and its
//   derivatives", INRIA research report 1893 (1993): per axis a fourth-order
//   causal and a fourth-order anticausal recursion with Deriche's published
//   coefficients, normalised to unit DC gain.  Each recursion starts in the
//   steady state of its border value, i.e. the volume is taken to continue
//   with its edge values (zero flux).  One thread runs one line: the
//   anticausal pass right to left into the output, then the causal pass left
//   to right adding itself.  ITK's own code is not available here, so its
//   results are not pinned; the filter is pinned by its defining properties
//   (impulse response against a sampled Gaussian, unit gain, border rule).
// * Smoothing (dtb_smooth_device, on request): a sampled Gaussian, weights
//   exp(-k^2 / (2 sigma^2)) for |k| <= ceil(4 sigma), normalised to sum 1,
//   zero-flux border (indices clamped into the volume).
//   Both filters form their sums in double with explicitly rounded
//   operations in a fixed order, so the result is a fixed function of the
//   input that a host restatement reproduces bit for bit.
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

// Coefficients of the recursive Gaussian of one axis (see the file comment):
// causal y+[i] = sum_k n[k] x[i-k] - sum_k d[k] y+[i-1-k], anticausal
// y-[i] = sum_k m[k] x[i+1+k] - sum_k d[k] y-[i+1+k] (k = 0..3); gc and ga
// the steady-state responses to a unit constant; on = 0 copies the axis.
struct Recursive {
    double n[4], m[4], d[4], gc, ga;
    int on;
};

// One axis of the recursive Gaussian: one thread per line of `len` samples
// at `stride`; lines along y and z are adjacent in x (coalesced).
template <typename T>
__global__ void k_recursive_axis(const T *__restrict__ in, T *__restrict__ out, int nx, int ny, int nz, int comps,
                                 int axis, Recursive rc) {
    const int len = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const long long stride = axis == 0 ? 1 : (axis == 1 ? (long long) nx : (long long) nx * ny);
    const long long lines = (long long) nx * ny * nz * comps / len;
    for (long long l = blockIdx.x * (long long) blockDim.x + threadIdx.x; l < lines;
         l += (long long) gridDim.x * blockDim.x) {
        long long base;
        if (axis == 0) {
            base = l * nx;
        } else if (axis == 1) {  // l = (c * nz + z) * nx + x
            const long long x = l % nx, cz = l / nx;
            base = cz * ny * (long long) nx + x;
        } else {  // l = c * ny * nx + y * nx + x
            const long long xy = l % ((long long) nx * ny), c = l / ((long long) nx * ny);
            base = c * nz * (long long) ny * nx + xy;
        }
        const T *x = in + base;
        T *y = out + base;
        if (!rc.on) {
            for (int i = 0; i < len; ++i) y[i * stride] = x[i * stride];
            continue;
        }
        // Anticausal pass, right to left, stored in the output.
        const double xe = (double) x[(long long) (len - 1) * stride];
        double xn0 = xe, xn1 = xe, xn2 = xe, xn3 = xe;
        double yn0 = __dmul_rn(xe, rc.ga), yn1 = yn0, yn2 = yn0, yn3 = yn0;
        for (int i = len - 1; i >= 0; --i) {
            double acc = __dmul_rn(rc.m[0], xn0);
            acc = __dadd_rn(acc, __dmul_rn(rc.m[1], xn1));
            acc = __dadd_rn(acc, __dmul_rn(rc.m[2], xn2));
            acc = __dadd_rn(acc, __dmul_rn(rc.m[3], xn3));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[0], yn0));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[1], yn1));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[2], yn2));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[3], yn3));
            y[(long long) i * stride] = (T) acc;
            xn3 = xn2;
            xn2 = xn1;
            xn1 = xn0;
            xn0 = (double) x[(long long) i * stride];
            yn3 = yn2;
            yn2 = yn1;
            yn1 = yn0;
            yn0 = acc;
        }
        // Causal pass, left to right, added to the stored anticausal part.
        const double x0 = (double) x[0];
        double xp0 = x0, xp1 = x0, xp2 = x0;
        double yp0 = __dmul_rn(x0, rc.gc), yp1 = yp0, yp2 = yp0, yp3 = yp0;
        for (int i = 0; i < len; ++i) {
            const double xi = (double) x[(long long) i * stride];
            double acc = __dmul_rn(rc.n[0], xi);
            acc = __dadd_rn(acc, __dmul_rn(rc.n[1], xp0));
            acc = __dadd_rn(acc, __dmul_rn(rc.n[2], xp1));
            acc = __dadd_rn(acc, __dmul_rn(rc.n[3], xp2));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[0], yp0));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[1], yp1));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[2], yp2));
            acc = __dsub_rn(acc, __dmul_rn(rc.d[3], yp3));
            T *o = y + (long long) i * stride;
            *o = (T) __dadd_rn(acc, (double) *o);
            xp2 = xp1;
            xp1 = xp0;
            xp0 = xi;
            yp3 = yp2;
            yp2 = yp1;
            yp1 = yp0;
            yp0 = acc;
        }
    }
}

// The x axis of the recursive Gaussian with coalesced memory access.  A warp
// owns 32 consecutive lines and moves them through shared memory in chunks
// of 32 samples: it loads and stores 32 consecutive samples of one line at a
// time, and each lane runs its own line's recursion over the chunk, with the
// order and roundings of k_recursive_axis (the results are the same bits).
constexpr int RX_W = 32, RX_P = RX_W + 1, RX_WARPS = 2;

template <typename T>
__global__ void __launch_bounds__(32 * RX_WARPS) k_recursive_x(const T *__restrict__ in, T *__restrict__ out, int nx,
                                                               long long lines, Recursive rc) {
    __shared__ T tiles[RX_WARPS][2][RX_W * RX_P];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T *tx = tiles[warp][0];  // input samples, [line][sample]
    T *ty = tiles[warp][1];  // output samples
    const int nchunks = (nx + RX_W - 1) / RX_W;
    // Moves chunk c0 .. c0+cn-1 of the warp's lines between global and shared memory.
    auto load = [&](T *tile, const T *src, long long l0, int c0, int cn) {
#pragma unroll 4
        for (int j = 0; j < RX_W; ++j)
            if (l0 + j < lines && lane < cn) tile[j * RX_P + lane] = src[(l0 + j) * nx + c0 + lane];
    };
    auto store = [&](const T *tile, long long l0, int c0, int cn) {
#pragma unroll 4
        for (int j = 0; j < RX_W; ++j)
            if (l0 + j < lines && lane < cn) out[(l0 + j) * nx + c0 + lane] = tile[j * RX_P + lane];
    };
    for (long long l0 = ((long long) blockIdx.x * RX_WARPS + warp) * RX_W; l0 < lines;
         l0 += (long long) gridDim.x * RX_WARPS * RX_W) {
        const long long line = l0 + lane;
        const bool live = line < lines;
        const T *row = in + (live ? line : 0) * nx;
        T *my_x = tx + lane * RX_P, *my_y = ty + lane * RX_P;
        if (!rc.on) {
            for (int c0 = 0; c0 < nx; c0 += RX_W) {
                const int cn = min(RX_W, nx - c0);
                load(tx, in, l0, c0, cn);
                __syncwarp();
                store(tx, l0, c0, cn);
                __syncwarp();
            }
            continue;
        }
        // Anticausal pass, chunks right to left, stored in the output.
        const double xe = live ? (double) row[nx - 1] : 0.0;
        double xn0 = xe, xn1 = xe, xn2 = xe, xn3 = xe;
        double yn0 = __dmul_rn(xe, rc.ga), yn1 = yn0, yn2 = yn0, yn3 = yn0;
        for (int ch = nchunks - 1; ch >= 0; --ch) {
            const int c0 = ch * RX_W, cn = min(RX_W, nx - c0);
            load(tx, in, l0, c0, cn);
            __syncwarp();
            if (live)
                for (int i = cn - 1; i >= 0; --i) {
                    double acc = __dmul_rn(rc.m[0], xn0);
                    acc = __dadd_rn(acc, __dmul_rn(rc.m[1], xn1));
                    acc = __dadd_rn(acc, __dmul_rn(rc.m[2], xn2));
                    acc = __dadd_rn(acc, __dmul_rn(rc.m[3], xn3));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[0], yn0));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[1], yn1));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[2], yn2));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[3], yn3));
                    my_y[i] = (T) acc;
                    xn3 = xn2;
                    xn2 = xn1;
                    xn1 = xn0;
                    xn0 = (double) my_x[i];
                    yn3 = yn2;
                    yn2 = yn1;
                    yn1 = yn0;
                    yn0 = acc;
                }
            __syncwarp();
            store(ty, l0, c0, cn);
            __syncwarp();
        }
        // Causal pass, chunks left to right, added to the stored anticausal part.
        const double x0 = live ? (double) row[0] : 0.0;
        double xp0 = x0, xp1 = x0, xp2 = x0;
        double yp0 = __dmul_rn(x0, rc.gc), yp1 = yp0, yp2 = yp0, yp3 = yp0;
        for (int ch = 0; ch < nchunks; ++ch) {
            const int c0 = ch * RX_W, cn = min(RX_W, nx - c0);
            load(tx, in, l0, c0, cn);
            load(ty, out, l0, c0, cn);
            __syncwarp();
            if (live)
                for (int i = 0; i < cn; ++i) {
                    const double xi = (double) my_x[i];
                    double acc = __dmul_rn(rc.n[0], xi);
                    acc = __dadd_rn(acc, __dmul_rn(rc.n[1], xp0));
                    acc = __dadd_rn(acc, __dmul_rn(rc.n[2], xp1));
                    acc = __dadd_rn(acc, __dmul_rn(rc.n[3], xp2));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[0], yp0));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[1], yp1));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[2], yp2));
                    acc = __dsub_rn(acc, __dmul_rn(rc.d[3], yp3));
                    my_y[i] = (T) __dadd_rn(acc, (double) my_y[i]);
                    xp2 = xp1;
                    xp1 = xp0;
                    xp0 = xi;
                    yp3 = yp2;
                    yp2 = yp1;
                    yp1 = yp0;
                    yp0 = acc;
                }
            __syncwarp();
            store(ty, l0, c0, cn);
            __syncwarp();
        }
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

// Deriche's fourth-order approximation of the Gaussian (INRIA RR-1893,
// 1993): for x >= 0 and unit sigma,
//   g(x) ~ (a0 cos(w0 x) + a1 sin(w0 x)) exp(-b0 x) + (c0 cos(w1 x) + c1 sin(w1 x)) exp(-b1 x).
// The recursions' numerators and denominator are the z-transforms of the
// causal part of g (two damped cosines) and of its mirror image; they are
// scaled so that the impulse response sums to 1.
constexpr double DERICHE_A0 = 1.680, DERICHE_A1 = 3.735, DERICHE_B0 = 1.783, DERICHE_W0 = 0.6318;
constexpr double DERICHE_C0 = -0.6803, DERICHE_C1 = -0.2598, DERICHE_B1 = 1.723, DERICHE_W1 = 1.997;
constexpr double RECURSIVE_MAX_SIGMA = 256.0;

bool recursive_coefficients(double sigma, Recursive *rc) {
    std::memset(rc, 0, sizeof *rc);
    if (!(sigma > 0.0)) return true;  // no smoothing along this axis
    if (!(sigma <= RECURSIVE_MAX_SIGMA)) return false;
    const double a0 = DERICHE_A0, a1 = DERICHE_A1, b0 = DERICHE_B0, w0 = DERICHE_W0;
    const double c0 = DERICHE_C0, c1 = DERICHE_C1, b1 = DERICHE_B1, w1 = DERICHE_W1;
    const double eb0 = std::exp(-b0 / sigma), eb1 = std::exp(-b1 / sigma);
    const double cw0 = std::cos(w0 / sigma), sw0 = std::sin(w0 / sigma);
    const double cw1 = std::cos(w1 / sigma), sw1 = std::sin(w1 / sigma);
    const double n0 = a0 + c0;
    const double n1 = eb1 * (c1 * sw1 - (c0 + 2.0 * a0) * cw1) + eb0 * (a1 * sw0 - (2.0 * c0 + a0) * cw0);
    const double n2 = (2.0 * eb0 * eb1 * ((a0 + c0) * cw1 * cw0 - a1 * cw1 * sw0 - c1 * cw0 * sw1) +
                       c0 * eb0 * eb0 + a0 * eb1 * eb1);
    const double n3 = eb1 * eb0 * eb0 * (c1 * sw1 - c0 * cw1) + eb0 * eb1 * eb1 * (a1 * sw0 - a0 * cw0);
    const double d1 = -2.0 * eb1 * cw1 - 2.0 * eb0 * cw0;
    const double d2 = 4.0 * cw1 * cw0 * eb0 * eb1 + eb1 * eb1 + eb0 * eb0;
    const double d3 = -2.0 * cw0 * eb0 * eb1 * eb1 - 2.0 * cw1 * eb1 * eb0 * eb0;
    const double d4 = eb0 * eb0 * eb1 * eb1;
    const double m1 = n1 - d1 * n0, m2 = n2 - d2 * n0, m3 = n3 - d3 * n0, m4 = -d4 * n0;
    const double den = 1.0 + d1 + d2 + d3 + d4;
    const double gain = (n0 + n1 + n2 + n3 + m1 + m2 + m3 + m4) / den;
    const double n[4] = {n0 / gain, n1 / gain, n2 / gain, n3 / gain};
    const double m[4] = {m1 / gain, m2 / gain, m3 / gain, m4 / gain};
    const double d[4] = {d1, d2, d3, d4};
    for (int k = 0; k < 4; ++k) {
        rc->n[k] = n[k];
        rc->m[k] = m[k];
        rc->d[k] = d[k];
    }
    rc->gc = (n[0] + n[1] + n[2] + n[3]) / den;
    rc->ga = (m[0] + m[1] + m[2] + m[3]) / den;
    rc->on = 1;
    return true;
}

template <typename T>
cudaError_t smooth_recursive(int comps, int nx, int ny, int nz, const Recursive (&rc)[3], const T *in, T *out,
                             T *scratch, cudaStream_t s) {
    const long long n = (long long) nx * ny * nz * comps;
    const long long xlines = n / nx;
    const long long xblocks = (xlines + 32 * RX_WARPS - 1) / (32 * RX_WARPS);
    k_recursive_x<T><<<(int) std::min<long long>(xblocks, 1 << 20), 32 * RX_WARPS, 0, s>>>(in, out, nx, xlines,
                                                                                            rc[0]);
    count_launch();
    k_recursive_axis<T><<<grid_for(n / ny), 256, 0, s>>>(out, scratch, nx, ny, nz, comps, 1, rc[1]);
    count_launch();
    k_recursive_axis<T><<<grid_for(n / nz), 256, 0, s>>>(scratch, out, nx, ny, nz, comps, 2, rc[2]);
    count_launch();
    return cudaGetLastError();
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

extern "C" int dtb_smooth_recursive_device(int precision, int comps, size_t nx, size_t ny, size_t nz,
                                           double sigma_x, double sigma_y, double sigma_z, const void *in,
                                           void *out, void *scratch, void *stream) {
    disptools_clear_error();
    if (!dims_ok(nx, ny, nz) || comps < 1) {
        report(__LINE__, __func__, "invalid dimensions");
        return DTB_ERR_ARGUMENT;
    }
    if (!in || !out || !scratch) {
        report(__LINE__, __func__, "null array");
        return DTB_ERR_ARGUMENT;
    }
    Recursive rc[3];
    if (!recursive_coefficients(sigma_x, &rc[0]) || !recursive_coefficients(sigma_y, &rc[1]) ||
        !recursive_coefficients(sigma_z, &rc[2])) {
        report(__LINE__, __func__, "sigma too large (at most 256 voxels)");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (precision == DTB_PRECISION_FP64)
        e = smooth_recursive<double>(comps, (int) nx, (int) ny, (int) nz, rc, static_cast<const double *>(in),
                                     static_cast<double *>(out), static_cast<double *>(scratch), s);
    else if (precision == DTB_PRECISION_MIXED)
        e = smooth_recursive<float>(comps, (int) nx, (int) ny, (int) nz, rc, static_cast<const float *>(in),
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
