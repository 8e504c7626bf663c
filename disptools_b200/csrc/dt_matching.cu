// The `matching` solver on the device: volume_matching_3d
// (src/VolumeMatching3D.c:689-796) with its optimiser (:408-557), cost
// (:81-187) and gradient (:191-403).
//
// Unknowns are deformed positions in voxel units: f holds the y coordinate,
// g the x coordinate and e the z coordinate of every grid point (1-based
// identity plus the displacement over the spacing, :740-750).  The cost
// runs over the cells (2 x 2 x 2 grid points, indexed by their lowest
// corner).  At each of a cell's 8 corners, J_c is the determinant of the
// differences of (f, g, e) along the three cell edges that meet there; the
// rows are the fields, the columns the axes y, x, z.  The cell costs
//     0.5 * [ (sum_c J_c - 8 V)^2  (when V > 0)  +  sum_c zeta (J_c - eps)^2 [J_c < eps] ]
// with V the target Jacobian of the cell's lowest voxel, eps = delta and
// zeta the regularisation weight.  Its gradient with respect to a corner
// value is sum_c w_c dJ_c/dX with w_c = (sum J - 8 V) [V > 0]
// + zeta (J_c - eps) [J_c < eps].  dJ_c/dX is the cofactor of the edge
// difference (a cross product of the other two field rows), with sign + at
// the upper end of the edge and - at the lower end.
//
// Arithmetic is FP32 like the reference's (this file is compiled without
// multiply-add contraction, as the reference's C is).  Each cell's cost is
// added in FP64 with a deterministic reduction, where the reference sums in
// float in loop order, so costs agree to float rounding.  The gradient
// scatters each cell's 24 contributions to its corners in 8 passes, one per
// parity class of cells: cells of one class share no grid point, so the
// passes are race-free and deterministic.  The step control runs on the host
// in the reference's order; each cost evaluation returns its FP64 sum and
// the maximum voxel error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dt_internal.h"

using namespace dtb;

namespace {

struct MatchArgs {
    const float *f, *g, *e;
    const float *TV;  // (nz - 1) (ny - 1) (nx - 1) cell targets
    int nx, ny, nz;
    float eps, zeta;
};

// Corner n of a cell: bits (k, x, y) = (n >> 2, (n >> 1) & 1, n & 1), the
// reference's corner names J000 .. J111 in order (:107-115).
__device__ __forceinline__ long long vtx(const MatchArgs &a, int i, int j, int k, int n) {
    return (long long) (k + (n >> 2)) * a.nx * a.ny + (long long) (j + (n & 1)) * a.nx + (i + ((n >> 1) & 1));
}

struct Cell {
    float J[8];
    float d[8][3][3];  // [corner][field f,g,e][axis y,x,z]
};

__device__ __forceinline__ void cell_jacobians(const MatchArgs &a, int i, int j, int k, Cell &c) {
    float X[3][8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const long long v = vtx(a, i, j, k, n);
        X[0][n] = a.f[v];
        X[1][n] = a.g[v];
        X[2][n] = a.e[v];
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const int ny_ = n ^ 1, nx_ = n ^ 2, nz_ = n ^ 4;  // neighbours along y, x, z
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            // differences in the +axis direction, whichever end n is
            c.d[n][q][0] = (n & 1) ? X[q][n] - X[q][ny_] : X[q][ny_] - X[q][n];
            c.d[n][q][1] = (n & 2) ? X[q][n] - X[q][nx_] : X[q][nx_] - X[q][n];
            c.d[n][q][2] = (n & 4) ? X[q][n] - X[q][nz_] : X[q][nz_] - X[q][n];
        }
        const float(*m)[3] = c.d[n];
        c.J[n] = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    }
}

__device__ __forceinline__ float sum_j(const Cell &c) {
    float s = c.J[0];
#pragma unroll
    for (int n = 1; n < 8; ++n) s += c.J[n];
    return s;
}

// Cost: per block, the FP64 sum of the cell costs and the maximum voxel
// error |sum J - 8 V| / 8 (in float, :176-179).
__global__ void k_match_cost(MatchArgs a, double2 *partial) {
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const long long cells = (long long) cx * cy * cz;
    double s = 0.0, mx = 0.0;
    for (long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x; t < cells;
         t += (long long) gridDim.x * blockDim.x) {
        const int i = (int) (t % cx);
        const int j = (int) ((t / cx) % cy);
        const int k = (int) (t / ((long long) cx * cy));
        Cell c;
        cell_jacobians(a, i, j, k, c);
        const float sJ = sum_j(c);
        const float V = a.TV[t];
        float cres = 0.0f;
        if (V > 0.0f) {
            const double r = (double) sJ - 8.0 * (double) V;
            cres = (float) ((double) cres + r * r);
        }
#pragma unroll
        for (int n = 0; n < 8; ++n)
            if (c.J[n] < a.eps) cres += a.zeta * (c.J[n] - a.eps) * (c.J[n] - a.eps);
        s += 0.5 * (double) cres;
        const float err = (float) (fabs((double) (sJ - 8.0f * V)) / 8.0);
        mx = fmax(mx, (double) err);
    }
    __shared__ double rs[32], rm[32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        rs[w] = s;
        rm[w] = mx;
    }
    __syncthreads();
    if (w == 0) {
        s = l < (int) (blockDim.x >> 5) ? rs[l] : 0.0;
        mx = l < (int) (blockDim.x >> 5) ? rm[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
            mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        }
        if (l == 0) partial[blockIdx.x] = make_double2(s, mx);
    }
}

// Folds the block partials in a fixed order.
__global__ void k_match_fold(const double2 *partial, int n, double2 *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0, mx = 0.0;
        for (int b = 0; b < n; ++b) {
            s += partial[b].x;
            mx = fmax(mx, partial[b].y);
        }
        *out = make_double2(s, mx);
    }
}

// Gradient: the cells of parity class `cls` (bits: i, j, k parity) add their
// contributions to df, dg, de (which start at zero).
__global__ void k_match_grad(MatchArgs a, float *df, float *dg, float *de, int cls) {
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const int px = cls & 1, py = (cls >> 1) & 1, pz = (cls >> 2) & 1;
    const int hx = (cx - px + 1) / 2, hy = (cy - py + 1) / 2, hz = (cz - pz + 1) / 2;
    const long long cells = (long long) hx * hy * hz;
    float *const out[3] = {df, dg, de};
    for (long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x; t < cells;
         t += (long long) gridDim.x * blockDim.x) {
        const int i = 2 * (int) (t % hx) + px;
        const int j = 2 * (int) ((t / hx) % hy) + py;
        const int k = 2 * (int) (t / ((long long) hx * hy)) + pz;
        Cell c;
        cell_jacobians(a, i, j, k, c);
        const float sJ = sum_j(c);
        const float V = a.TV[((long long) k * cy + j) * cx + i];
        const float cE = V > 0.0f ? (float) ((double) sJ - 8.0 * (double) V) : 0.0f;
        float acc[8][3];
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
            for (int q = 0; q < 3; ++q) acc[n][q] = 0.0f;
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const float w = cE + (c.J[n] < a.eps ? a.zeta * (c.J[n] - a.eps) : 0.0f);
            if (w == 0.0f) continue;
            const float(*m)[3] = c.d[n];
            // cofactors: dJ / d(row q, axis ax)
            float cof[3][3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int q1 = (q + 1) % 3, q2 = (q + 2) % 3;
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
                    cof[q][ax] = m[q1][a1] * m[q2][a2] - m[q1][a2] * m[q2][a1];
                }
            }
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const int bit = ax == 0 ? 1 : (ax == 1 ? 2 : 4);
                const int hi = n | bit, lo = n & ~bit;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float t2 = w * cof[q][ax];
                    acc[hi][q] += t2;
                    acc[lo][q] -= t2;
                }
            }
        }
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const long long v = vtx(a, i, j, k, n);
#pragma unroll
            for (int q = 0; q < 3; ++q) out[q][v] += acc[n][q];
        }
    }
}

__global__ void k_match_move(const float *f, const float *g, const float *e, const float *df, const float *dg,
                             const float *de, float alpha, float *nf, float *ng, float *ne, long long n) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        nf[i] = f[i] - alpha * df[i];
        ng[i] = g[i] - alpha * dg[i];
        ne[i] = e[i] - alpha * de[i];
    }
}

int grid_for(long long n) {
    const long long b = (n + 255) / 256;
    return (int) std::max<long long>(1, std::min<long long>(b, 148 * 16));
}

void report(int line, const char *function, const char *message) {
    disptools_error_state *s = disptools_get_error();
    s->error = true;
    s->line = line;
    std::snprintf(s->file, sizeof s->file, "%s", __FILE__);
    std::snprintf(s->function, sizeof s->function, "%s", function);
    std::snprintf(s->message, sizeof s->message, "%s", message);
    s->trace[0] = '\0';
}

#define M_CUDA(x)                                                   \
    do {                                                            \
        const cudaError_t e_ = (x);                                 \
        if (e_ != cudaSuccess) {                                    \
            cudaGetLastError();                                     \
            report(__LINE__, __func__, cudaGetErrorString(e_));     \
            return DTB_ERR_CUDA;                                    \
        }                                                           \
    } while (0)

struct DeviceBuffers {
    std::vector<void *> p;
    ~DeviceBuffers() {
        for (void *q : p) cudaFree(q);
    }
    template <typename U>
    U *take(size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, n * sizeof(U)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        p.push_back(q);
        return static_cast<U *>(q);
    }
};

}  // namespace

// volume_matching_3d with statistics; `mask` is not used, as by the
// reference (:727).  Returns DTB_OK or a DTB_ERR_* code.
extern "C" int dtb_volume_matching(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz, const double *J,
                                   const bool *mask, const dtb_params *params, double *field,
                                   dtb_solve_stats *stats) {
    (void) mask;
    disptools_clear_error();
    if (!J || !field || !params) {
        report(__LINE__, __func__, "null argument");
        return DTB_ERR_ARGUMENT;
    }
    if (nx < 2 || ny < 2 || nz < 2 || nx * ny * nz >= (1ull << 31)) {
        report(__LINE__, __func__, "every axis needs at least 2 voxels");
        return DTB_ERR_ARGUMENT;
    }
    if (!(dx > 0.0 && dy > 0.0 && dz > 0.0)) {
        report(__LINE__, __func__, "spacing must be positive");
        return DTB_ERR_ARGUMENT;
    }
    const dtb_params &p = *params;
    const long long n = (long long) (nx * ny * nz);
    const long long cells = (long long) (nx - 1) * (ny - 1) * (nz - 1);
    // Host preparation as in :740-756: positions from the initial field, the
    // cell targets from the lowest voxel of each cell.
    std::vector<float> h_f(n), h_g(n), h_e(n), h_tv(cells);
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                const size_t v = (z * ny + y) * nx + x;
                h_f[v] = (float) ((float) (y + 1) + field[1 * n + v] / dy);
                h_g[v] = (float) ((float) (x + 1) + field[0 * n + v] / dx);
                h_e[v] = (float) ((float) (z + 1) + field[2 * n + v] / dz);
            }
    for (size_t z = 0; z + 1 < nz; ++z)
        for (size_t y = 0; y + 1 < ny; ++y)
            for (size_t x = 0; x + 1 < nx; ++x)
                h_tv[(z * (ny - 1) + y) * (nx - 1) + x] = (float) J[(z * ny + y) * nx + x];

    DeviceBuffers b;
    float *f = b.take<float>(n), *g = b.take<float>(n), *e = b.take<float>(n);
    float *nf = b.take<float>(n), *ng = b.take<float>(n), *ne = b.take<float>(n);
    float *df = b.take<float>(n), *dg = b.take<float>(n), *de = b.take<float>(n);
    float *tv = b.take<float>(cells);
    const int cgrid = grid_for(cells);
    double2 *partial = b.take<double2>(cgrid + 1);
    if (!f || !g || !e || !nf || !ng || !ne || !df || !dg || !de || !tv || !partial) {
        report(__LINE__, __func__, "cannot allocate device buffers");
        return DTB_ERR_ALLOC;
    }
    cudaStream_t s = nullptr;
    M_CUDA(cudaMemcpy(f, h_f.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    M_CUDA(cudaMemcpy(g, h_g.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    M_CUDA(cudaMemcpy(e, h_e.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    M_CUDA(cudaMemcpy(tv, h_tv.data(), cells * sizeof(float), cudaMemcpyHostToDevice));

    const float eps = (float) p.delta, zeta = (float) p.zeta;
    double2 h_res;
    double max_voxel_error = DBL_MAX;
    // Cost of (x, y, z) positions; updates max_voxel_error like the
    // reference's global (:103, :176-179).
    auto cost = [&](const float *cf, const float *cg, const float *ce, float *H) -> int {
        MatchArgs a{cf, cg, ce, tv, (int) nx, (int) ny, (int) nz, eps, zeta};
        k_match_cost<<<cgrid, 256, 0, s>>>(a, partial);
        count_launch();
        k_match_fold<<<1, 32, 0, s>>>(partial, cgrid, partial + cgrid);
        count_launch();
        M_CUDA(cudaGetLastError());
        M_CUDA(cudaMemcpy(&h_res, partial + cgrid, sizeof h_res, cudaMemcpyDeviceToHost));
        *H = (float) h_res.x;
        max_voxel_error = h_res.y;
        return DTB_OK;
    };
    auto grads = [&]() -> int {
        M_CUDA(cudaMemsetAsync(df, 0, n * sizeof(float), s));
        M_CUDA(cudaMemsetAsync(dg, 0, n * sizeof(float), s));
        M_CUDA(cudaMemsetAsync(de, 0, n * sizeof(float), s));
        MatchArgs a{f, g, e, tv, (int) nx, (int) ny, (int) nz, eps, zeta};
        for (int cls = 0; cls < 8; ++cls) {
            k_match_grad<<<grid_for(cells / 8 + 1), 128, 0, s>>>(a, df, dg, de, cls);
            count_launch();
        }
        M_CUDA(cudaGetLastError());
        return DTB_OK;
    };
    auto move = [&](float alpha) -> int {
        k_match_move<<<grid_for(n), 256, 0, s>>>(f, g, e, df, dg, de, alpha, nf, ng, ne, n);
        count_launch();
        M_CUDA(cudaGetLastError());
        return DTB_OK;
    };
#define M_DO(x)                      \
    do {                             \
        const int rc_ = (x);         \
        if (rc_ != DTB_OK) return rc_; \
    } while (0)

    // The optimiser of :408-557.
    const long long maxit = p.it_max;
    float alpha = 1.0f, Hcur = 0.0f, Hmark, nH;
    M_DO(cost(f, g, e, &Hcur));
    long long itnum = 0;
    while (itnum < maxit && alpha > 0.000000001 && max_voxel_error > p.epsilon) {
        Hmark = Hcur;
        M_DO(grads());
        M_DO(move(alpha));
        M_DO(cost(nf, ng, ne, &nH));
        float Hnext;
        if (nH < Hmark) {
            if (itnum == 0) {
                while (nH < Hmark) {
                    Hmark = nH;
                    alpha *= 2.0f;
                    M_DO(move(alpha));
                    M_DO(cost(nf, ng, ne, &nH));
                }
                alpha *= 0.5f;
                M_DO(move(alpha));
                Hnext = Hmark;
            } else {
                Hnext = nH;
                alpha = (float) ((double) alpha * 1.05);  // float times a double constant, as in :476
            }
        } else {
            while (nH > Hmark && alpha > .000000001) {
                alpha *= 0.5f;
                M_DO(move(alpha));
                M_DO(cost(nf, ng, ne, &nH));
            }
            Hnext = nH;
        }
        if (alpha > .000000001) {
            std::swap(f, nf);
            std::swap(g, ng);
            std::swap(e, ne);
            Hcur = Hnext;
            itnum++;
        }
    }
#undef M_DO

    // Back to displacements in the caller's layout (:777-787).
    M_CUDA(cudaMemcpy(h_f.data(), f, n * sizeof(float), cudaMemcpyDeviceToHost));
    M_CUDA(cudaMemcpy(h_g.data(), g, n * sizeof(float), cudaMemcpyDeviceToHost));
    M_CUDA(cudaMemcpy(h_e.data(), e, n * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                const size_t v = (z * ny + y) * nx + x;
                field[0 * n + v] = (double) (h_g[v] - (float) (x + 1)) * dx;
                field[1 * n + v] = (double) (h_f[v] - (float) (y + 1)) * dy;
                field[2 * n + v] = (double) (h_e[v] - (float) (z + 1)) * dz;
            }
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->iterations = itnum;
        stats->error = Hcur;
        stats->max_error = max_voxel_error;
        stats->eta = alpha;
        stats->precision = DTB_PRECISION_MIXED;
        stats->reason = itnum >= maxit ? DTB_STOP_IT_MAX
                                       : (alpha > 0.000000001 ? DTB_STOP_EPSILON : DTB_STOP_ETA);
    }
    return DTB_OK;
}

// Replaces volume_matching_3d (src/VolumeMatching3D.c:689-796), computed
// on the current device.
extern "C" void volume_matching_3d(const size_t nx, const size_t ny, const size_t nz, const double dx,
                                   const double dy, const double dz, const double *J, const bool *mask,
                                   const double epsilon, const double tolerance, double eta, const double eta_max,
                                   const double alpha, const double beta, const double gamma, const double delta,
                                   const double zeta, const double theta, const double iota, const bool strict,
                                   const size_t it_max, double *field) {
    dtb_params p;
    std::memset(&p, 0, sizeof p);
    p.epsilon = epsilon;
    p.tolerance = tolerance;
    p.eta = eta;
    p.eta_max = eta_max;
    p.alpha = alpha;
    p.beta = beta;
    p.gamma = gamma;
    p.delta = delta;
    p.zeta = zeta;
    p.theta = theta;
    p.iota = iota;
    p.strict = strict;
    p.it_max = (long long) it_max;
    dtb_volume_matching(nx, ny, nz, dx, dy, dz, J, mask, &p, field, nullptr);
}
