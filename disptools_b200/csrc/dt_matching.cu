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
// float in loop order, so costs agree to float rounding.
//
// Both kernels march along z over tiles of 32 x 8 columns and stage each
// plane of positions in shared memory once.  The cost kernel forms the
// trial move p - alpha dp where it stages a plane (and writes the moved
// positions), and its last block folds the block sums.  The gradient kernel
// forms each cell's 24 contributions to its corners in shared memory; every
// grid point then adds the shares of its 8 cells in a fixed order, so the
// gradient needs no atomics and is deterministic.  The step control runs on
// the host in the reference's order; each cost evaluation returns its FP64
// sum and the maximum voxel error.  The conversions between displacements
// and positions run on the device too.
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

// A trial move p - alpha dp, formed where the cost kernel stages a plane.
struct MoveArgs {
    const float *df, *dg, *de;
    float alpha;
    float *nf, *ng, *ne;  // moved positions of the points a block owns
};

// Tiles of the z-marching kernels.  A block covers 32 x 8 columns of cells
// (cost) or of grid points (gradient) over a run of planes.  Every plane of
// positions a block needs is staged in shared memory once, for the three
// fields, as a box of 34 x 10 points with origin (x0 - 1, y0 - 1).
constexpr int MT_X = 32, MT_Y = 8, MT_THREADS = MT_X * MT_Y;
constexpr int MB_W = MT_X + 2, MB_H = MT_Y + 2, MB_PLANE = MB_W * MB_H;
constexpr int MB_ELEMS = 3 * MB_PLANE;
constexpr int MB_PER_THREAD = (MB_ELEMS + MT_THREADS - 1) / MT_THREADS;
// The gradient kernel's cells per layer: lowest corners x0 - 1 .. x0 + 31,
// y0 - 1 .. y0 + 7 (every cell that has a corner among the block's points).
constexpr int MG_CX = MT_X + 1, MG_CY = MT_Y + 1, MG_CELLS = MG_CX * MG_CY;

// Corner n of a cell: bits (k, x, y) = (n >> 2, (n >> 1) & 1, n & 1), the
// reference's corner names J000 .. J111 in order (:107-115).
struct Cell {
    float J[8];
    float d[8][3][3];  // [corner][field f,g,e][axis y,x,z]
};

// Corner values X[field][corner] of the cell whose lowest corner is box
// point (bx, by) of the staged planes lo (the cell's lower plane) and hi.
__device__ __forceinline__ void cell_corners(const float *lo, const float *hi, int bx, int by, float (&X)[3][8]) {
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const float *P = (n >> 2) ? hi : lo;
        const int o = (by + (n & 1)) * MB_W + bx + ((n >> 1) & 1);
#pragma unroll
        for (int q = 0; q < 3; ++q) X[q][n] = P[q * MB_PLANE + o];
    }
}

__device__ __forceinline__ void cell_jacobians(const float (&X)[3][8], Cell &c) {
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

// Loads plane z of the box at (x0 - 1, y0 - 1) into registers, zero outside
// the volume.  With MOVE the values are the moved positions p - alpha dp
// (the reference's move, :525-530, same rounding), and those of the points
// inside [x0, ox1) x [y0, oy1) are also written to the next-position arrays
// when `own` (the block owns the plane).
template <bool MOVE>
__device__ __forceinline__ void load_plane(const MatchArgs &a, const MoveArgs &m, int x0, int y0, int z, bool own,
                                           int ox1, int oy1, float (&r)[MB_PER_THREAD]) {
    const bool zin = z >= 0 && z < a.nz;
    const int zo = z * a.nx * a.ny;
#pragma unroll
    for (int k = 0; k < MB_PER_THREAD; ++k) {
        const int i = (int) threadIdx.x + k * MT_THREADS;
        float val = 0.0f;
        if (i < MB_ELEMS && zin) {
            const int q = i / MB_PLANE, rem = i - q * MB_PLANE, by = rem / MB_W, bx = rem - by * MB_W;
            const int x = x0 - 1 + bx, y = y0 - 1 + by;
            if (x >= 0 && x < a.nx && y >= 0 && y < a.ny) {
                const int v = zo + y * a.nx + x;
                val = __ldg((q == 0 ? a.f : (q == 1 ? a.g : a.e)) + v);
                if constexpr (MOVE) {
                    val = val - m.alpha * __ldg((q == 0 ? m.df : (q == 1 ? m.dg : m.de)) + v);
                    if (own && x >= x0 && x < ox1 && y >= y0 && y < oy1) (q == 0 ? m.nf : (q == 1 ? m.ng : m.ne))[v] = val;
                }
            }
        }
        r[k] = val;
    }
}

__device__ __forceinline__ void store_plane(float *pl, const float (&r)[MB_PER_THREAD]) {
#pragma unroll
    for (int k = 0; k < MB_PER_THREAD; ++k) {
        const int i = (int) threadIdx.x + k * MT_THREADS;
        if (i < MB_ELEMS) pl[i] = r[k];
    }
}

// Cost (:81-187) of the positions, or with MOVE of the moved positions,
// which it also writes.  Block (bx, by, bz) takes the cells with lowest
// corner in [32 bx, 32 bx + 32) x [8 by, 8 by + 8) and layers
// [zc bz, zc bz + zc); each thread one column of cells, the planes staged in
// a ring of three.  Per block: the FP64 sum of the cell costs and the
// maximum voxel error |sum J - 8 V| / 8 (in float, :176-179), each in a
// fixed order; the last block to finish folds the block results in a fixed
// order into *result and resets the counter.
template <bool MOVE>
__global__ void __launch_bounds__(MT_THREADS) k_match_cost(MatchArgs a, MoveArgs m, int zc, double2 *partial,
                                                           unsigned *counter, double2 *result) {
    __shared__ float pl[3][MB_ELEMS];
    __shared__ double rs[MT_THREADS / 32], rm[MT_THREADS / 32];
    __shared__ bool last;
    const int tid = threadIdx.x, px = tid % MT_X, py = tid / MT_X;
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const int x0 = blockIdx.x * MT_X, y0 = blockIdx.y * MT_Y, zb = blockIdx.z * zc;
    const int ze = min(zb + zc, cz);  // layers [zb, ze), planes zb .. ze
    // Points a block owns (written with MOVE): its 32 x 8 columns, the last
    // tile of a row or column also the volume's last point; planes
    // [zb, zb + zc), the last run also plane nz - 1.
    const int ox1 = x0 + MT_X >= cx ? a.nx : x0 + MT_X;
    const int oy1 = y0 + MT_Y >= cy ? a.ny : y0 + MT_Y;
    const bool last_z = ze == cz;
    float r[MB_PER_THREAD];
    load_plane<MOVE>(a, m, x0, y0, zb, true, ox1, oy1, r);
    store_plane(pl[0], r);
    load_plane<MOVE>(a, m, x0, y0, zb + 1, zb + 1 < ze || last_z, ox1, oy1, r);
    store_plane(pl[1], r);
    __syncthreads();
    double s = 0.0, mx = 0.0;
    const int x = x0 + px, y = y0 + py;
    const bool col = x < cx && y < cy;
    for (int k = zb; k < ze; ++k) {
        const int t = k - zb;
        const bool pre = k + 2 <= ze;
        if (pre) load_plane<MOVE>(a, m, x0, y0, k + 2, k + 2 < ze || last_z, ox1, oy1, r);
        if (col) {
            float X[3][8];
            cell_corners(pl[t % 3], pl[(t + 1) % 3], px + 1, py + 1, X);
            Cell c;
            cell_jacobians(X, c);
            const float sJ = sum_j(c);
            const float V = __ldg(a.TV + (k * cy + y) * cx + x);
            float cres = 0.0f;
            if (V > 0.0f) {
                const double rr = (double) sJ - 8.0 * (double) V;
                cres = (float) ((double) cres + rr * rr);
            }
#pragma unroll
            for (int n = 0; n < 8; ++n)
                if (c.J[n] < a.eps) cres += a.zeta * (c.J[n] - a.eps) * (c.J[n] - a.eps);
            s += 0.5 * (double) cres;
            const float err = (float) (fabs((double) (sJ - 8.0f * V)) / 8.0);
            mx = fmax(mx, (double) err);
        }
        if (pre) store_plane(pl[(t + 2) % 3], r);
        __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    const int w = tid >> 5, l = tid & 31;
    if (l == 0) {
        rs[w] = s;
        rm[w] = mx;
    }
    __syncthreads();
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    if (tid == 0) {
        double bs = rs[0], bm = rm[0];
        for (int i = 1; i < MT_THREADS / 32; ++i) {
            bs += rs[i];
            bm = fmax(bm, rm[i]);
        }
        partial[(blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = make_double2(bs, bm);
        __threadfence();
        last = atomicAdd(counter, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    s = 0.0;
    mx = 0.0;
    for (unsigned b = tid; b < nblocks; b += MT_THREADS) {
        const double2 p = __ldcg(partial + b);
        s += p.x;
        mx = fmax(mx, p.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    __syncthreads();
    if (l == 0) {
        rs[w] = s;
        rm[w] = mx;
    }
    __syncthreads();
    if (tid == 0) {
        double bs = rs[0], bm = rm[0];
        for (int i = 1; i < MT_THREADS / 32; ++i) {
            bs += rs[i];
            bm = fmax(bm, rm[i]);
        }
        *result = make_double2(bs, bm);
        *counter = 0u;
    }
}

// Gradient (:191-403) of the cost at the positions, written to df, dg, de.
// Block (bx, by, bz) owns the grid points [32 bx, 32 bx + 32) x
// [8 by, 8 by + 8) x [zc bz, zc bz + zc).  Per layer k of cells (lowest
// corners at plane k) it forms the contributions of the 33 x 9 cells that
// touch its points (per corner: sum_c w_c dJ_c/dX, see the file comment)
// into shared memory; each thread then adds, for its point, the four cells'
// shares at their lower corners to the shares the layer below left at the
// upper corners (plane k complete, in a fixed order) and keeps the upper
// corners' shares for plane k + 1.  No atomics, no zeroing pass.
__global__ void __launch_bounds__(MT_THREADS) k_match_grad(MatchArgs a, int zc, float *df, float *dg, float *de) {
    __shared__ float pl[3][MB_ELEMS];
    __shared__ float cs[24][MG_CELLS];  // [corner * 3 + field][cell]
    const int tid = threadIdx.x, px = tid % MT_X, py = tid / MT_X;
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const int x0 = blockIdx.x * MT_X, y0 = blockIdx.y * MT_Y, zb = blockIdx.z * zc;
    const int ze = min(zb + zc, a.nz);  // points' planes [zb, ze); cell layers zb - 1 .. ze - 1
    const MoveArgs none{};
    float r[MB_PER_THREAD];
    load_plane<false>(a, none, x0, y0, zb - 1, false, 0, 0, r);
    store_plane(pl[0], r);
    load_plane<false>(a, none, x0, y0, zb, false, 0, 0, r);
    store_plane(pl[1], r);
    __syncthreads();
    const int x = x0 + px, y = y0 + py;
    float *const out[3] = {df, dg, de};
    float pend[3] = {0.0f, 0.0f, 0.0f};
    for (int k = zb - 1; k < ze; ++k) {
        const int t = k - (zb - 1);
        const bool pre = k + 2 <= ze;
        if (pre) load_plane<false>(a, none, x0, y0, k + 2, false, 0, 0, r);
        for (int c = tid; c < MG_CELLS; c += MT_THREADS) {
            const int ccy = c / MG_CX, ccx = c - ccy * MG_CX;
            const int i = x0 - 1 + ccx, j = y0 - 1 + ccy;
            float acc[8][3];
#pragma unroll
            for (int n = 0; n < 8; ++n)
#pragma unroll
                for (int q = 0; q < 3; ++q) acc[n][q] = 0.0f;
            if (i >= 0 && i < cx && j >= 0 && j < cy && k >= 0 && k < cz) {
                float X[3][8];
                cell_corners(pl[t % 3], pl[(t + 1) % 3], ccx, ccy, X);
                Cell cl;
                cell_jacobians(X, cl);
                const float sJ = sum_j(cl);
                const float V = __ldg(a.TV + (k * cy + j) * cx + i);
                const float cE = V > 0.0f ? (float) ((double) sJ - 8.0 * (double) V) : 0.0f;
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    const float w = cE + (cl.J[n] < a.eps ? a.zeta * (cl.J[n] - a.eps) : 0.0f);
                    if (w == 0.0f) continue;
                    const float(*mm)[3] = cl.d[n];
                    // cofactors: dJ / d(row q, axis ax)
                    float cof[3][3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const int q1 = (q + 1) % 3, q2 = (q + 2) % 3;
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) {
                            const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
                            cof[q][ax] = mm[q1][a1] * mm[q2][a2] - mm[q1][a2] * mm[q2][a1];
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
            }
#pragma unroll
            for (int n = 0; n < 8; ++n)
#pragma unroll
                for (int q = 0; q < 3; ++q) cs[n * 3 + q][c] = acc[n][q];
        }
        __syncthreads();
        // The point (x, y) is corner 3 of cell (px, py), corner 1 of
        // (px + 1, py), corner 2 of (px, py + 1) and corner 0 of
        // (px + 1, py + 1) at plane k; corners 7, 5, 6, 4 at plane k + 1.
        const int c00 = py * MG_CX + px, c10 = c00 + 1, c01 = c00 + MG_CX, c11 = c01 + 1;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float low = cs[3 * 3 + q][c00] + cs[1 * 3 + q][c10] + cs[2 * 3 + q][c01] + cs[0 * 3 + q][c11];
            const float up = cs[7 * 3 + q][c00] + cs[5 * 3 + q][c10] + cs[6 * 3 + q][c01] + cs[4 * 3 + q][c11];
            if (k >= zb && x < a.nx && y < a.ny) out[q][(k * a.ny + y) * a.nx + x] = pend[q] + low;
            pend[q] = up;
        }
        if (pre) store_plane(pl[(t + 2) % 3], r);
        __syncthreads();
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

// Positions in voxel units from the initial field, and the cell targets
// from the lowest voxel of each cell (:740-756, the same roundings).
__global__ void k_match_prepare(const double *field, const double *J, int nx, int ny, int nz, double dx, double dy,
                                double dz, float *f, float *g, float *e, float *tv) {
    const long long n = (long long) nx * ny * nz;
    for (long long v = blockIdx.x * (long long) blockDim.x + threadIdx.x; v < n;
         v += (long long) gridDim.x * blockDim.x) {
        const int x = (int) (v % nx), y = (int) ((v / nx) % ny), z = (int) (v / ((long long) nx * ny));
        f[v] = (float) ((float) (y + 1) + field[1 * n + v] / dy);
        g[v] = (float) ((float) (x + 1) + field[0 * n + v] / dx);
        e[v] = (float) ((float) (z + 1) + field[2 * n + v] / dz);
        if (x + 1 < nx && y + 1 < ny && z + 1 < nz)
            tv[((long long) z * (ny - 1) + y) * (nx - 1) + x] = (float) J[v];
    }
}

// Back to displacements in the caller's layout (:777-787).
__global__ void k_match_finish(const float *f, const float *g, const float *e, int nx, int ny, int nz, double dx,
                               double dy, double dz, double *field) {
    const long long n = (long long) nx * ny * nz;
    for (long long v = blockIdx.x * (long long) blockDim.x + threadIdx.x; v < n;
         v += (long long) gridDim.x * blockDim.x) {
        const int x = (int) (v % nx), y = (int) ((v / nx) % ny), z = (int) (v / ((long long) nx * ny));
        field[0 * n + v] = (double) (g[v] - (float) (x + 1)) * dx;
        field[1 * n + v] = (double) (f[v] - (float) (y + 1)) * dy;
        field[2 * n + v] = (double) (e[v] - (float) (z + 1)) * dz;
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
    DeviceBuffers b;
    float *f = b.take<float>(n), *g = b.take<float>(n), *e = b.take<float>(n);
    float *nf = b.take<float>(n), *ng = b.take<float>(n), *ne = b.take<float>(n);
    float *df = b.take<float>(n), *dg = b.take<float>(n), *de = b.take<float>(n);
    float *tv = b.take<float>(cells);
    double *dfield = b.take<double>(3 * n), *dJ = b.take<double>(n);
    // Launch shapes: 32 x 8 columns per block, runs of zc planes, about
    // eight blocks per SM in all.
    const int ncx = (int) nx - 1, ncy = (int) ny - 1, ncz = (int) nz - 1;
    auto zrun = [](long long tiles, int depth) {
        const long long want = 148 * 8;
        return (int) std::max<long long>(4, std::min<long long>(depth, (tiles * depth + want - 1) / want));
    };
    const int zc_cost = zrun((long long) ((ncx + MT_X - 1) / MT_X) * ((ncy + MT_Y - 1) / MT_Y), ncz);
    const int zc_grad = zrun((long long) (((int) nx + MT_X - 1) / MT_X) * (((int) ny + MT_Y - 1) / MT_Y), (int) nz);
    const dim3 cost_grid((ncx + MT_X - 1) / MT_X, (ncy + MT_Y - 1) / MT_Y, (ncz + zc_cost - 1) / zc_cost);
    const dim3 grad_grid(((int) nx + MT_X - 1) / MT_X, ((int) ny + MT_Y - 1) / MT_Y, ((int) nz + zc_grad - 1) / zc_grad);
    const int cost_blocks = (int) (cost_grid.x * cost_grid.y * cost_grid.z);
    double2 *partial = b.take<double2>(cost_blocks + 1);
    unsigned *counter = b.take<unsigned>(1);
    if (!f || !g || !e || !nf || !ng || !ne || !df || !dg || !de || !tv || !dfield || !dJ || !partial || !counter) {
        report(__LINE__, __func__, "cannot allocate device buffers");
        return DTB_ERR_ALLOC;
    }
    cudaStream_t s = nullptr;
    M_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    M_CUDA(cudaMemcpy(dfield, field, 3 * n * sizeof(double), cudaMemcpyHostToDevice));
    M_CUDA(cudaMemcpy(dJ, J, n * sizeof(double), cudaMemcpyHostToDevice));
    k_match_prepare<<<grid_for(n), 256, 0, s>>>(dfield, dJ, (int) nx, (int) ny, (int) nz, dx, dy, dz, f, g, e, tv);
    count_launch();
    M_CUDA(cudaGetLastError());

    const float eps = (float) p.delta, zeta = (float) p.zeta;
    double2 h_res;
    double max_voxel_error = DBL_MAX;
    // Cost of the current positions (alpha < 0) or of the positions moved by
    // alpha, which are then in (nf, ng, ne); updates max_voxel_error like the
    // reference's global (:103, :176-179).
    auto cost = [&](float alpha, float *H) -> int {
        const MatchArgs a{f, g, e, tv, (int) nx, (int) ny, (int) nz, eps, zeta};
        double2 *res = partial + cost_blocks;
        if (alpha < 0.0f) {
            k_match_cost<false><<<cost_grid, MT_THREADS, 0, s>>>(a, MoveArgs{}, zc_cost, partial, counter, res);
        } else {
            const MoveArgs mv{df, dg, de, alpha, nf, ng, ne};
            k_match_cost<true><<<cost_grid, MT_THREADS, 0, s>>>(a, mv, zc_cost, partial, counter, res);
        }
        count_launch();
        M_CUDA(cudaGetLastError());
        M_CUDA(cudaMemcpy(&h_res, res, sizeof h_res, cudaMemcpyDeviceToHost));
        *H = (float) h_res.x;
        max_voxel_error = h_res.y;
        return DTB_OK;
    };
    auto grads = [&]() -> int {
        const MatchArgs a{f, g, e, tv, (int) nx, (int) ny, (int) nz, eps, zeta};
        k_match_grad<<<grad_grid, MT_THREADS, 0, s>>>(a, zc_grad, df, dg, de);
        count_launch();
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
    M_DO(cost(-1.0f, &Hcur));
    long long itnum = 0;
    while (itnum < maxit && alpha > 0.000000001 && max_voxel_error > p.epsilon) {
        Hmark = Hcur;
        M_DO(grads());
        M_DO(cost(alpha, &nH));  // move and cost in one pass
        float Hnext;
        if (nH < Hmark) {
            if (itnum == 0) {
                while (nH < Hmark) {
                    Hmark = nH;
                    alpha *= 2.0f;
                    M_DO(cost(alpha, &nH));
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
                M_DO(cost(alpha, &nH));
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
    k_match_finish<<<grid_for(n), 256, 0, s>>>(f, g, e, (int) nx, (int) ny, (int) nz, dx, dy, dz, dfield);
    count_launch();
    M_CUDA(cudaGetLastError());
    M_CUDA(cudaMemcpy(field, dfield, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
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
