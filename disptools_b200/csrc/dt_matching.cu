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

// Positions are one array of 3 n floats, f (y), g (x) and e (z) in turn, as
// are the step and the moved positions; element (q, z, y, x) lies at
// q n + (z ny + y) nx + x (below 2^32 by the entry point's size check).
struct MatchArgs {
    const float *pos;
    const float *TV;  // (nz - 1) (ny - 1) (nx - 1) cell targets
    int nx, ny, nz;
    unsigned n;  // grid points
    float eps, zeta;
};

// A trial move p - alpha dp, formed where the cost kernel stages a plane.
struct MoveArgs {
    const float *step;
    float alpha;
    float *next;  // moved positions of the points a block owns
};

// Tiles of the z-marching kernels.  A block of 256 threads covers 32
// columns along x and a few rows along y over a run of planes.  Every plane
// of positions a block needs is staged in shared memory once, for the three
// fields, as a box of 34 x (rows + 2) points with origin (x0 - 1, y0 - 1).
constexpr int MT_X = 32, MT_THREADS = 256, MB_W = MT_X + 2;
template <int TY>
struct Box {
    static constexpr int H = TY + 2, PLANE = MB_W * H, ELEMS = 3 * PLANE;
    static constexpr int PER_THREAD = (ELEMS + MT_THREADS - 1) / MT_THREADS;
};
// Cost: 32 x 8 cells per block, one per thread.
constexpr int MC_Y = 8;
using CostBox = Box<MC_Y>;
static_assert(MT_X * MC_Y == MT_THREADS, "one cell per thread");
// Gradient: 32 x 6 grid points per block; per layer the 33 x 7 cells that
// touch them (lowest corners x0 - 1 .. x0 + 31, y0 - 1 .. y0 + 5), one per
// thread.
constexpr int MG_Y = 6, MG_CX = MT_X + 1, MG_CY = MG_Y + 1, MG_CELLS = MG_CX * MG_CY;
using GradBox = Box<MG_Y>;
static_assert(MG_CELLS <= MT_THREADS, "one cell per thread");

// Corner n of a cell: bits (k, x, y) = (n >> 2, (n >> 1) & 1, n & 1), the
// reference's corner names J000 .. J111 in order (:107-115).
struct Cell {
    float J[8];
    float d[8][3][3];  // [corner][field f,g,e][axis y,x,z]
};

// Corner values X[field][corner] of the cell whose lowest corner is box
// point (bx, by) of the staged planes lo (the cell's lower plane) and hi.
template <typename B>
__device__ __forceinline__ void cell_corners(const float *lo, const float *hi, int bx, int by, float (&X)[3][8]) {
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const float *P = (n >> 2) ? hi : lo;
        const int o = (by + (n & 1)) * MB_W + bx + ((n >> 1) & 1);
#pragma unroll
        for (int q = 0; q < 3; ++q) X[q][n] = P[q * B::PLANE + o];
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

// This thread's elements of a box plane, fixed for the whole run: the
// offset q n + y nx + x of each (~0u outside the volume or the box) and
// whether the block owns its column.
template <typename B>
struct PlaneMap {
    unsigned off[B::PER_THREAD];
    unsigned own;  // bit k: element k lies in [x0, ox1) x [y0, oy1)
};

template <typename B>
__device__ __forceinline__ void plane_map(const MatchArgs &a, int x0, int y0, int ox1, int oy1, PlaneMap<B> &pm) {
    pm.own = 0u;
#pragma unroll
    for (int k = 0; k < B::PER_THREAD; ++k) {
        const int i = (int) threadIdx.x + k * MT_THREADS;
        pm.off[k] = ~0u;
        if (i < B::ELEMS) {
            const int q = i / B::PLANE, rem = i - q * B::PLANE, by = rem / MB_W, bx = rem - by * MB_W;
            const int x = x0 - 1 + bx, y = y0 - 1 + by;
            if (x >= 0 && x < a.nx && y >= 0 && y < a.ny) {
                pm.off[k] = (unsigned) q * a.n + (unsigned) (y * a.nx + x);
                if (x >= x0 && x < ox1 && y >= y0 && y < oy1) pm.own |= 1u << k;
            }
        }
    }
}

// A plane on its way to shared memory: the raw positions (and with MOVE the
// raw step) of this thread's elements, held in registers from the loads'
// issue to their commit two layers later.
template <typename B, bool MOVE>
struct PlaneRegs {
    float v[B::PER_THREAD];
    float d[MOVE ? B::PER_THREAD : 1];
};

// Issues the loads of plane z, zero outside the volume.
template <typename B, bool MOVE>
__device__ __forceinline__ void plane_issue(const MatchArgs &a, const MoveArgs &m, const PlaneMap<B> &pm, int z,
                                            PlaneRegs<B, MOVE> &r) {
    const bool zin = z >= 0 && z < a.nz;
    const unsigned zo = (unsigned) z * (unsigned) (a.nx * a.ny);
#pragma unroll
    for (int k = 0; k < B::PER_THREAD; ++k) {
        r.v[k] = 0.0f;
        if constexpr (MOVE) r.d[k] = 0.0f;
        if (zin && pm.off[k] != ~0u) {
            r.v[k] = __ldg(a.pos + (pm.off[k] + zo));
            if constexpr (MOVE) r.d[k] = __ldg(m.step + (pm.off[k] + zo));
        }
    }
}

// Stores plane z to the shared slot `pl`.  With MOVE the values stored are
// the moved positions p - alpha dp (the reference's move, :525-530, same
// rounding); those of the block's own columns also go to the next positions
// when `own` (the block owns the plane).
template <typename B, bool MOVE>
__device__ __forceinline__ void plane_commit(const MatchArgs &a, const MoveArgs &m, const PlaneMap<B> &pm, int z,
                                             bool own, const PlaneRegs<B, MOVE> &r, float *pl) {
    const unsigned zo = (unsigned) z * (unsigned) (a.nx * a.ny);
#pragma unroll
    for (int k = 0; k < B::PER_THREAD; ++k) {
        const int i = (int) threadIdx.x + k * MT_THREADS;
        if (i >= B::ELEMS) continue;
        float val = r.v[k];
        if constexpr (MOVE) {
            val = val - m.alpha * r.d[k];
            if (own && ((pm.own >> k) & 1u)) m.next[pm.off[k] + zo] = val;
        }
        pl[i] = val;
    }
}

// Cost (:81-187) of the positions, or with MOVE of the moved positions,
// which it also writes.  Block (bx, by, bz) takes the cells with lowest
// corner in [32 bx, 32 bx + 32) x [8 by, 8 by + 8) and layers
// [zc bz, zc bz + zc); each thread one column of cells, the planes staged in
// a ring of three (two more in flight) and the cell targets loaded a layer
// ahead.  Per block: the FP64 sum of the cell costs and the maximum voxel
// error |sum J - 8 V| / 8 (in float, :176-179), each in a fixed order; the
// last block to finish folds the block results in a fixed order into
// *result and resets the counter.
template <bool MOVE>
__global__ void __launch_bounds__(MT_THREADS) k_match_cost(MatchArgs a, MoveArgs m, int zc, double2 *partial,
                                                           unsigned *counter, double2 *result) {
    using B = CostBox;
    __shared__ float pl[3][B::ELEMS];
    __shared__ double rs[MT_THREADS / 32], rm[MT_THREADS / 32];
    __shared__ bool last;
    const int tid = threadIdx.x, px = tid % MT_X, py = tid / MT_X;
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const int x0 = blockIdx.x * MT_X, y0 = blockIdx.y * MC_Y, zb = blockIdx.z * zc;
    const int ze = min(zb + zc, cz);  // layers [zb, ze), planes zb .. ze
    // Points a block owns (written with MOVE): its 32 x 8 columns, the last
    // tile of a row or column also the volume's last point; planes
    // [zb, zb + zc), the last run also plane nz - 1.
    const int ox1 = x0 + MT_X >= cx ? a.nx : x0 + MT_X;
    const int oy1 = y0 + MC_Y >= cy ? a.ny : y0 + MC_Y;
    const bool last_z = ze == cz;
    auto own = [&](int z) { return z < ze || last_z; };
    const int x = x0 + px, y = y0 + py;
    const bool col = x < cx && y < cy;
    const float *tvp = a.TV + (col ? y * cx + x : 0);
    PlaneMap<B> pm;
    plane_map<B>(a, x0, y0, ox1, oy1, pm);
    // Planes zb .. ze: the first two staged now, two more in flight.
    PlaneRegs<B, MOVE> ra, rb;
    plane_issue<B, MOVE>(a, m, pm, zb, ra);
    plane_issue<B, MOVE>(a, m, pm, zb + 1, rb);
    plane_commit<B, MOVE>(a, m, pm, zb, true, ra, pl[0]);
    plane_commit<B, MOVE>(a, m, pm, zb + 1, own(zb + 1), rb, pl[1]);
    if (zb + 2 <= ze) plane_issue<B, MOVE>(a, m, pm, zb + 2, ra);
    if (zb + 3 <= ze) plane_issue<B, MOVE>(a, m, pm, zb + 3, rb);
    float tv_next = col ? __ldg(tvp + zb * cy * cx) : 0.0f;
    __syncthreads();
    double s = 0.0, mx = 0.0;
    for (int k = zb; k < ze; ++k) {
        const int t = k - zb;
        // Plane k + 2 (slot of plane k - 1, free since the last barrier)
        // from the loads issued two layers ago; plane k + 4 issued.
        if (k + 2 <= ze) plane_commit<B, MOVE>(a, m, pm, k + 2, own(k + 2), ra, pl[(t + 2) % 3]);
        ra = rb;
        if (k + 4 <= ze) plane_issue<B, MOVE>(a, m, pm, k + 4, rb);
        const float V = tv_next;
        if (col && k + 1 < ze) tv_next = __ldg(tvp + (k + 1) * cy * cx);
        if (col) {
            float X[3][8];
            cell_corners<B>(pl[t % 3], pl[(t + 1) % 3], px + 1, py + 1, X);
            Cell c;
            cell_jacobians(X, c);
            const float sJ = sum_j(c);
            float cres = 0.0f;
            if (V > 0.0f) {
                const double rr = (double) sJ - 8.0 * (double) V;
                cres = (float) ((double) cres + rr * rr);
            }
            // The barrier terms, in corner order; none when every J >= eps.
            float jmin = c.J[0];
#pragma unroll
            for (int n = 1; n < 8; ++n) jmin = fminf(jmin, c.J[n]);
            if (jmin < a.eps) {
#pragma unroll
                for (int n = 0; n < 8; ++n)
                    if (c.J[n] < a.eps) cres += a.zeta * (c.J[n] - a.eps) * (c.J[n] - a.eps);
            }
            s += 0.5 * (double) cres;
            const float err = (float) (fabs((double) (sJ - 8.0f * V)) / 8.0);
            mx = fmax(mx, (double) err);
        }
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

// The contributions of a cell to its corners: per cell edge (lo, hi) along
// an axis, both ends' terms w_c cof_c[q][axis] go + to hi and - to lo.
// FLAT: every corner has w = cE (no J below eps), so the two terms share it.
template <bool FLAT>
__device__ __forceinline__ void edge_terms(float cE, const float (&w)[8], const float (&cof)[8][3][3],
                                           float (&acc)[8][3]) {
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int bit = ax == 0 ? 1 : (ax == 1 ? 2 : 4);
#pragma unroll
        for (int lo = 0; lo < 8; ++lo) {
            if (lo & bit) continue;
            const int hi = lo | bit;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float E = FLAT ? cE * (cof[lo][q][ax] + cof[hi][q][ax])
                                     : w[lo] * cof[lo][q][ax] + w[hi] * cof[hi][q][ax];
                if (ax == 0) {
                    acc[hi][q] = E;
                    acc[lo][q] = -E;
                } else {
                    acc[hi][q] += E;
                    acc[lo][q] -= E;
                }
            }
        }
    }
}

// Gradient (:191-403) of the cost at the positions, written to `step`.
// Block (bx, by, bz) owns the grid points [32 bx, 32 bx + 32) x
// [6 by, 6 by + 6) x [zc bz, zc bz + zc).  Per layer k of cells (lowest
// corners at plane k) each thread forms the contributions of one of the
// 33 x 7 cells that touch the block's points (per corner: sum_c w_c dJ_c/dX,
// see the file comment) into shared memory; each of the first 192 threads
// then adds, for its point, the four cells' shares at their lower corners to
// the shares the layer below left at the upper corners (plane k complete, in
// a fixed order) and keeps the upper corners' shares for plane k + 1.  No
// atomics, no zeroing pass.
__global__ void __launch_bounds__(MT_THREADS) k_match_grad(MatchArgs a, int zc, float *step) {
    using B = GradBox;
    __shared__ float pl[3][B::ELEMS];
    __shared__ float cs[24][MG_CELLS];  // [corner * 3 + field][cell]
    const int tid = threadIdx.x;
    const int cx = a.nx - 1, cy = a.ny - 1, cz = a.nz - 1;
    const int x0 = blockIdx.x * MT_X, y0 = blockIdx.y * MG_Y, zb = blockIdx.z * zc;
    const int ze = min(zb + zc, a.nz);  // points' planes [zb, ze); cell layers zb - 1 .. ze - 1
    // This thread's cell column: lowest corner (i, j), box point (ccx, ccy),
    // slot cid = 33 ccy + ccx.  Warps 0-6 take the rows' first 32 cells
    // (a warp reads one box row: no bank conflicts), the first 7 lanes of
    // warp 7 the last column.
    const int ccy = tid < MG_CY * MT_X ? tid / MT_X : tid - MG_CY * MT_X;
    const int ccx = tid < MG_CY * MT_X ? tid % MT_X : MT_X;
    const int cid = ccy * MG_CX + ccx;
    const int i = x0 - 1 + ccx, j = y0 - 1 + ccy;
    const bool ccol = tid < MG_CELLS && i >= 0 && i < cx && j >= 0 && j < cy;
    const float *tvp = a.TV + (ccol ? j * cx + i : 0);
    const MoveArgs none{};
    PlaneMap<B> pm;
    plane_map<B>(a, x0, y0, 0, 0, pm);
    // Planes zb - 1 .. ze: the first two staged now, two more in flight.
    PlaneRegs<B, false> ra, rb;
    plane_issue<B, false>(a, none, pm, zb - 1, ra);
    plane_issue<B, false>(a, none, pm, zb, rb);
    plane_commit<B, false>(a, none, pm, zb - 1, false, ra, pl[0]);
    plane_commit<B, false>(a, none, pm, zb, false, rb, pl[1]);
    if (zb + 1 <= ze) plane_issue<B, false>(a, none, pm, zb + 1, ra);
    if (zb + 2 <= ze) plane_issue<B, false>(a, none, pm, zb + 2, rb);
    float tv_next = ccol && zb >= 1 ? __ldg(tvp + (zb - 1) * cy * cx) : 0.0f;
    __syncthreads();
    // This thread's point (gather phase): the first 192 threads.
    const int px = tid % MT_X, py = tid / MT_X;
    const int x = x0 + px, y = y0 + py;
    const bool gpt = py < MG_Y && x < a.nx && y < a.ny;
    float pend[3] = {0.0f, 0.0f, 0.0f};
    for (int k = zb - 1; k < ze; ++k) {
        const int t = k - (zb - 1);
        if (k + 2 <= ze) plane_commit<B, false>(a, none, pm, k + 2, false, ra, pl[(t + 2) % 3]);
        ra = rb;
        if (k + 4 <= ze) plane_issue<B, false>(a, none, pm, k + 4, rb);
        const float V = tv_next;
        if (ccol && k + 1 < cz && k + 1 < ze) tv_next = __ldg(tvp + (k + 1) * cy * cx);
        if (tid < MG_CELLS) {
            float acc[8][3];
            if (ccol && k >= 0 && k < cz) {
                float X[3][8];
                cell_corners<B>(pl[t % 3], pl[(t + 1) % 3], ccx, ccy, X);
                // Per corner the cofactors of its difference matrix
                // (dJ / d(row q, axis ax)), and J from the first row's:
                // m00 c00 + m01 c01 + m02 c02 rounds exactly as the
                // expansion in cell_jacobians (c01 is the negated minor).
                float cof[8][3][3], J[8];
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    const int ny_ = n ^ 1, nx_ = n ^ 2, nz_ = n ^ 4;
                    float mm[3][3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        mm[q][0] = (n & 1) ? X[q][n] - X[q][ny_] : X[q][ny_] - X[q][n];
                        mm[q][1] = (n & 2) ? X[q][n] - X[q][nx_] : X[q][nx_] - X[q][n];
                        mm[q][2] = (n & 4) ? X[q][n] - X[q][nz_] : X[q][nz_] - X[q][n];
                    }
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const int q1 = (q + 1) % 3, q2 = (q + 2) % 3;
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) {
                            const int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
                            cof[n][q][ax] = mm[q1][a1] * mm[q2][a2] - mm[q1][a2] * mm[q2][a1];
                        }
                    }
                    J[n] = mm[0][0] * cof[n][0][0] + mm[0][1] * cof[n][0][1] + mm[0][2] * cof[n][0][2];
                }
                float sJ = J[0], jmin = J[0];
#pragma unroll
                for (int n = 1; n < 8; ++n) {
                    sJ += J[n];
                    jmin = fminf(jmin, J[n]);
                }
                const float cE = V > 0.0f ? (float) ((double) sJ - 8.0 * (double) V) : 0.0f;
                float w[8];
#pragma unroll
                for (int n = 0; n < 8; ++n) w[n] = cE + (J[n] < a.eps ? a.zeta * (J[n] - a.eps) : 0.0f);
                // With no J below eps every corner's weight is cE, which the
                // two terms of an edge then share.
                if (jmin >= a.eps)
                    edge_terms<true>(cE, w, cof, acc);
                else
                    edge_terms<false>(cE, w, cof, acc);
            } else {
#pragma unroll
                for (int n = 0; n < 8; ++n)
#pragma unroll
                    for (int q = 0; q < 3; ++q) acc[n][q] = 0.0f;
            }
#pragma unroll
            for (int n = 0; n < 8; ++n)
#pragma unroll
                for (int q = 0; q < 3; ++q) cs[n * 3 + q][cid] = acc[n][q];
        }
        __syncthreads();
        // The point (x, y) is corner 3 of cell (px, py), corner 1 of
        // (px + 1, py), corner 2 of (px, py + 1) and corner 0 of
        // (px + 1, py + 1) at plane k; corners 7, 5, 6, 4 at plane k + 1.
        if (py < MG_Y) {
            const int c00 = py * MG_CX + px, c10 = c00 + 1, c01 = c00 + MG_CX, c11 = c01 + 1;
            const unsigned v = (unsigned) ((k * a.ny + y) * a.nx + x);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float low = cs[3 * 3 + q][c00] + cs[1 * 3 + q][c10] + cs[2 * 3 + q][c01] + cs[0 * 3 + q][c11];
                const float up = cs[7 * 3 + q][c00] + cs[5 * 3 + q][c10] + cs[6 * 3 + q][c01] + cs[4 * 3 + q][c11];
                if (k >= zb && gpt) step[(unsigned) q * a.n + v] = pend[q] + low;
                pend[q] = up;
            }
        }
        __syncthreads();
    }
}

// The move p - alpha dp (:525-530) of every grid point.
__global__ void k_match_move(const float *cur, const float *step, float alpha, float *next, long long n3) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n3;
         i += (long long) gridDim.x * blockDim.x)
        next[i] = cur[i] - alpha * step[i];
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

// Four timing events, destroyed with the object.
struct Events {
    cudaEvent_t e[4] = {};
    bool create() {
        for (cudaEvent_t &x : e)
            if (cudaEventCreate(&x) != cudaSuccess) {
                cudaGetLastError();
                x = nullptr;
                return false;
            }
        return true;
    }
    ~Events() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
};

}  // namespace

namespace {

// The solve.  J [nz][ny][nx] and field [3][nz][ny][nx] (in: the initial
// guess, out: the result) are host arrays, copied in and out, or with
// `device` device arrays used in place; the work runs on `s`.  `entry`
// names the caller in argument errors.  Returns DTB_OK or a DTB_ERR_* code.
int matching_solve(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz, const double *J,
                   const dtb_params *params, double *field, dtb_solve_stats *stats, bool device, cudaStream_t s,
                   const char *entry) {
    disptools_clear_error();
    if (!J || !field || !params) {
        report(__LINE__, entry, "null argument");
        return DTB_ERR_ARGUMENT;
    }
    if (nx < 2 || ny < 2 || nz < 2) {
        report(__LINE__, entry, "every axis needs at least 2 voxels");
        return DTB_ERR_ARGUMENT;
    }
    if (3 * nx * ny * nz >= (1ull << 32)) {
        report(__LINE__, entry, "volume too large (3 n must stay below 2^32)");
        return DTB_ERR_ARGUMENT;
    }
    if (!(dx > 0.0 && dy > 0.0 && dz > 0.0)) {
        report(__LINE__, entry, "spacing must be positive");
        return DTB_ERR_ARGUMENT;
    }
    const dtb_params &p = *params;
    const long long n = (long long) (nx * ny * nz);
    const long long cells = (long long) (nx - 1) * (ny - 1) * (nz - 1);
    DeviceBuffers b;
    // Positions (current and moved) and the gradient step, [3][n] each.
    float *cur = b.take<float>(3 * n), *next = b.take<float>(3 * n), *step = b.take<float>(3 * n);
    float *tv = b.take<float>(cells);
    double *dfield = device ? field : b.take<double>(3 * n);
    const double *dJ = device ? J : b.take<double>(n);
    // Launch shapes: 32 x 8 cell columns (cost) or 32 x 6 point columns
    // (gradient) per block, runs of zc planes, about eight blocks per SM in all.
    const int ncx = (int) nx - 1, ncy = (int) ny - 1, ncz = (int) nz - 1;
    auto zrun = [](long long tiles, int depth) {
        const long long want = 148 * 8;
        return (int) std::max<long long>(4, std::min<long long>(depth, (tiles * depth + want - 1) / want));
    };
    const int zc_cost = zrun((long long) ((ncx + MT_X - 1) / MT_X) * ((ncy + MC_Y - 1) / MC_Y), ncz);
    const int zc_grad = zrun((long long) (((int) nx + MT_X - 1) / MT_X) * (((int) ny + MG_Y - 1) / MG_Y), (int) nz);
    const dim3 cost_grid((ncx + MT_X - 1) / MT_X, (ncy + MC_Y - 1) / MC_Y, (ncz + zc_cost - 1) / zc_cost);
    const dim3 grad_grid(((int) nx + MT_X - 1) / MT_X, ((int) ny + MG_Y - 1) / MG_Y, ((int) nz + zc_grad - 1) / zc_grad);
    const int cost_blocks = (int) (cost_grid.x * cost_grid.y * cost_grid.z);
    double2 *partial = b.take<double2>(cost_blocks + 1);
    unsigned *counter = b.take<unsigned>(1);
    if (!cur || !next || !step || !tv || !dfield || !dJ || !partial || !counter) {
        report(__LINE__, __func__, "cannot allocate device buffers");
        return DTB_ERR_ALLOC;
    }
    M_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    if (!device) {
        M_CUDA(cudaMemcpyAsync(dfield, field, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
        M_CUDA(cudaMemcpyAsync(const_cast<double *>(dJ), J, n * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    k_match_prepare<<<grid_for(n), 256, 0, s>>>(dfield, dJ, (int) nx, (int) ny, (int) nz, dx, dy, dz, cur, cur + n,
                                                cur + 2 * n, tv);
    count_launch();
    M_CUDA(cudaGetLastError());

    const float eps = (float) p.delta, zeta = (float) p.zeta;
    double2 h_res;
    double max_voxel_error = DBL_MAX;
    // Profiling (dtb_set_profiling): events around the gradient and cost
    // launches, read after the host wait that follows every cost.
    Events ev;
    const bool prof = profiling_on() && ev.create();
    bool grad_timed = false;
    // Cost of the current positions (alpha < 0) or of the positions moved by
    // alpha, which are then in `next`; updates max_voxel_error like the
    // reference's global (:103, :176-179).
    auto cost = [&](float alpha, float *H) -> int {
        const MatchArgs a{cur, tv, (int) nx, (int) ny, (int) nz, (unsigned) n, eps, zeta};
        double2 *res = partial + cost_blocks;
        if (prof) M_CUDA(cudaEventRecord(ev.e[2], s));
        if (alpha < 0.0f) {
            k_match_cost<false><<<cost_grid, MT_THREADS, 0, s>>>(a, MoveArgs{}, zc_cost, partial, counter, res);
        } else {
            const MoveArgs mv{step, alpha, next};
            k_match_cost<true><<<cost_grid, MT_THREADS, 0, s>>>(a, mv, zc_cost, partial, counter, res);
        }
        count_launch();
        M_CUDA(cudaGetLastError());
        if (prof) M_CUDA(cudaEventRecord(ev.e[3], s));
        M_CUDA(cudaMemcpyAsync(&h_res, res, sizeof h_res, cudaMemcpyDeviceToHost, s));
        M_CUDA(cudaStreamSynchronize(s));
        *H = (float) h_res.x;
        max_voxel_error = h_res.y;
        if (prof) {
            float ms = 0.0f;
            if (grad_timed && cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]) == cudaSuccess)
                profile_match(PROF_MATCH_GRAD, ms);
            if (cudaEventElapsedTime(&ms, ev.e[2], ev.e[3]) == cudaSuccess) profile_match(PROF_MATCH_COST, ms);
            grad_timed = false;
        }
        return DTB_OK;
    };
    auto grads = [&]() -> int {
        const MatchArgs a{cur, tv, (int) nx, (int) ny, (int) nz, (unsigned) n, eps, zeta};
        if (prof) M_CUDA(cudaEventRecord(ev.e[0], s));
        k_match_grad<<<grad_grid, MT_THREADS, 0, s>>>(a, zc_grad, step);
        count_launch();
        M_CUDA(cudaGetLastError());
        if (prof) {
            M_CUDA(cudaEventRecord(ev.e[1], s));
            grad_timed = true;
        }
        return DTB_OK;
    };
    auto move = [&](float alpha) -> int {
        k_match_move<<<grid_for(3 * n), 256, 0, s>>>(cur, step, alpha, next, 3 * n);
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
            std::swap(cur, next);
            Hcur = Hnext;
            itnum++;
        }
    }
#undef M_DO

    // Back to displacements in the caller's layout (:777-787).
    k_match_finish<<<grid_for(n), 256, 0, s>>>(cur, cur + n, cur + 2 * n, (int) nx, (int) ny, (int) nz, dx, dy, dz,
                                               dfield);
    count_launch();
    M_CUDA(cudaGetLastError());
    if (!device) M_CUDA(cudaMemcpyAsync(field, dfield, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    M_CUDA(cudaStreamSynchronize(s));
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

}  // namespace

// volume_matching_3d with statistics, host arrays; `mask` is not used, as by
// the reference (:727).  Returns DTB_OK or a DTB_ERR_* code.
extern "C" int dtb_volume_matching(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz, const double *J,
                                   const bool *mask, const dtb_params *params, double *field,
                                   dtb_solve_stats *stats) {
    (void) mask;
    return matching_solve(nx, ny, nz, dx, dy, dz, J, params, field, stats, false, nullptr, __func__);
}

// The same on device arrays (J and field device pointers of doubles), on
// `stream`; returns once the solve is complete.
extern "C" int dtb_volume_matching_device(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                                          const double *J, const dtb_params *params, double *field,
                                          dtb_solve_stats *stats, void *stream) {
    return matching_solve(nx, ny, nz, dx, dy, dz, J, params, field, stats, true,
                          static_cast<cudaStream_t>(stream), __func__);
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
