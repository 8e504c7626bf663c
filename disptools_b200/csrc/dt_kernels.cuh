// Stencil kernels of the displacement-field generator (sm_100a).
//
// Included by dt_kernels_f32.cu (FP32 field and stencils; FMA contraction
// allowed) and dt_kernels_f64.cu (FP64; compiled with -fmad=false so the
// per-voxel arithmetic rounds exactly like the reference C library).
//
// Every kernel is a 2.5-D stencil: a block of BX x BY threads owns one x-y
// tile and marches a range of z planes, keeping a ring of planes (with an
// x-y halo) in shared memory.  Reductions are FP64 whatever the element type:
// each tile writes one partial, and the last tile of a volume to finish (an
// atomic ticket, no spinning) folds the partials in a fixed order and runs
// that volume's step control.  The result is deterministic run to run.
#pragma once

#include <cfloat>
#include <cstdint>
#include <type_traits>

#include "dt_internal.h"

namespace dtb {

enum { S_FWD = 0, S_BWD = 1, S_C2 = 2, S_C4 = 3 };

// Coefficients of src/headers/jacobian_macros.h:4-5.
template <typename T> struct FD;
template <> struct FD<double> {
    static constexpr double two_thirds = 0.666666666666666666666666666;
    static constexpr double one_twelfth = 0.083333333333333333333333333;
};
template <> struct FD<float> {
    static constexpr float two_thirds = 0.666666666666666666666666666f;
    static constexpr float one_twelfth = 0.083333333333333333333333333f;
};

// One-sided and central differences with the operation order of
// src/headers/jacobian_macros.h:7-148 (values at offsets m2 m1 0 p1 p2).
template <typename T>
__device__ __forceinline__ T fd_fwd(T a0, T p1, T p2, T ih) {
    return (T(-1.5) * a0 + T(2.0) * p1 - T(0.5) * p2) * ih;
}
template <typename T>
__device__ __forceinline__ T fd_bwd(T a0, T m1, T m2, T ih) {
    return (T(1.5) * a0 - T(2.0) * m1 + T(0.5) * m2) * ih;
}
template <typename T>
__device__ __forceinline__ T fd_c2(T p1, T m1, T ih) {
    return (p1 - m1) * ih * T(.5);
}
template <typename T>
__device__ __forceinline__ T fd_c4(T p1, T m1, T p2, T m2, T ih) {
    return ((p1 - m1) * FD<T>::two_thirds - (p2 - m2) * FD<T>::one_twelfth) * ih;
}

// det(I + a), first-row expansion as det3/det3j (src/headers/disptools.h:185-199).
template <typename T>
__device__ __forceinline__ T det_i_plus(const T a[3][3]) {
    const T a11 = a[0][0] + T(1.0), a12 = a[0][1], a13 = a[0][2];
    const T a21 = a[1][0], a22 = a[1][1] + T(1.0), a23 = a[1][2];
    const T a31 = a[2][0], a32 = a[2][1], a33 = a[2][2] + T(1.0);
    return a11 * (a22 * a33 - a23 * a32) - a12 * (a21 * a33 - a23 * a31) +
           a13 * (a21 * a32 - a22 * a31);
}

// ------------------------------------------------------------------------
// FP32 pairs.  sm_100 executes add, sub, mul and fma on the two FP32 halves
// of a 64-bit register pair as one instruction; each half rounds as the
// scalar operation does.  The FP32 stencils below state every rounding
// (no contraction left to the compiler), so the scalar and the paired forms
// give the same bits for a voxel, whichever evaluator a tile takes.
// ------------------------------------------------------------------------
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const unsigned long long *>(&a)),
          "l"(*reinterpret_cast<const unsigned long long *>(&b)));
    return *reinterpret_cast<const float2 *>(&d);
}
__device__ __forceinline__ float2 p_splat(float a) { return make_float2(a, a); }

// Fourth-order central difference of FP32 values with the spacing folded
// into the weights, k1 = 2/3 ih and k2n = -1/12 ih:
// (p1 - m1) k1 + (p2 - m2) k2n, one product and one fused multiply-add.
__device__ __forceinline__ float c4_folded(float p1, float m1, float p2, float m2, float k1, float k2n) {
    return __fmaf_rn(__fsub_rn(p1, m1), k1, __fmul_rn(__fsub_rn(p2, m2), k2n));
}
__device__ __forceinline__ float2 c4_folded2(float2 p1, float2 m1, float2 p2, float2 m2, float2 k1, float2 k2n) {
    return p_fma(p_sub(p1, m1), k1, p_mul(p_sub(p2, m2), k2n));
}
// The same with the first difference already formed.
__device__ __forceinline__ float2 c4_folded2d(float2 d1, float2 p2, float2 m2, float2 k1, float2 k2n) {
    return p_fma(d1, k1, p_mul(p_sub(p2, m2), k2n));
}

// det(I + a) in FP32, the expansion above with each rounding stated: the
// three minors as differences of products, then a11 c1 - a12 c2 and the
// last term fused.
template <>
__device__ __forceinline__ float det_i_plus<float>(const float a[3][3]) {
    const float a11 = __fadd_rn(a[0][0], 1.f), a22 = __fadd_rn(a[1][1], 1.f), a33 = __fadd_rn(a[2][2], 1.f);
    const float c1 = __fsub_rn(__fmul_rn(a22, a33), __fmul_rn(a[1][2], a[2][1]));
    const float c2 = __fsub_rn(__fmul_rn(a[1][0], a33), __fmul_rn(a[1][2], a[2][0]));
    const float c3 = __fsub_rn(__fmul_rn(a[1][0], a[2][1]), __fmul_rn(a22, a[2][0]));
    return __fmaf_rn(a[0][2], c3, __fsub_rn(__fmul_rn(a11, c1), __fmul_rn(a[0][1], c2)));
}
__device__ __forceinline__ float2 det_i_plus2(const float2 a[3][3]) {
    const float2 one = p_splat(1.f);
    const float2 a11 = p_add(a[0][0], one), a22 = p_add(a[1][1], one), a33 = p_add(a[2][2], one);
    const float2 c1 = p_sub(p_mul(a22, a33), p_mul(a[1][2], a[2][1]));
    const float2 c2 = p_sub(p_mul(a[1][0], a33), p_mul(a[1][2], a[2][0]));
    const float2 c3 = p_sub(p_mul(a[1][0], a[2][1]), p_mul(a22, a[2][0]));
    return p_fma(a[0][2], c3, p_sub(p_mul(a11, c1), p_mul(a[0][1], c2)));
}

// Scheme along each axis at voxel (x, y, z): the case analysis of
// src/jacobian.c:70-242 stated per voxel.  Outer layer: one-sided along the
// axes where the voxel is at 0 / n-1, central second order along the others.
// Otherwise central second order on the penultimate layer (or everywhere
// when order == 2), central fourth order inside.
__device__ __forceinline__ void schemes_at(int x, int y, int z, const Geom &g, int k[3]) {
    const int p[3] = {x, y, z};
    const int n[3] = {g.nx, g.ny, g.nz};
    bool outer = false, pen = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        outer |= (p[a] == 0) | (p[a] == n[a] - 1);
        pen |= (p[a] == 1) | (p[a] == n[a] - 2);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (outer)
            k[a] = p[a] == 0 ? S_FWD : (p[a] == n[a] - 1 ? S_BWD : S_C2);
        else
            k[a] = (g.order == 2 || pen) ? S_C2 : S_C4;
    }
}

__device__ __forceinline__ int ring_slot(int z, int ns) {
    int s = z % ns;
    return s < 0 ? s + ns : s;
}

// Shared-memory ring of z planes: [NS][3][PY][PX].
template <typename T, int PX, int PY>
struct Ring {
    T *base;
    __device__ __forceinline__ T &at(int slot, int c, int ly, int lx) const {
        return base[((slot * 3 + c) * PY + ly) * PX + lx];
    }
};

// Derivative of component c along axis `a` with scheme k at ring cell
// (lx, ly) of plane z (slots of z-2..z+2 in s[0..4]).
template <typename T, int PX, int PY>
__device__ __forceinline__ T ring_deriv(const Ring<T, PX, PY> &r, const int s[5], int c, int lx,
                                        int ly, int a, int k, T ih) {
    auto val = [&](int o) -> T {
        if (a == 0) return r.at(s[2], c, ly, lx + o);
        if (a == 1) return r.at(s[2], c, ly + o, lx);
        return r.at(s[2 + o], c, ly, lx);
    };
    switch (k) {
    case S_FWD: return fd_fwd<T>(val(0), val(1), val(2), ih);
    case S_BWD: return fd_bwd<T>(val(0), val(-1), val(-2), ih);
    case S_C2: return fd_c2<T>(val(1), val(-1), ih);
    default: return fd_c4<T>(val(1), val(-1), val(2), val(-2), ih);
    }
}

template <typename T, int PX, int PY>
__device__ __forceinline__ void ring_matrix(const Ring<T, PX, PY> &r, const int s[5], int lx, int ly,
                                            const int k[3], const T ih[3], T a[3][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) a[c][ax] = ring_deriv<T, PX, PY>(r, s, c, lx, ly, ax, k[ax], ih[ax]);
}

// Per-voxel error of src/headers/error.h:128-142.
template <typename T>
__device__ __forceinline__ T voxel_error(T J, T Jt, bool in_mask, T tol) {
    const T e = J - Jt;
    if (in_mask) return e;
    const T ae = fabs(e);
    return ae < tol ? T(0.0) : copysign(ae - tol, e);
}

__device__ __forceinline__ bool is_normal(double x) {
    const double a = fabs(x);
    return a >= DBL_MIN && a <= DBL_MAX;
}

// ------------------------------------------------------------------------
// Step control (one thread, FP64), the decision logic of
// src/displacement_field_gradient.c:289-416 and
// src/displacement_field_greedy.c:161-233.
// ------------------------------------------------------------------------
__device__ __forceinline__ void finish(SolverState *st, int reason) {
    st->done = 1;
    st->reason = reason;
}

__device__ __forceinline__ void log_line(SolverState *st, int kind, double E, double M) {
    if (st->log && st->log_n < st->log_cap) {
        IterLog &l = st->log[st->log_n++];
        l.it = st->it;
        l.kind = kind;
        l.pad = 0;
        l.E = E;
        l.M = M;
        l.eta = st->eta;
    }
}

__device__ inline void control_after_trial(SolverState *st, double E, double M) {
    st->E = E;
    st->M = M;
    switch (st->phase) {
    case PH_EVAL0:
        st->E0 = E;
        st->M0 = M;
        st->E_last = E;
        st->ret_E = E;
        st->ret_M = M;
        st->it = 0;
        if (st->algorithm == DTB_ALGORITHM_GRADIENT) log_line(st, 0, E, M);  // :272-277
        st->it = 1;
        if (st->algorithm == DTB_ALGORITHM_GRADIENT) {
            st->phase = PH_SEARCH;
            st->need_gradient = 1;
            st->eta *= st->alpha;  // :291
        } else {
            st->phase = PH_GREEDY;
            if (st->it_max < 1) finish(st, DTB_STOP_IT_MAX);
        }
        break;
    case PH_SEARCH:
        st->trials++;
        if (st->eta < st->eta_max && E - st->E_last > -st->gamma * st->eta * st->gn2) {  // :313
            st->eta *= st->alpha;
        } else {
            st->eta /= st->alpha * st->alpha;  // :317
            st->E_last = st->E0;               // :320-326
            st->M_last = DBL_MAX;
            st->phase = PH_MAIN;
            st->it = 1;
            if (st->it_max < 1) {
                finish(st, DTB_STOP_IT_MAX);
            } else {
                // Iteration 1 recomputes the gradient of the same field with
                // the same error map (:332-339); the stored one is identical.
                st->eta *= st->alpha;  // :342-343
                st->eta = st->eta > st->eta_max ? st->eta_max : st->eta;
            }
        }
        break;
    case PH_MAIN: {
        st->trials++;
        const bool eta_good = st->eta >= st->iota;  // :366-374
        const bool ag = E - st->E_last > -st->gamma * st->eta * st->gn2;
        const bool sc = st->strict && M > st->M_last;
        if (eta_good && (ag || sc)) {
            st->eta *= st->beta;
            break;
        }
        log_line(st, 0, E, M);  // :377-383
        if (!is_normal(E)) finish(st, DTB_STOP_ERROR_EXPLODED);  // :387-410
        else if (st->eta < st->iota) finish(st, DTB_STOP_ETA);
        else if (1.0 - E / st->E_last < st->theta) finish(st, DTB_STOP_THETA);
        else if (!is_normal(M)) finish(st, DTB_STOP_MAX_EXPLODED);
        else if (M < st->epsilon) finish(st, DTB_STOP_EPSILON);
        else {
            st->E_last = E;  // :413-415
            st->M_last = M;
            st->ret_E = E;
            st->ret_M = M;
            st->old_buf ^= 1;
            st->it++;
            if (st->it > st->it_max) {
                finish(st, DTB_STOP_IT_MAX);
            } else {
                st->need_gradient = 1;
                st->eta *= st->alpha;
                st->eta = st->eta > st->eta_max ? st->eta_max : st->eta;
            }
        }
        break;
    }
    case PH_GREEDY:
        st->trials++;
        st->v_cur ^= 1;  // the error map just written is the current one, accepted or not
        log_line(st, 0, E, M);                                    // :184-189
        if (!is_normal(E)) finish(st, DTB_STOP_ERROR_EXPLODED);  // :193-196
        else if (E >= st->E_last) {                               // :198-213
            st->eta *= st->beta;
            if (st->eta < st->iota) finish(st, DTB_STOP_ETA);
            else log_line(st, 1, E, M);
        } else if (1.0 - E / st->E_last < st->theta) finish(st, DTB_STOP_THETA);
        else if (!is_normal(M)) finish(st, DTB_STOP_MAX_EXPLODED);
        else if (M < st->epsilon) finish(st, DTB_STOP_EPSILON);
        else {
            st->E_last = E;
            st->ret_E = E;
            st->ret_M = M;
            st->old_buf ^= 1;
            st->it++;
            if (st->it > st->it_max) finish(st, DTB_STOP_IT_MAX);
        }
        break;
    }
}

// ------------------------------------------------------------------------
// Block reductions (deterministic: shuffles and a fixed tree).
// ------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Returns (sum, max) of a block of NTH threads, TXW threads wide, in thread
// 0; `red` holds 2 * NTH / 32 doubles.
template <int NTH, int TXW>
__device__ __forceinline__ double2 block_reduce_n(double s, double m, double *red) {
    static_assert(NTH <= 1024 && NTH % 32 == 0, "block size");
    const int tid = threadIdx.y * TXW + threadIdx.x;
    s = warp_sum(s);
    m = warp_max(m);
    if ((tid & 31) == 0) {
        red[tid >> 5] = s;
        red[NTH / 32 + (tid >> 5)] = m;
    }
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (tid < 32) {
        s = tid < NTH / 32 ? red[tid] : 0.0;
        m = tid < NTH / 32 ? red[NTH / 32 + tid] : 0.0;
        s = warp_sum(s);
        m = warp_max(m);
        r = make_double2(s, m);
    }
    __syncthreads();
    return r;
}

// Counts a finished tile of a volume and returns true in every thread of the
// block that finished its last one (blocks TXW threads wide).
template <int TXW>
__device__ __forceinline__ bool publish_partial_n(unsigned int *ticket, int ntiles, int *s_flag) {
    const int tid = threadIdx.y * TXW + threadIdx.x;
    if (tid == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        *s_flag = (t == (unsigned int) (ntiles - 1));
    }
    __syncthreads();
    const bool last = *s_flag;
    if (last) __threadfence();
    return last;
}

template <typename T>
__device__ __forceinline__ T ldcg(const T *p) {
    return __ldcg(p);
}
__device__ __forceinline__ int ldcg_int(const int *p) { return __ldcg(p); }

// ------------------------------------------------------------------------
// Jacobian map kernel: J = det(I + grad f) of field[0] into jout
// (src/jacobian.c:113-241), for fields in any row layout.  A block owns a
// BX x BY tile and marches bz planes with a five-plane shared ring (halo 2).
// ------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_jacobian(const VolumeDesc<T> *__restrict__ vols,
                                                 const int *__restrict__ tile_vol, int total_tiles) {
    constexpr int H = 2, PX = BX + 2 * H, PY = BY + 2 * H, NS = 5;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Ring<T, PX, PY> ring{reinterpret_cast<T *>(smem_raw)};

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;

    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const VolumeDesc<T> &V = vols[tile_vol[tile]];
        const Geom g = V.g;
        const int lt = tile - V.tile_begin;
        const int txi = lt % V.tiles_x, tyi = (lt / V.tiles_x) % V.tiles_y, tzi = lt / (V.tiles_x * V.tiles_y);
        const int x0 = txi * BX, y0 = tyi * BY, z0 = tzi * V.bz;
        const int z1 = min(z0 + V.bz, g.nz);
        const T *src = V.field[0];
        const T ih[3] = {(T) g.ih[0], (T) g.ih[1], (T) g.ih[2]};

        // Fill the ring slot of plane zq (tile + halo 2; 0 outside the volume).
        auto load_plane = [&](int zq) {
            const int slot = ring_slot(zq, NS);
            const bool zin = zq >= 0 && zq < g.nz;
            for (int i = tid; i < 3 * PY * PX; i += NT) {
                const int c = i / (PY * PX);
                const int r = i - c * (PY * PX);
                const int ly = r / PX, lx = r - ly * PX;
                const int gx = x0 - H + lx, gy = y0 - H + ly;
                T val = T(0);
                if (zin && gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny)
                    val = src[c * g.cs + (long long) zq * g.zs + (long long) gy * g.ys + gx];
                ring.at(slot, c, ly, lx) = val;
            }
        };

        for (int zq = z0 - 2; zq < z0 + 2; ++zq) load_plane(zq);

        const int x = x0 + tx, y = y0 + ty;
        const bool in_xy = x < g.nx && y < g.ny;
        for (int z = z0; z < z1; ++z) {
            load_plane(z + 2);
            __syncthreads();
            if (in_xy) {
                int k[3];
                schemes_at(x, y, z, g, k);
                const int s[5] = {ring_slot(z - 2, NS), ring_slot(z - 1, NS), ring_slot(z, NS),
                                  ring_slot(z + 1, NS), ring_slot(z + 2, NS)};
                T a[3][3];
                ring_matrix<T, PX, PY>(ring, s, tx + H, ty + H, k, ih, a);
                V.jout[(long long) z * g.zs + (long long) y * g.ys + x] = det_i_plus<T>(a);
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------
// Exact adjoint of the Jacobian stencil (for autograd).
// Pass 1: W[c][a](p) = w(p) * cof_ca(I + A(p)) * ih_a, A the stencil matrix.
// Pass 2: grad_c(q) = sum_a sum_t W[c][a](q - t e_a) * kappa(k_a(q - t e_a), t).
// W is dense, [9][nz][ny][nx] with component stride wn.
// ------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T gload_deriv(const T *f, long long o, long long s, int k, T ih) {
    switch (k) {
    case S_FWD: return fd_fwd<T>(f[o], f[o + s], f[o + 2 * s], ih);
    case S_BWD: return fd_bwd<T>(f[o], f[o - s], f[o - 2 * s], ih);
    case S_C2: return fd_c2<T>(f[o + s], f[o - s], ih);
    default: return fd_c4<T>(f[o + s], f[o - s], f[o + 2 * s], f[o - 2 * s], ih);
    }
}

template <typename T>
__global__ void k_adjoint_w(Geom g, const T *__restrict__ f, const T *__restrict__ gJ, T *__restrict__ W,
                            long long wn) {
    const long long N = (long long) g.nx * g.ny * g.nz;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < N;
         i += (long long) gridDim.x * blockDim.x) {
        const int x = (int) (i % g.nx);
        const int y = (int) ((i / g.nx) % g.ny);
        const int z = (int) (i / ((long long) g.nx * g.ny));
        int k[3];
        schemes_at(x, y, z, g, k);
        const long long o = (long long) z * g.zs + (long long) y * g.ys + x;
        const long long st[3] = {1, g.ys, g.zs};
        T m[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int a = 0; a < 3; ++a) m[c][a] = gload_deriv<T>(f + c * g.cs, o, st[a], k[a], (T) g.ih[a]) + (c == a ? T(1) : T(0));
        const T w = gJ[o];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int c0 = a == 0 ? 1 : 0, c1 = a == 2 ? 1 : 2;
                const T minor = m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0];
                const T cof = ((c + a) & 1) ? -minor : minor;
                W[(c * 3 + a) * wn + i] = w * cof * (T) g.ih[a];
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ T kappa(int k, int t) {
    switch (k) {
    case S_FWD: return t == 0 ? T(-1.5) : t == 1 ? T(2.0) : t == 2 ? T(-0.5) : T(0);
    case S_BWD: return t == 0 ? T(1.5) : t == -1 ? T(-2.0) : t == -2 ? T(0.5) : T(0);
    case S_C2: return t == 1 ? T(.5) : t == -1 ? T(-.5) : T(0);
    default:
        return t == 1 ? FD<T>::two_thirds : t == -1 ? -FD<T>::two_thirds
             : t == 2 ? -FD<T>::one_twelfth : t == -2 ? FD<T>::one_twelfth : T(0);
    }
}

// Voxel coordinates of a dense index; 32-bit division when the volume has
// fewer than 2^32 voxels (64-bit division costs several times as much).
__device__ __forceinline__ void voxel_of(long long i, const Geom &g, bool small, int q[3]) {
    if (small) {
        const unsigned u = (unsigned) i, r = u / (unsigned) g.nx;
        q[0] = (int) (u - r * (unsigned) g.nx);
        q[1] = (int) (r % (unsigned) g.ny);
        q[2] = (int) (r / (unsigned) g.ny);
    } else {
        q[0] = (int) (i % g.nx);
        q[1] = (int) ((i / g.nx) % g.ny);
        q[2] = (int) (i / ((long long) g.nx * g.ny));
    }
}

template <typename T>
__global__ void k_adjoint_gather(Geom g, const T *__restrict__ W, long long wn, T *__restrict__ out) {
    const long long N = (long long) g.nx * g.ny * g.nz;
    const bool small = N < (1ll << 32);
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < N;
         i += (long long) gridDim.x * blockDim.x) {
        int q[3];
        voxel_of(i, g, small, q);
        const int n[3] = {g.nx, g.ny, g.nz};
        const long long dstr[3] = {1, g.nx, (long long) g.nx * g.ny};  // W is dense
        T acc[3] = {T(0), T(0), T(0)};
        // At least four voxels from every face (order 4): each tap's voxel
        // uses the fourth-order central scheme on its axis, so the weights
        // are constants.  Same taps and summation order as the general path.
        const bool deep = g.order == 4 && q[0] >= 4 && q[0] <= g.nx - 5 && q[1] >= 4 && q[1] <= g.ny - 5 &&
                          q[2] >= 4 && q[2] <= g.nz - 5;
        if (deep) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int t = -2; t <= 2; ++t) {
                    if (t == 0) continue;
                    const T kp = kappa<T>(S_C4, t);
                    const long long pi = i - t * dstr[a];
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[c] += W[(c * 3 + a) * wn + pi] * kp;
                }
            const long long o = (long long) q[2] * g.zs + (long long) q[1] * g.ys + q[0];
#pragma unroll
            for (int c = 0; c < 3; ++c) out[c * g.cs + o] = acc[c];
            continue;
        }
        // The scheme of tap voxel p = q - t e_a along a (schemes_at(p)[a]):
        // p differs from q only along a, so the outer / penultimate flags of
        // the other two axes come from q once.
        bool ob[3], pb[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            ob[b] = q[b] == 0 || q[b] == n[b] - 1;
            pb[b] = q[b] == 1 || q[b] == n[b] - 2;
        }
        // One axis at a time (a rolled loop keeps few loads in flight and
        // few registers); per-axis values by selects, not array indexing.
#pragma unroll 1
        for (int a = 0; a < 3; ++a) {
            const bool o_other = (a != 0 && ob[0]) || (a != 1 && ob[1]) || (a != 2 && ob[2]);
            const bool p_other = (a != 0 && pb[0]) || (a != 1 && pb[1]) || (a != 2 && pb[2]);
            const int qa = a == 0 ? q[0] : (a == 1 ? q[1] : q[2]);
            const int na = a == 0 ? n[0] : (a == 1 ? n[1] : n[2]);
            const long long da = a == 0 ? dstr[0] : (a == 1 ? dstr[1] : dstr[2]);
            const T *w0 = W + a * wn, *w1 = W + (3 + a) * wn, *w2 = W + (6 + a) * wn;
#pragma unroll
            for (int t = -2; t <= 2; ++t) {
                const int pa = qa - t;
                if (pa < 0 || pa >= na) continue;
                const bool outer = o_other || pa == 0 || pa == na - 1;
                const bool pen = p_other || pa == 1 || pa == na - 2;
                const int k = outer ? (pa == 0 ? S_FWD : (pa == na - 1 ? S_BWD : S_C2))
                                    : ((g.order == 2 || pen) ? S_C2 : S_C4);
                const T kp = kappa<T>(k, t);
                if (kp == T(0)) continue;
                const long long pi = i - t * da;
                acc[0] += w0[pi] * kp;
                acc[1] += w1[pi] * kp;
                acc[2] += w2[pi] * kp;
            }
        }
        const long long o = (long long) q[2] * g.zs + (long long) q[1] * g.ys + q[0];
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c * g.cs + o] = acc[c];
    }
}

// ------------------------------------------------------------------------
// Element-wise helpers.
// ------------------------------------------------------------------------
template <typename T>
__global__ void k_convert(const void *__restrict__ src, int src_is_double, T *__restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x)
        dst[i] = src_is_double ? (T) static_cast<const double *>(src)[i] : (T) static_cast<const float *>(src)[i];
}

template <typename T>
__global__ void k_to_double(const T *__restrict__ src, double *__restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x)
        dst[i] = (double) src[i];
}

// src/jacobian.c:29-55
template <typename T>
__global__ void k_regularise(T *__restrict__ J, long long n, T eps) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x)
        if (J[i] < eps) J[i] = eps;
}

// ------------------------------------------------------------------------
// Launch wrappers.
// ------------------------------------------------------------------------
inline int elementwise_grid(long long n) {
    long long b = (n + 255) / 256;
    return (int) (b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

template <typename T>
cudaError_t launch_jacobian(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                            cudaStream_t s) {
    constexpr int smem = jacobian_smem_bytes<T>();
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_jacobian<T>, smem, devs);
    if (attr != cudaSuccess) return attr;
    k_jacobian<T><<<grid, dim3(BX, BY), smem, s>>>(vols, tile_vol, total_tiles);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjoint(const Geom &g, const T *field, const T *gJ, T *W, long long wn, T *gout, bool w_done,
                           cudaStream_t s) {
    const long long N = (long long) g.nx * g.ny * g.nz;
    if (!w_done) {
        k_adjoint_w<T><<<elementwise_grid(N), 256, 0, s>>>(g, field, gJ, W, wn);
        count_launch();
    }
    k_adjoint_gather<T><<<elementwise_grid(N), 256, 0, s>>>(g, W, wn, gout);
    count_launch();
    return cudaGetLastError();
}

// One thread per (row y, plane z, component): the row's two end voxels, and
// the whole row on the y and z faces.
template <typename T>
__global__ void k_boundary_nonzero(const T *__restrict__ f, Geom g, int *flag) {
    using U = typename std::conditional<sizeof(T) == 4, unsigned int, unsigned long long>::type;
    const long long rows = 3ll * g.ny * g.nz;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < rows;
         i += (long long) gridDim.x * blockDim.x) {
        const int y = (int) (i % g.ny), z = (int) ((i / g.ny) % g.nz), c = (int) (i / ((long long) g.ny * g.nz));
        const U *row = reinterpret_cast<const U *>(f + c * g.cs + (long long) z * g.zs + (long long) y * g.ys);
        U any = row[0] | row[g.nx - 1];
        if (y == 0 || y == g.ny - 1 || z == 0 || z == g.nz - 1)
            for (int x = 1; x < g.nx - 1; ++x) any |= row[x];
        if (any) *flag = 1;
    }
}

template <typename T>
cudaError_t launch_boundary_nonzero(const T *field, const Geom &g, int *flag, cudaStream_t s) {
    const long long rows = 3ll * g.ny * g.nz;
    k_boundary_nonzero<T><<<elementwise_grid(rows), 256, 0, s>>>(field, g, flag);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_convert(const void *src, int src_is_double, T *dst, long long n, cudaStream_t s) {
    k_convert<T><<<elementwise_grid(n), 256, 0, s>>>(src, src_is_double, dst, n);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_to_double(const T *src, double *dst, long long n, cudaStream_t s) {
    k_to_double<T><<<elementwise_grid(n), 256, 0, s>>>(src, dst, n);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_regularise(T *J, long long n, double eps, cudaStream_t s) {
    k_regularise<T><<<elementwise_grid(n), 256, 0, s>>>(J, n, (T) eps);
    count_launch();
    return cudaGetLastError();
}

#define DTB_INSTANTIATE(T)                                                                                   \
    template cudaError_t launch_jacobian<T>(const VolumeDesc<T> *, const int *, int, int, cudaStream_t);     \
    template cudaError_t launch_adjoint<T>(const Geom &, const T *, const T *, T *, long long, T *, bool,    \
                                           cudaStream_t);                                                    \
    template cudaError_t launch_convert<T>(const void *, int, T *, long long, cudaStream_t);                 \
    template cudaError_t launch_to_double<T>(const T *, double *, long long, cudaStream_t);                  \
    template cudaError_t launch_regularise<T>(T *, long long, double, cudaStream_t);                        \
    template cudaError_t launch_boundary_nonzero<T>(const T *, const Geom &, int *, cudaStream_t);

}  // namespace dtb
