// TMA-pipelined kernels of the solvers (sm_100a).
//
// Both kernels march a TXW x TT_Y tile through its z range.  One elected thread streams one box per input per plane into a ring
// of shared-memory stages with cp.async.bulk.tensor, completion tracked by an
// mbarrier per stage; the other threads issue no global loads for the stencil
// inputs.  Boxes start 4 voxels left of the tile so the innermost TMA
// coordinate stays 16-byte aligned; planes outside the volume arrive
// zero-filled.
//
// k_trial_tma     candidate = field[old] - eta * grad, formed once per plane
//                 in shared memory and written to field[1-old]; each thread
//                 keeps its own two columns of candidate values (five planes)
//                 in registers for the z differences, so shared memory holds
//                 three candidate planes.  Jacobian, masked error, regularised
//                 error e' per voxel; FP64 partials and the on-device step
//                 control in the last tile.  Instantiated with GREEDY, it is
//                 the greedy method's trial (error-map update, error map
//                 stored instead of e').
// k_gradient_tma  g = sum_k +-ih_k (P_ik(p - e_k) - P_ik(p + e_k)) with
//                 P_ik = e' * minor_ik(I + grad u) (second-order central
//                 differences, src/displacement_field_gradient.c:26-145),
//                 from field[old] and the stored e' of that field.
#pragma once

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "dt_kernels.cuh"
#include "dt_tma.cuh"

namespace dtb {

constexpr int TMA_HX = 4;                  // x halo of the boxes (16-byte aligned start)
constexpr int TMA_HY = 2;                  // y halo
constexpr int TMA_PY = TT_Y + 2 * TMA_HY;  // 20

// Box geometry of a tile TXW voxels wide: TXW + 8 by TT_Y + 4 per plane.
template <int TXW>
struct Box {
    static constexpr int PX = TXW + 2 * TMA_HX;
    static constexpr int PLANE = TMA_PY * PX;  // elements of one component plane
};

template <typename T, int TXW, bool GREEDY = false>
struct TrialTmaLayout {
    static constexpr int TMA_PX = Box<TXW>::PX;
    static constexpr int TMA_PLANE = Box<TXW>::PLANE;
    static constexpr int S = 3;  // pipeline stages
    // Candidate planes in shared memory: z (read by the stencil), z+1, z+2,
    // and the one being formed, so forming the next plane needs no barrier
    // against the current stencil reads.
    static constexpr int R = 4;
    static constexpr int U_BYTES = 3 * TMA_PLANE * (int) sizeof(T);
    // Greedy method: the error map, one plane per iteration, one row wider
    // on each y side than the field box (the update reads v(p +- e_k)), into
    // a ring of RV planes of its own: forming candidate plane q reads the
    // planes q-1, q, q+1 loaded by the last three iterations, and loads run
    // S iterations ahead.  The gradient method's stage holds the g box.
    static constexpr int VPY = TMA_PY + 2;
    static constexpr int V_PLANE = VPY * TMA_PX;
    static constexpr int V_BYTES = V_PLANE * (int) sizeof(T);
    static constexpr int V_SLOT = (V_BYTES + 127) / 128 * 128;
    static constexpr int RV = S + 2;
    static constexpr int G_BYTES = GREEDY ? 0 : U_BYTES;
    static constexpr int JT_BYTES = TXW * TT_Y * (int) sizeof(T);
    static constexpr int MASK_BYTES = TXW * TT_Y;
    static constexpr int JT_OFF = U_BYTES + G_BYTES;
    static constexpr int MASK_OFF = JT_OFF + JT_BYTES;
    static constexpr int STAGE_BYTES = MASK_OFF + MASK_BYTES;  // u, g (or v), Jt, mask
    static_assert(STAGE_BYTES % 128 == 0, "stages stay 128-byte aligned");
    static constexpr int RING_OFF = S * STAGE_BYTES;
    static constexpr int VRING_OFF = RING_OFF + R * U_BYTES;
    static constexpr int BAR_OFF = VRING_OFF + (GREEDY ? RV * V_SLOT : 0);
    static constexpr int BYTES = BAR_OFF + S * 8;
};

template <typename T, int TXW>
struct GradTmaLayout {
    static constexpr int TMA_PX = Box<TXW>::PX;
    static constexpr int TMA_PLANE = Box<TXW>::PLANE;
    static constexpr int S = sizeof(T) == 4 ? 5 : 4;  // stages double as the plane ring (u, e')
    static constexpr int U_BYTES = 3 * TMA_PLANE * (int) sizeof(T);
    static constexpr int E_BYTES = TMA_PLANE * (int) sizeof(T);
    static constexpr int STAGE_BYTES = U_BYTES + E_BYTES;
    static constexpr int PXP = TXW + 4, PYP = TT_Y + 2;  // P terms: tile + 1 each side, pair-aligned columns
    static constexpr int NP = 3;  // planes of P_x, P_y terms (one barrier per plane)
    static constexpr int P_OFF = S * STAGE_BYTES;  // P_x, P_y terms: [NP][6][PYP][PXP]
    static constexpr int P_BYTES = NP * 6 * PYP * PXP * (int) sizeof(T);
    static constexpr int BAR_OFF = P_OFF + P_BYTES;
    static constexpr int BYTES = BAR_OFF + S * 8;
};

// Takes the next tile of a persistent launch (-1 when none is left; the
// block is then counted out and the last one resets the queue).  BDX is the
// block's x dimension.
template <int BDX>
__device__ __forceinline__ int take_tile(TileQueue *q, int total, int *s_tile) {
    const int tid = threadIdx.y * BDX + threadIdx.x;
    __syncthreads();  // everyone has read the previous s_tile
    if (tid == 0) {
        int t = (int) atomicAdd(&q->next, 1u);
        if (t >= total) {
            t = -1;
            __threadfence();
            if (atomicAdd(&q->exited, 1u) == gridDim.x - 1) {
                q->next = 0;
                q->exited = 0;
                __threadfence();
            }
        }
        *s_tile = t;
    }
    __syncthreads();
    return *s_tile;
}

// TMA destinations must be 128-byte aligned in the shared window; the launch
// asks for 128 spare bytes.
__device__ __forceinline__ unsigned char *align_smem_128(unsigned char *p) {
    const uint32_t a = smem_u32(p);
    return p + ((128u - (a & 127u)) & 127u);
}

// Records a lost transfer: the volume stops with an error flag that the host
// reports, and the calling thread waits (bounded) for the transfers of
// iterations [from, to) that were issued but not consumed, so none lands in
// shared memory after the block has left.
template <int S>
__device__ __forceinline__ void tma_fault(SolverState *st, uint64_t *bars, uint32_t kbase, int from, int to) {
    atomicExch(&st->fault, 1);
    atomicExch(&st->done, 1);
    for (int j = from; j < to; ++j) {
        const uint32_t k = kbase + j;
        mbar_wait_bounded(&bars[k % S], (k / S) & 1u, 1u << 16);
    }
}

// Two voxels adjacent in x, loaded or stored as one 8-byte (float) or
// 16-byte (double) access.
template <typename T>
struct PairOf;
template <>
struct PairOf<float> {
    using type = float2;
};
template <>
struct PairOf<double> {
    using type = double2;
};
template <typename T>
__device__ __forceinline__ typename PairOf<T>::type ld_pair(const T *p) {
    return *reinterpret_cast<const typename PairOf<T>::type *>(p);
}
template <typename T>
__device__ __forceinline__ void st_pair(T *p, T a, T b) {
    typename PairOf<T>::type v;
    v.x = a;
    v.y = b;
    *reinterpret_cast<typename PairOf<T>::type *>(p) = v;
}

// 16 bytes of consecutive elements.
template <typename T>
using Vec16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;

// Greedy candidate of plane q over the field box `ub`, written to `out`
// (both [3][TMA_PY][PX]):
// * interior voxels: u + dd_k (v(p + e_k) - v(p - e_k))
//   (src/displacement_field_greedy.c:30-63, same operation order);
// * other voxels of the volume: the new field buffer's own content, which
//   greedy_prefetch_stale has already copied into `out` (the caller waits
//   for its own copies first), or +0 when `stale_zero` says that content is
//   +0 everywhere on the boundary;
// * outside the volume: 0 (the field box arrives zero-filled there).
// `vm`, `vc`, `vn` are the error map's planes q-1, q, q+1, rows
// y0-3 .. y0+TT_Y+2, columns as in the field box.  A thread forms the three components of one
// 16-byte run of x with vector reads; a run that is not all interior picks
// each voxel's value by its class.  Values formed at non-interior voxels
// (from zero-filled or clamped neighbours) are discarded.  The box's first
// and last columns lack an x neighbour; no stencil reads them.
template <typename T, typename L>
__device__ __forceinline__ void greedy_form(const T *ub, const T *vm, const T *vc, const T *vn, T *out, int tid,
                                            int nth, const Geom &g, int x0, int y0, int q, const T *dd,
                                            bool stale_zero) {
    using V4 = Vec16<T>;
    constexpr int VEC = 16 / (int) sizeof(T);
    constexpr int PX = L::TMA_PX, UP = L::TMA_PLANE;
    constexpr int CPR = PX / VEC, NPOS = TMA_PY * CPR;  // runs per row, per plane
    static_assert(PX % VEC == 0, "rows split in whole runs");
    const bool q_in = q >= 1 && q <= g.nz - 2;
    const bool q_vol = q >= 0 && q < g.nz;
    auto ld = [](const T *p) { return *reinterpret_cast<const V4 *>(p); };
    auto el = [](const V4 &v, int e) { return reinterpret_cast<const T *>(&v)[e]; };
    for (int i = nth - 1 - tid; i < NPOS; i += nth) {  // as greedy_prefetch_stale
        const int ly = i / CPR;
        const int lxc = (i - ly * CPR) * VEC;
        const int gy = y0 - TMA_HY + ly, gx = x0 - TMA_HX + lxc;
        const int o = ly * PX + lxc;           // run offset in a field-box plane
        const int vo = (ly + 1) * PX + lxc;    // the same run in an error-map plane
        const T *vp = vc + vo;                 // v at the run's voxels
        const bool row_in = q_in && gy >= 1 && gy <= g.ny - 2;
        const bool all_in = row_in && gx >= 1 && gx + VEC - 1 <= g.nx - 2;
        // Classes of the run's voxels: formed (interior) or kept (the
        // prefetched stale value); the others keep the zero of the box.
        unsigned formed_m = 0, keep_m = 0;
        if (!all_in) {
            const bool yz_vol = q_vol && gy >= 0 && gy < g.ny;
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const int x = gx + e;
                const bool interior = row_in && x >= 1 && x <= g.nx - 2;
                formed_m |= (unsigned) interior << e;
                keep_m |= (unsigned) (yz_vol && x >= 0 && x < g.nx && !interior) << e;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T hi[VEC], lo[VEC];
            if (c == 0) {
                const V4 cur = ld(vp);
                const V4 prv = lxc >= VEC ? ld(vp - VEC) : cur;
                const V4 nxt = lxc + VEC < PX ? ld(vp + VEC) : cur;
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    hi[e] = e + 1 < VEC ? el(cur, e + 1) : el(nxt, 0);
                    lo[e] = e > 0 ? el(cur, e - 1) : el(prv, VEC - 1);
                }
            } else {
                const V4 h = c == 1 ? ld(vp + PX) : ld(vn + vo), l = c == 1 ? ld(vp - PX) : ld(vm + vo);
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    hi[e] = el(h, e);
                    lo[e] = el(l, e);
                }
            }
            const T ddc = dd[c];
            V4 a = ld(ub + c * UP + o);
            T *pa = reinterpret_cast<T *>(&a);
            // u + dd (v(+) - v(-)); FP32 as one fused multiply-add (in pairs
            // when the whole run is formed), FP64 in the reference's order.
            auto upd = [&](T u, T h, T l) -> T {
                if constexpr (sizeof(T) == 4) return __fmaf_rn(ddc, __fsub_rn(h, l), u);
                else return u + ddc * (h - l);
            };
            if (all_in) {
                if constexpr (sizeof(T) == 4) {
                    const float2 dd2 = p_splat(ddc);
                    const float2 a01 = p_fma(dd2, p_sub(make_float2(hi[0], hi[1]), make_float2(lo[0], lo[1])),
                                             make_float2(pa[0], pa[1]));
                    const float2 a23 = p_fma(dd2, p_sub(make_float2(hi[2], hi[3]), make_float2(lo[2], lo[3])),
                                             make_float2(pa[2], pa[3]));
                    a = make_float4(a01.x, a01.y, a23.x, a23.y);
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) pa[e] = upd(pa[e], hi[e], lo[e]);
                }
            } else {
                V4 old;
                if (stale_zero) {
                    T *po = reinterpret_cast<T *>(&old);
#pragma unroll
                    for (int e = 0; e < VEC; ++e) po[e] = T(0);
                } else {
                    old = ld(out + c * UP + o);
                }
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    const T f = upd(pa[e], hi[e], lo[e]);
                    pa[e] = (formed_m >> e) & 1u ? f : ((keep_m >> e) & 1u ? el(old, e) : pa[e]);
                }
            }
            *reinterpret_cast<V4 *>(out + c * UP + o) = a;
        }
    }
}

// Copies, for the runs greedy_form gives this thread, the new field
// buffer's content at the volume's boundary voxels of plane q into `out` (the
// candidate plane q's ring slot), asynchronously: issued one plane ahead, the
// loads overlap the current plane's work.  Boundary voxels are never written
// by the greedy update, so `dst` holds constant values there.
template <typename T, typename L>
__device__ __forceinline__ void greedy_prefetch_stale(T *out, int tid, int nth, const Geom &g, int x0, int y0, int q,
                                                      const T *dst) {
    constexpr int VEC = 16 / (int) sizeof(T);
    constexpr int PX = L::TMA_PX, UP = L::TMA_PLANE;
    constexpr int CPR = PX / VEC, NPOS = TMA_PY * CPR;
    if (q < 0 || q >= g.nz) return;
    const bool q_in = q >= 1 && q <= g.nz - 2;
    // A box of interior voxels only has no stale values.
    if (q_in && x0 - TMA_HX >= 1 && x0 - TMA_HX + PX - 1 <= g.nx - 2 && y0 - TMA_HY >= 1 &&
        y0 - TMA_HY + TMA_PY - 1 <= g.ny - 2)
        return;
    // Runs counted from the last thread (the first threads' warp issues the
    // loads), the same mapping as greedy_form.
    for (int i = nth - 1 - tid; i < NPOS; i += nth) {
        const int ly = i / CPR;
        const int lxc = (i - ly * CPR) * VEC;
        const int gy = y0 - TMA_HY + ly, gx = x0 - TMA_HX + lxc;
        if (gy < 0 || gy >= g.ny) continue;
        const bool row_in = q_in && gy >= 1 && gy <= g.ny - 2;
        if (row_in && gx >= 1 && gx + VEC - 1 <= g.nx - 2) continue;  // all interior
        const int o = ly * PX + lxc;
        const T *drow = dst + (long long) q * g.zs + (long long) gy * g.ys + gx;
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            const int x = gx + e;
            if (x < 0 || x >= g.nx || (row_in && x >= 1 && x <= g.nx - 2)) continue;
#pragma unroll
            for (int c = 0; c < 3; ++c) cp_async_elem<(int) sizeof(T)>(out + c * UP + o + e, drow + c * g.cs + e);
        }
    }
    cp_async_commit();
}

// The Jacobian matrices minus I of the two voxels (x, x + 1) of row y of
// plane ze, each handed to finish(v, a) when the voxel lies in the volume.
// `jp` is the plane's field box in shared memory ([3][TMA_PY][PX], column lx
// holds x, row ly holds y); zq holds the two columns' values of planes
// ze-2 .. ze+2 per component as pairs (x, x + 1).  FP32 folds the spacing into the fourth-order
// weights; the FP64 path keeps the reference's operation order.  Three
// evaluators:
// * rows and planes inside [2, n-3] of a tile whose columns all lie inside
//   [2, nx-3] use the fourth-order stencil only;
// * interior rows of a tile that reaches an x end select the scheme per
//   voxel without branching;
// * rows or planes on the two outer layers take the general path.
// The trial kernel keeps the same evaluator inline: calling this function
// there changes its register allocation (it then spills).  In FP32, a
// `finish2` functor (not null) takes the first evaluator's two matrices at
// once, as pairs (x, x + 1) of each entry.
template <typename T, int TMA_PX, int TMA_PLANE, typename F, typename F2 = std::nullptr_t>
__device__ __forceinline__ void stencil_pair(const typename PairOf<T>::type (&zq)[3][5], const T *jp, int lx,
                                             int ly, int x, int y,
                                             int ze, const Geom &g, const T (&ih)[3], bool row_in,
                                             bool tile_x_in, F &&finish, F2 &&finish2 = nullptr) {
    const T k1[3] = {FD<T>::two_thirds * ih[0], FD<T>::two_thirds * ih[1], FD<T>::two_thirds * ih[2]};
    const T k2n[3] = {-FD<T>::one_twelfth * ih[0], -FD<T>::one_twelfth * ih[1], -FD<T>::one_twelfth * ih[2]};
    auto c4 = [&](T p1, T m1, T p2, T m2, int ax) -> T {
        if constexpr (sizeof(T) == 4) return c4_folded(p1, m1, p2, m2, k1[ax], k2n[ax]);
        return fd_c4<T>(p1, m1, p2, m2, ih[ax]);
    };
    constexpr bool PAIRED = sizeof(T) == 4 && !std::is_same<typename std::decay<F2>::type, std::nullptr_t>::value;
    if constexpr (PAIRED) {
        if (row_in && tile_x_in) {
            float2 a[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx;
                const float2 xm = ld_pair(p - 2), xc = ld_pair(p), xp = ld_pair(p + 2);
                const float2 dx1 = make_float2(__fsub_rn(xc.y, xm.y), __fsub_rn(xp.x, xc.x));
                a[c][0] = c4_folded2d(dx1, xp, xm, p_splat(k1[0]), p_splat(k2n[0]));
                const float2 ym1 = ld_pair(p - TMA_PX), yp1 = ld_pair(p + TMA_PX);
                const float2 ym2 = ld_pair(p - 2 * TMA_PX), yp2 = ld_pair(p + 2 * TMA_PX);
                a[c][1] = c4_folded2(yp1, ym1, yp2, ym2, p_splat(k1[1]), p_splat(k2n[1]));
                a[c][2] = c4_folded2(zq[c][3], zq[c][1], zq[c][4], zq[c][0], p_splat(k1[2]), p_splat(k2n[2]));
            }
            finish2(a);
            return;
        }
    }
    if (row_in && tile_x_in) {
        T a0[3][3], a1[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx;
            const auto xm = ld_pair(p - 2), xc = ld_pair(p), xp = ld_pair(p + 2);
            a0[c][0] = c4(xc.y, xm.y, xp.x, xm.x, 0);
            a1[c][0] = c4(xp.x, xc.x, xp.y, xm.y, 0);
            const auto ym1 = ld_pair(p - TMA_PX), yp1 = ld_pair(p + TMA_PX);
            const auto ym2 = ld_pair(p - 2 * TMA_PX), yp2 = ld_pair(p + 2 * TMA_PX);
            a0[c][1] = c4(yp1.x, ym1.x, yp2.x, ym2.x, 1);
            a1[c][1] = c4(yp1.y, ym1.y, yp2.y, ym2.y, 1);
            a0[c][2] = c4(zq[c][3].x, zq[c][1].x, zq[c][4].x, zq[c][0].x, 2);
            a1[c][2] = c4(zq[c][3].y, zq[c][1].y, zq[c][4].y, zq[c][0].y, 2);
        }
        finish(0, a0);
        finish(1, a1);
    } else if (row_in) {
        // Interior row: the scheme depends on x only
        // (src/jacobian.c:113-241): outer column -> one-sided
        // in x and second-order central in y, z; penultimate
        // column -> second-order central; else fourth order.
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int xv = x + v;
            if (xv >= g.nx) continue;
            const bool xo_lo = xv == 0, xo_hi = xv == g.nx - 1;
            const bool second = xo_lo || xo_hi || xv == 1 || xv == g.nx - 2;
            T a[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx + v;
                const T fx = xo_lo ? fd_fwd<T>(p[0], p[1], p[2], ih[0])
                                   : (xo_hi ? fd_bwd<T>(p[0], p[-1], p[-2], ih[0])
                                            : fd_c2<T>(p[1], p[-1], ih[0]));
                const T cx4 = c4(p[1], p[-1], p[2], p[-2], 0);
                a[c][0] = second ? fx : cx4;
                const T cy4 = c4(p[TMA_PX], p[-TMA_PX], p[2 * TMA_PX], p[-2 * TMA_PX], 1);
                const T cy2 = fd_c2<T>(p[TMA_PX], p[-TMA_PX], ih[1]);
                a[c][1] = second ? cy2 : cy4;
                T zv[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) zv[k] = v ? zq[c][k].y : zq[c][k].x;
                const T cz4 = c4(zv[3], zv[1], zv[4], zv[0], 2);
                const T cz2 = fd_c2<T>(zv[3], zv[1], ih[2]);
                a[c][2] = second ? cz2 : cz4;
            }
            finish(v, a);
        }
    } else {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int xv = x + v;
            if (xv >= g.nx) continue;
            int kk[3];
            schemes_at(xv, y, ze, g, kk);
            T a[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx + v;
                const T vx[5] = {p[-2], p[-1], p[0], p[1], p[2]};
                const T vy[5] = {p[-2 * TMA_PX], p[-TMA_PX], p[0], p[TMA_PX], p[2 * TMA_PX]};
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    T vz[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) vz[k] = v ? zq[c][k].y : zq[c][k].x;
                    const T *w = ax == 0 ? vx : (ax == 1 ? vy : vz);
                    T d;
                    switch (kk[ax]) {
                    case S_FWD: d = fd_fwd<T>(w[2], w[3], w[4], ih[ax]); break;
                    case S_BWD: d = fd_bwd<T>(w[2], w[1], w[0], ih[ax]); break;
                    case S_C2: d = fd_c2<T>(w[3], w[1], ih[ax]); break;
                    default: d = c4(w[3], w[1], w[4], w[0], ax); break;
                    }
                    a[c][ax] = d;
                }
            }
            finish(v, a);
        }
    }
}

// Block of TXW / 2 x TYT threads; each thread owns two adjacent columns
// (x, x + 1) of TT_Y / TYT rows of the tile, so every shared-memory read of
// the stencil and every global store covers two voxels.  A warp spans the
// whole tile width (TXW / 2 divides 32), which makes the evaluator choice
// below uniform across a warp except on rows near the y ends.  Two resident
// blocks per SM for FP32 (shared memory allows no more), one for FP64; the
// bound caps the registers accordingly.
//
// GREEDY instantiates the greedy method's trial (src/displacement_field_greedy.c:
// 23-67): the candidate is u + (eta d_k / 2) (v(p + e_k) - v(p - e_k)) on
// interior voxels, v the error map of the accepted field, streamed as one box
// of three planes per candidate plane; voxels on the volume boundary keep the
// content of the new field buffer, and the stored map is the error itself.
template <typename T, int TXW, int TYT, bool GREEDY = false>
__global__ void __launch_bounds__(TXW / 2 * TYT, (TXW / 2 * TYT <= 256 && sizeof(T) == 4) ? 2 : 1)
    k_trial_tma(const VolumeDesc<T> *__restrict__ vols, const int *__restrict__ tile_vol, int total_tiles,
                unsigned char *__restrict__ work_flag, TileQueue *queue, int pf) {
    using L = TrialTmaLayout<T, TXW, GREEDY>;
    constexpr int TPX = TXW / 2, NTH = TPX * TYT, RYT = TT_Y / TYT;
    constexpr int TMA_PX = L::TMA_PX, TMA_PLANE = L::TMA_PLANE;
    static_assert(TPX <= 32 && 32 % TPX == 0, "a warp spans whole tile rows");
    static_assert((L::R & (L::R - 1)) == 0, "ring size is a power of two");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    T *ring = reinterpret_cast<T *>(smem + L::RING_OFF);
    T *vring = reinterpret_cast<T *>(smem + L::VRING_OFF);  // greedy: error-map planes
    __shared__ double red[2 * (NTH / 32)];
    __shared__ int s_flag, s_fault;
    __shared__ T s_dd[3];  // greedy steps of the current tile

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx;
    if (tid == 0) {
        for (int s = 0; s < L::S; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_fault = 0;
    }
    __syncthreads();
    uint32_t kbase = 0;  // iterations consumed by this block (mbarrier phases)
    uint32_t vbase = 0;  // greedy: error-map planes loaded by this block (ring position)

    __shared__ int s_tile;
    for (int tile = take_tile<TPX>(queue, total_tiles, &s_tile); tile >= 0;
         tile = take_tile<TPX>(queue, total_tiles, &s_tile)) {
        const VolumeDesc<T> &V = vols[tile_vol[tile]];
        SolverState *st = V.st;
        if (ldcg_int(&st->done)) continue;
        const Geom g = V.g;
        const int phase = ldcg_int(&st->phase);
        const int old_b = ldcg_int(&st->old_buf);
        const int v_cur = GREEDY ? ldcg_int(&st->v_cur) : 0;
        // Greedy: the new buffer's boundary values are all +0 when it is
        // buffer 1 or the initial field's boundary is; no copies then.
        const bool stale_zero = GREEDY && (old_b == 0 || !ldcg_int(&st->b0_nonzero));
        const double eta = __ldcg(&st->eta);
        const bool trial = phase != PH_EVAL0;
        const int lt = tile - V.tile_begin;
        const int txi = lt % V.tiles_x, tyi = (lt / V.tiles_x) % V.tiles_y, tzi = lt / (V.tiles_x * V.tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * V.bz;
        const int z1 = min(z0 + V.bz, g.nz);
        const int n_it = z1 - z0 + 4;  // candidate planes z0-2 .. z1+1
        const CUtensorMap *tm_u = V.tm_field[old_b];
        const CUtensorMap *tm_g = GREEDY ? V.tm_v[v_cur] : V.tm_grad;
        T *dst = V.field[old_b ^ 1];
        // Gradient method: e' of the evaluated field; greedy: its error map.
        T *ep_out = GREEDY ? V.v[trial ? v_cur ^ 1 : v_cur] : V.ep[trial ? old_b ^ 1 : old_b];
        const T eta_t = (T) eta;
        if (GREEDY) {
            // Greedy steps along x, y, z (src/displacement_field_greedy.c:36-38).
            if (tid < 3) s_dd[tid] = (T) (eta * V.g.sp[tid] * .5);  // V.g: no local copy indexed
            __syncthreads();
        }
        const T ih[3] = {(T) g.ih[0], (T) g.ih[1], (T) g.ih[2]};
        const T tol = (T) st->tolerance, delta = (T) st->delta, zeta = (T) st->zeta;

        int issued_n = 0;  // iterations whose loads were issued (thread 0)
        const unsigned wait_limit = V.wait_limit ? V.wait_limit : (1u << 22);
        // Issues the loads of iteration j (candidate plane z0-2+j) into its stage.
        auto issue = [&](int j) {
            issued_n = j + 1;
            if (trial && tile == V.drop_tile && j == V.drop_it) return;  // failure-path test only
            const uint32_t k = kbase + j;
            const int s = k % L::S;
            unsigned char *sb = smem + s * L::STAGE_BYTES;
            const int q = z0 - 2 + j, ze = q - 2;
            const bool with_target = ze >= z0 && ze < z1;
            // Greedy: error-map plane q+1 (and, with the first plane, q-1
            // and q), plane p into ring slot (vbase + p - z0 + 3) % RV.
            const int nv = GREEDY && trial ? (j == 0 ? 3 : 1) : 0;
            const uint32_t bytes = L::U_BYTES + (trial && !GREEDY ? L::U_BYTES : 0) + nv * L::V_BYTES +
                                   (with_target ? L::JT_BYTES + L::MASK_BYTES : 0);
            mbar_arrive_expect_tx(&bars[s], bytes);
            tma_load_4d(sb, tm_u, &bars[s], x0 - TMA_HX, y0 - TMA_HY, q, 0);
            if (trial) {
                if (GREEDY)
                    for (int p = q + 2 - nv; p <= q + 1; ++p)
                        tma_load_3d(vring + ((vbase + (uint32_t) (p - z0 + 3)) % L::RV) * (L::V_SLOT / sizeof(T)),
                                    tm_g, &bars[s], x0 - TMA_HX, y0 - TMA_HY - 1, p);
                else
                    tma_load_4d(sb + L::U_BYTES, tm_g, &bars[s], x0 - TMA_HX, y0 - TMA_HY, q, 0);
            }
            if (with_target) {
                tma_load_3d(sb + L::JT_OFF, V.tm_Jt, &bars[s], x0, y0, ze);
                tma_load_3d(sb + L::MASK_OFF, V.tm_mask, &bars[s], x0, y0, ze);
            }
            // Warm L2 with the boxes of iteration j + pf.
            if (pf > 0 && j + pf < n_it) {
                const int qp = q + pf, zp = qp - 2;
                tma_prefetch_4d(tm_u, x0 - TMA_HX, y0 - TMA_HY, qp, 0);
                if (trial) tma_prefetch_4d(tm_g, x0 - TMA_HX, y0 - TMA_HY, qp, 0);
                if (zp >= z0 && zp < z1) {
                    tma_prefetch_3d(V.tm_Jt, x0, y0, zp);
                    tma_prefetch_3d(V.tm_mask, x0, y0, zp);
                }
            }
        };

        if (tid == 0) {
            tmap_acquire(tm_u);
            tmap_acquire(tm_g);
            tmap_acquire(V.tm_Jt);
            tmap_acquire(V.tm_mask);
            for (int j = 0; j < min(L::S, n_it); ++j) issue(j);
        }

        const int x = x0 + 2 * tx;     // this thread's columns: x, x + 1
        const int lx = 2 * tx + TMA_HX;  // their box column
        const bool pair_in = x + 1 < g.nx;
        // Own columns: candidate values of planes q-4 .. q (z differences),
        // one pair (x, x + 1) per row, component and plane.
        using P2 = typename PairOf<T>::type;
        P2 zq[RYT][3][5];
#pragma unroll
        for (int r = 0; r < RYT; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 5; ++k) zq[r][c][k] = P2{T(0), T(0)};
        double acc_s = 0.0;
        T acc_mt = T(0);
        bool failed = false;
        int fail_it = 0;
        long long qoff = (long long) (z0 - 2) * g.zs;  // offset of plane q
        // Greedy trial: stale boundary values of the first candidate plane
        // (its ring slot is free: the tile queue's barrier has passed).
        if (GREEDY && trial && !stale_zero)
            greedy_prefetch_stale<T, L>(ring + (size_t) ((z0 - 2) & (L::R - 1)) * 3 * TMA_PLANE, tid, NTH, g, x0, y0,
                                        z0 - 2, dst);
        for (int it = 0; it < n_it; ++it, qoff += g.zs) {
            const uint32_t k = kbase + it;
            const int s = k % L::S;
            const uint32_t par = (k / L::S) & 1u;
            // Every thread waits for the stage itself (bounded); a timeout is
            // agreed on after the barrier below, so all threads leave together.
            const bool ok = mbar_wait_bounded(&bars[s], par, wait_limit);
            if (!ok) s_fault = 1;
            const unsigned char *sb = smem + s * L::STAGE_BYTES;
            const int q = z0 - 2 + it, ze = q - 2;
            T *slot = ring + (size_t) (q & (L::R - 1)) * 3 * TMA_PLANE;
            // Candidate plane q (tile + halo): u - eta g, vectorised.
            if (ok) {
                constexpr int VEC = 16 / (int) sizeof(T);
                using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
                const V4 *u4 = reinterpret_cast<const V4 *>(sb);
                const V4 *g4 = reinterpret_cast<const V4 *>(sb + L::U_BYTES);
                V4 *c4 = reinterpret_cast<V4 *>(slot);
                if (GREEDY && trial) {
                    if (!stale_zero) cp_async_wait_all();  // this thread's stale values of plane q
                    auto vplane = [&](int p) -> const T * {
                        return vring + ((vbase + (uint32_t) (p - z0 + 3)) % L::RV) * (L::V_SLOT / sizeof(T));
                    };
                    greedy_form<T, L>(reinterpret_cast<const T *>(sb), vplane(q - 1), vplane(q), vplane(q + 1), slot,
                                      tid, NTH, g, x0, y0, q, s_dd, stale_zero);
                } else
                // Counted from the last thread: the runs left over after
                // whole sweeps go to the last warps, not to warp 0, whose
                // thread 0 also issues the loads.
                for (int i = NTH - 1 - tid; i < 3 * TMA_PLANE / VEC; i += NTH) {
                    V4 a = u4[i];
                    if (trial) {
                        const V4 b = g4[i];
                        T *pa = reinterpret_cast<T *>(&a);
                        const T *pb = reinterpret_cast<const T *>(&b);
#pragma unroll
                        for (int e = 0; e < VEC; ++e) pa[e] = pa[e] - eta_t * pb[e];
                    }
                    c4[i] = a;
                }
            }
            const bool eval = ze >= z0 && ze < z1;
            T jt[RYT][2];
            bool msk[RYT][2];
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                jt[r][0] = jt[r][1] = T(0);
                msk[r][0] = msk[r][1] = false;
                if (eval && ok) {
                    const int o = (ty + r * TYT) * TXW + 2 * tx;
                    const auto j2 = ld_pair(reinterpret_cast<const T *>(sb + L::JT_OFF) + o);
                    const unsigned short m2 = *reinterpret_cast<const unsigned short *>(sb + L::MASK_OFF + o);
                    jt[r][0] = j2.x;
                    jt[r][1] = j2.y;
                    msk[r][0] = (m2 & 0xffu) != 0;
                    msk[r][1] = (m2 >> 8) != 0;
                }
            }
            __syncthreads();
            if (s_fault) {
                failed = true;
                fail_it = it;
                break;
            }
            if (tid == 0 && it + L::S < n_it) issue(it + L::S);
            // Greedy trial: stale boundary values of plane q+1, into its ring
            // slot, which held plane q-3: every warp has finished reading it
            // (the stencil of the previous iteration) at the barrier above.
            if (GREEDY && trial && !stale_zero && it + 1 < n_it)
                greedy_prefetch_stale<T, L>(ring + (size_t) ((q + 1) & (L::R - 1)) * 3 * TMA_PLANE, tid, NTH, g, x0,
                                            y0, q + 1, dst);
            // Shift the own-column queues by plane q; store the candidate.
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                const int ly = ty + r * TYT + TMA_HY;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) zq[r][c][kk] = zq[r][c][kk + 1];
                    zq[r][c][4] = ld_pair(slot + c * TMA_PLANE + ly * TMA_PX + lx);
                }
                const int y = y0 + ty + r * TYT;
                if (trial && x < g.nx && y < g.ny && q >= z0 && q < z1) {
                    T *o = dst + qoff + (long long) y * g.ys + x;
                    if (pair_in) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) st_pair(o + c * g.cs, zq[r][c][4].x, zq[r][c][4].y);
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; ++c) o[c * g.cs] = zq[r][c][4].x;
                    }
                }
            }
            if (eval) {
                const T *jp = ring + (size_t) (ze & (L::R - 1)) * 3 * TMA_PLANE;
                // Fourth-order weights with the spacing folded in (FP32); the
                // FP64 path keeps the reference's operation order.
                const T k1[3] = {FD<T>::two_thirds * ih[0], FD<T>::two_thirds * ih[1], FD<T>::two_thirds * ih[2]};
                const T k2n[3] = {-FD<T>::one_twelfth * ih[0], -FD<T>::one_twelfth * ih[1],
                                  -FD<T>::one_twelfth * ih[2]};
                auto c4 = [&](T p1, T m1, T p2, T m2, int ax) -> T {
                    if constexpr (sizeof(T) == 4) return c4_folded(p1, m1, p2, m2, k1[ax], k2n[ax]);
                    else return fd_c4<T>(p1, m1, p2, m2, ih[ax]);
                };
                // Three evaluators: rows and planes inside [2, n-3] of a tile
                // whose columns all lie inside [2, nx-3] use the fourth-order
                // stencil only; interior rows of a tile that reaches an x end
                // select the scheme per voxel without branching; rows or
                // planes on the two outer layers take the general path.
                const bool plane_in = ze >= 2 && ze <= g.nz - 3;
                const bool tile_x_in = x0 >= 2 && x0 + TXW - 1 <= g.nx - 3;
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    const int y = y0 + ty + r * TYT;
                    const bool row_in = plane_in && y >= 2 && y <= g.ny - 3;
                    const int ly = ty + r * TYT + TMA_HY;
                    if (x >= g.nx || y >= g.ny) continue;
                    T epv[2];
                    // Error terms of voxel v from its Jacobian (finish_j) or
                    // its Jacobian matrix minus I (finish).
                    auto finish_j = [&](int v, const T J) {
                        const T vv = voxel_error<T>(J, jt[r][v], msk[r][v], tol);
                        acc_s += (double) vv * (double) vv;
                        const T av = fabs(vv);  // the maximum is exact in the element type
                        if (msk[r][v] && av > acc_mt) acc_mt = av;
                        T ep = vv;
                        if (!GREEDY && J < delta) ep += zeta * (J - delta);  // src/displacement_field_gradient.c:71-88
                        epv[v] = ep;
                    };
                    auto finish = [&](int v, const T (&a)[3][3]) { finish_j(v, det_i_plus<T>(a)); };
                    if (row_in && tile_x_in) {
                        if constexpr (sizeof(T) == 4) {
                            // Both voxels at once, as FP32 pairs.
                            float2 a[3][3];
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx;
                                const float2 xm = ld_pair(p - 2), xc = ld_pair(p), xp = ld_pair(p + 2);
                                const float2 dx1 = make_float2(__fsub_rn(xc.y, xm.y), __fsub_rn(xp.x, xc.x));
                                a[c][0] = c4_folded2d(dx1, xp, xm, p_splat(k1[0]), p_splat(k2n[0]));
                                const float2 ym1 = ld_pair(p - TMA_PX), yp1 = ld_pair(p + TMA_PX);
                                const float2 ym2 = ld_pair(p - 2 * TMA_PX), yp2 = ld_pair(p + 2 * TMA_PX);
                                a[c][1] = c4_folded2(yp1, ym1, yp2, ym2, p_splat(k1[1]), p_splat(k2n[1]));
                                a[c][2] = c4_folded2(zq[r][c][3], zq[r][c][1], zq[r][c][4], zq[r][c][0],
                                                     p_splat(k1[2]), p_splat(k2n[2]));
                            }
                            const float2 J2 = det_i_plus2(a);
                            finish_j(0, J2.x);
                            finish_j(1, J2.y);
                        } else {
                            T a0[3][3], a1[3][3];
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx;
                                const auto xm = ld_pair(p - 2), xc = ld_pair(p), xp = ld_pair(p + 2);
                                a0[c][0] = c4(xc.y, xm.y, xp.x, xm.x, 0);
                                a1[c][0] = c4(xp.x, xc.x, xp.y, xm.y, 0);
                                const auto ym1 = ld_pair(p - TMA_PX), yp1 = ld_pair(p + TMA_PX);
                                const auto ym2 = ld_pair(p - 2 * TMA_PX), yp2 = ld_pair(p + 2 * TMA_PX);
                                a0[c][1] = c4(yp1.x, ym1.x, yp2.x, ym2.x, 1);
                                a1[c][1] = c4(yp1.y, ym1.y, yp2.y, ym2.y, 1);
                                a0[c][2] = c4(zq[r][c][3].x, zq[r][c][1].x, zq[r][c][4].x, zq[r][c][0].x, 2);
                                a1[c][2] = c4(zq[r][c][3].y, zq[r][c][1].y, zq[r][c][4].y, zq[r][c][0].y, 2);
                            }
                            finish(0, a0);
                            finish(1, a1);
                        }
                    } else if (row_in) {
                        // Interior row: the scheme depends on x only
                        // (src/jacobian.c:113-241): outer column -> one-sided
                        // in x and second-order central in y, z; penultimate
                        // column -> second-order central; else fourth order.
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            const int xv = x + v;
                            if (xv >= g.nx) continue;
                            const bool xo_lo = xv == 0, xo_hi = xv == g.nx - 1;
                            const bool second = xo_lo || xo_hi || xv == 1 || xv == g.nx - 2;
                            T a[3][3];
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx + v;
                                const T fx = xo_lo ? fd_fwd<T>(p[0], p[1], p[2], ih[0])
                                                   : (xo_hi ? fd_bwd<T>(p[0], p[-1], p[-2], ih[0])
                                                            : fd_c2<T>(p[1], p[-1], ih[0]));
                                const T cx4 = c4(p[1], p[-1], p[2], p[-2], 0);
                                a[c][0] = second ? fx : cx4;
                                const T cy4 = c4(p[TMA_PX], p[-TMA_PX], p[2 * TMA_PX], p[-2 * TMA_PX], 1);
                                const T cy2 = fd_c2<T>(p[TMA_PX], p[-TMA_PX], ih[1]);
                                a[c][1] = second ? cy2 : cy4;
                                T zv[5];
#pragma unroll
                                for (int k = 0; k < 5; ++k) zv[k] = v ? zq[r][c][k].y : zq[r][c][k].x;
                                const T cz4 = c4(zv[3], zv[1], zv[4], zv[0], 2);
                                const T cz2 = fd_c2<T>(zv[3], zv[1], ih[2]);
                                a[c][2] = second ? cz2 : cz4;
                            }
                            finish(v, a);
                        }
                    } else {
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            const int xv = x + v;
                            if (xv >= g.nx) continue;
                            int kk[3];
                            schemes_at(xv, y, ze, g, kk);
                            T a[3][3];
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const T *p = jp + c * TMA_PLANE + ly * TMA_PX + lx + v;
                                const T vx[5] = {p[-2], p[-1], p[0], p[1], p[2]};
                                const T vy[5] = {p[-2 * TMA_PX], p[-TMA_PX], p[0], p[TMA_PX], p[2 * TMA_PX]};
                                T vz[5];
#pragma unroll
                                for (int k = 0; k < 5; ++k) vz[k] = v ? zq[r][c][k].y : zq[r][c][k].x;
#pragma unroll
                                for (int ax = 0; ax < 3; ++ax) {
                                    const T *w = ax == 0 ? vx : (ax == 1 ? vy : vz);
                                    T d;
                                    switch (kk[ax]) {
                                    case S_FWD: d = fd_fwd<T>(w[2], w[3], w[4], ih[ax]); break;
                                    case S_BWD: d = fd_bwd<T>(w[2], w[1], w[0], ih[ax]); break;
                                    case S_C2: d = fd_c2<T>(w[3], w[1], ih[ax]); break;
                                    default: d = c4(w[3], w[1], w[4], w[0], ax); break;
                                    }
                                    a[c][ax] = d;
                                }
                            }
                            finish(v, a);
                        }
                    }
                    T *o = ep_out + (qoff - 2 * g.zs) + (long long) y * g.ys + x;
                    if (pair_in)
                        st_pair(o, epv[0], epv[1]);
                    else
                        o[0] = epv[0];
                }
            }
        }
        if (failed) {
            if (GREEDY) cp_async_wait_all();  // no element copy lands after the block has left
            if (tid == 0) tma_fault<L::S>(st, bars, kbase, fail_it + 1, issued_n);
            __syncthreads();
            return;
        }
        kbase += n_it;
        vbase += n_it + 2;

        const double2 rr = block_reduce_n<NTH, TPX>(acc_s, (double) acc_mt, red);
        if (tid == 0) V.part_t[lt] = rr;
        if (publish_partial_n<TPX>(&st->ticket_t, V.ntiles, &s_flag)) {
            // Each thread folds a fixed subset of the tile partials, so the
            // total does not depend on timing.
            double ssum = 0.0, smax = 0.0;
            for (int i = tid; i < V.ntiles; i += NTH) {
                const double2 pp = __ldcg(&V.part_t[i]);
                ssum += pp.x;
                smax = fmax(smax, pp.y);
            }
            const double2 tot = block_reduce_n<NTH, TPX>(ssum, smax, red);
            if (tid == 0) {
                st->ticket_t = 0;
                control_after_trial(st, tot.x, tot.y);
                if (work_flag) *work_flag = 1;
                __threadfence();
            }
        }
        __syncthreads();
    }
}

// Halo tasks of the gradient kernel's P terms per plane: x sides (one cell
// each) and y sides (two cells each), one per thread of their own warps.
template <int TXW>
__host__ __device__ constexpr int grad_halo_rows() {
    return (2 * TT_Y + TXW) / (TXW / 2);
}

// Block of TXW / 2 x (TYT + grad_halo_rows) threads.  The first TYT rows
// own the tile: each thread two adjacent columns (x, x + 1) of TT_Y / TYT
// rows, so the field, e' and P-term reads and the gradient stores are pairs.
// The last rows compute the P terms of the tile's halo cells, so no warp
// does halo work on top of its own cells.  Two resident blocks per SM for
// FP32 (shared memory allows no more), one for FP64.
template <typename T, int TXW, int TYT>
__global__ void __launch_bounds__(TXW / 2 * (TYT + grad_halo_rows<TXW>()), sizeof(T) == 4 ? 2 : 1)
    k_gradient_tma(const VolumeDesc<T> *__restrict__ vols, const int *__restrict__ tile_vol, int total_tiles,
                   unsigned char *__restrict__ work_flag, TileQueue *queue, int pf) {
    using L = GradTmaLayout<T, TXW>;
    constexpr int TPX = TXW / 2, RYT = TT_Y / TYT;
    constexpr int NHALO = 2 * TT_Y + TXW;  // halo tasks: x sides (one cell each), y sides (two cells each)
    constexpr int NOWN = TPX * TYT, NTH = NOWN + NHALO;
    constexpr int TMA_PX = L::TMA_PX, TMA_PLANE = L::TMA_PLANE;
    constexpr int PXP = L::PXP, PYP = L::PYP;
    static_assert(TPX <= 32 && 32 % TPX == 0, "a warp spans whole tile rows");
    static_assert(NHALO % TPX == 0 && NHALO / TPX == grad_halo_rows<TXW>(), "whole halo rows");
    static_assert(NOWN % 32 == 0, "owner and halo threads in separate warps");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    T *pxy = reinterpret_cast<T *>(smem + L::P_OFF);
    __shared__ double red[2 * (NTH / 32)];
    __shared__ int s_flag, s_fault;
    // P terms of the x (t = 0..2) and y (t = 3..5) directions.  P column c
    // holds x = x0 + c - 2 (so the own pairs start at even columns), P row r
    // holds y = y0 + r - 1.
    auto PT = [&](int slot, int t, int r, int c) -> T * { return pxy + ((slot * 6 + t) * PYP + r) * PXP + c; };

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx;
    const bool own = ty < TYT;  // owner threads (the others: halo tasks)
    if (tid == 0) {
        for (int s = 0; s < L::S; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_fault = 0;
    }
    __syncthreads();
    uint32_t kbase = 0;

    __shared__ int s_tile;
    for (int tile = take_tile<TPX>(queue, total_tiles, &s_tile); tile >= 0;
         tile = take_tile<TPX>(queue, total_tiles, &s_tile)) {
        const VolumeDesc<T> &V = vols[tile_vol[tile]];
        SolverState *st = V.st;
        if (ldcg_int(&st->done) || !ldcg_int(&st->need_gradient)) continue;
        const Geom g = V.g;
        const int old_b = ldcg_int(&st->old_buf);
        const int lt = tile - V.tile_begin;
        const int txi = lt % V.tiles_x, tyi = (lt / V.tiles_x) % V.tiles_y, tzi = lt / (V.tiles_x * V.tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * V.bz;
        const int z1 = min(z0 + V.bz, g.nz);
        const int n_it = z1 - z0 + 4;  // u planes z0-2 .. z1+1
        const CUtensorMap *tm_u = V.tm_field[old_b];
        const CUtensorMap *tm_e = V.tm_ep[old_b];
        const T ihx = (T) g.ih[0], ihy = (T) g.ih[1], ihz = (T) g.ih[2];
        // Second-order central difference (p1 - m1) * ih * 0.5.  In FP32 the
        // factor 0.5 ih is folded into one constant: halving is exact, so the
        // result is the same, with one multiply fewer.
        const T hx = ihx * T(0.5), hy = ihy * T(0.5), hz = ihz * T(0.5);
        auto c2 = [&](T p1, T m1, int ax) -> T {
            if (sizeof(T) == 4) return (p1 - m1) * (ax == 0 ? hx : (ax == 1 ? hy : hz));
            return fd_c2<T>(p1, m1, ax == 0 ? ihx : (ax == 1 ? ihy : ihz));
        };

        int issued_n = 0;
        auto issue = [&](int j) {
            issued_n = j + 1;
            const uint32_t k = kbase + j;
            const int s = k % L::S;
            unsigned char *sb = smem + s * L::STAGE_BYTES;
            const int q = z0 - 2 + j;
            mbar_arrive_expect_tx(&bars[s], L::U_BYTES + L::E_BYTES);
            tma_load_4d(sb, tm_u, &bars[s], x0 - TMA_HX, y0 - TMA_HY, q, 0);
            tma_load_3d(sb + L::U_BYTES, tm_e, &bars[s], x0 - TMA_HX, y0 - TMA_HY, q);
            // Warm L2 with the boxes of iteration j + pf.
            if (pf > 0 && j + pf < n_it) {
                tma_prefetch_4d(tm_u, x0 - TMA_HX, y0 - TMA_HY, q + pf, 0);
                tma_prefetch_3d(tm_e, x0 - TMA_HX, y0 - TMA_HY, q + pf);
            }
        };
        if (tid == 0) {
            tmap_acquire(tm_u);
            tmap_acquire(tm_e);
            for (int j = 0; j < min(L::S, n_it); ++j) issue(j);
        }
        auto stage_u = [&](int j) -> const T * {
            return reinterpret_cast<const T *>(smem + ((kbase + j) % L::S) * L::STAGE_BYTES);
        };
        auto stage_e = [&](int j) -> const T * {
            return reinterpret_cast<const T *>(smem + ((kbase + j) % L::S) * L::STAGE_BYTES + L::U_BYTES);
        };

        const int x = x0 + 2 * tx;       // this thread's columns: x, x + 1
        const int lx = 2 * tx + TMA_HX;  // their box column
        const int cp = 2 * tx + 2;       // their P column
        // P_z terms of the own cells (x, x + 1 as one pair): planes p-2, p-1
        // and the one computed now.
        using P2 = typename PairOf<T>::type;
        P2 pz_m2[RYT][3], pz_m1[RYT][3];
#pragma unroll
        for (int r = 0; r < RYT; ++r)
#pragma unroll
            for (int i = 0; i < 3; ++i) pz_m2[r][i] = pz_m1[r][i] = P2{T(0), T(0)};
        double acc = 0.0;
        bool failed = false;
        int fail_it = 0;
        long long zoff = (long long) (z0 - 4) * g.zs;  // offset of gradient plane z = q - 2
        for (int it = 0; it < n_it; ++it, zoff += g.zs) {
            const uint32_t k = kbase + it;
            const int s = k % L::S;
            const uint32_t par = (k / L::S) & 1u;
            const bool ok = mbar_wait_bounded(&bars[s], par);
            if (!ok) s_fault = 1;
            const int q = z0 - 2 + it;
            const int p = q - 1;  // plane of P computed now (needs u(q-2..q), e'(q-1))
            P2 pz_new[RYT][3];
#pragma unroll
            for (int r = 0; r < RYT; ++r)
#pragma unroll
                for (int i = 0; i < 3; ++i) pz_new[r][i] = P2{T(0), T(0)};
            if (it >= 2 && ok) {
                const T *um = stage_u(it - 2), *u0 = stage_u(it - 1), *up = stage_u(it);
                const T *e0 = stage_e(it - 1);
                const int ps = ring_slot(p, L::NP);
                // FP32 states every rounding, so the scalar (halo) and the
                // paired (own) cells give the same bits: a minor is a
                // difference of two products, a diagonal entry d h + 1 one
                // fused multiply-add.
                auto minor = [](const T m[3][3], int i, int kk) -> T {
                    const int r0 = i == 0 ? 1 : 0, r1 = i == 2 ? 1 : 2;
                    const int c0 = kk == 0 ? 1 : 0, c1 = kk == 2 ? 1 : 2;
                    if constexpr (sizeof(T) == 4)
                        return __fsub_rn(__fmul_rn(m[r0][c0], m[r1][c1]), __fmul_rn(m[r0][c1], m[r1][c0]));
                    else return m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0];
                };
                // M = I + grad u (second-order central) at box cell (cx, cy).
                auto mat = [&](int cx, int cy, T m[3][3]) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int o = c * TMA_PLANE + cy * TMA_PX + cx;
                        if constexpr (sizeof(T) == 4) {
                            const float d[3] = {__fsub_rn(u0[o + 1], u0[o - 1]),
                                                __fsub_rn(u0[o + TMA_PX], u0[o - TMA_PX]), __fsub_rn(up[o], um[o])};
                            const float h[3] = {hx, hy, hz};
#pragma unroll
                            for (int a = 0; a < 3; ++a)
                                m[c][a] = a == c ? __fmaf_rn(d[a], h[a], 1.f) : __fmul_rn(d[a], h[a]);
                        } else {
                            m[c][0] = c2(u0[o + 1], u0[o - 1], 0);
                            m[c][1] = c2(u0[o + TMA_PX], u0[o - TMA_PX], 1);
                            m[c][2] = c2(up[o], um[o], 2);
                            m[c][c] += T(1.0);
                        }
                    }
                };
                // The same for the pair of box cells (cx, cy), (cx + 1, cy); cx even.
                auto mat_pair = [&](int cx, int cy, T m0[3][3], T m1[3][3]) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int o = c * TMA_PLANE + cy * TMA_PX + cx;
                        const auto xm = ld_pair(u0 + o - 2), xc = ld_pair(u0 + o), xp = ld_pair(u0 + o + 2);
                        const auto ym = ld_pair(u0 + o - TMA_PX), yp = ld_pair(u0 + o + TMA_PX);
                        const auto zm = ld_pair(um + o), zp = ld_pair(up + o);
                        m0[c][0] = c2(xc.y, xm.y, 0);
                        m1[c][0] = c2(xp.x, xc.x, 0);
                        m0[c][1] = c2(yp.x, ym.x, 1);
                        m1[c][1] = c2(yp.y, ym.y, 1);
                        m0[c][2] = c2(zp.x, zm.x, 2);
                        m1[c][2] = c2(zp.y, zm.y, 2);
                        m0[c][c] += T(1.0);
                        m1[c][c] += T(1.0);
                    }
                };
                // FP32: M of the pair (cx, cy), (cx + 1, cy) as pairs, and
                // the minors as pairs (the arithmetic of mat and minor).
                auto mat_pair2 = [&](int cx, int cy, P2 M[3][3]) {
                    if constexpr (sizeof(T) == 4) {
                        const float2 h2[3] = {p_splat(hx), p_splat(hy), p_splat(hz)};
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const int o = c * TMA_PLANE + cy * TMA_PX + cx;
                            const float2 xm = ld_pair(u0 + o - 2), xc = ld_pair(u0 + o), xp = ld_pair(u0 + o + 2);
                            const float2 ym = ld_pair(u0 + o - TMA_PX), yp = ld_pair(u0 + o + TMA_PX);
                            const float2 zm = ld_pair(um + o), zp = ld_pair(up + o);
                            const float2 d[3] = {make_float2(__fsub_rn(xc.y, xm.y), __fsub_rn(xp.x, xc.x)),
                                                 p_sub(yp, ym), p_sub(zp, zm)};
#pragma unroll
                            for (int a = 0; a < 3; ++a)
                                M[c][a] = a == c ? p_fma(d[a], h2[a], p_splat(1.f)) : p_mul(d[a], h2[a]);
                        }
                    }
                };
                auto minor2 = [](const P2 M[3][3], int i, int kk) -> P2 {
                    const int r0 = i == 0 ? 1 : 0, r1 = i == 2 ? 1 : 2;
                    const int c0 = kk == 0 ? 1 : 0, c1 = kk == 2 ? 1 : 2;
                    if constexpr (sizeof(T) == 4)
                        return p_sub(p_mul(M[r0][c0], M[r1][c1]), p_mul(M[r0][c1], M[r1][c0]));
                    else return P2{};
                };
                auto st2 = [](T *p, P2 v) { *reinterpret_cast<P2 *>(p) = v; };
#pragma unroll
                for (int r = 0; r < RYT; ++r) {  // own cells: all nine terms (P_z in registers)
                    if (!own) break;
                    const int ly = ty + r * TYT + TMA_HY, rp = ty + r * TYT + 1;
                    if constexpr (sizeof(T) == 4) {
                        float2 M[3][3];
                        mat_pair2(lx, ly, M);
                        const float2 ep = ld_pair(e0 + ly * TMA_PX + lx);
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            st2(PT(ps, i, rp, cp), p_mul(ep, minor2(M, i, 0)));
                            st2(PT(ps, 3 + i, rp, cp), p_mul(ep, minor2(M, i, 1)));
                            pz_new[r][i] = p_mul(ep, minor2(M, i, 2));
                        }
                    } else {
                        T m0[3][3], m1[3][3];
                        mat_pair(lx, ly, m0, m1);
                        const auto ep = ld_pair(e0 + ly * TMA_PX + lx);
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            st_pair(PT(ps, i, rp, cp), ep.x * minor(m0, i, 0), ep.y * minor(m1, i, 0));
                            st_pair(PT(ps, 3 + i, rp, cp), ep.x * minor(m0, i, 1), ep.y * minor(m1, i, 1));
                            pz_new[r][i] = P2{ep.x * minor(m0, i, 2), ep.y * minor(m1, i, 2)};
                        }
                    }
                }
                // Halo cells, on the halo threads: P_x on the two side
                // columns, P_y on the two end rows (pairs).
                const int h = tid - NOWN;
                if (h >= 0 && h < 2 * TT_Y) {
                    const int side = h / TT_Y, row = h % TT_Y;
                    const int c = side ? TXW + 2 : 1;
                    const int cx = c - 2 + TMA_HX, cy = row + TMA_HY;
                    T m[3][3];
                    mat(cx, cy, m);
                    const T ep = e0[cy * TMA_PX + cx];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        if constexpr (sizeof(T) == 4) *PT(ps, i, row + 1, c) = __fmul_rn(ep, minor(m, i, 0));
                        else *PT(ps, i, row + 1, c) = ep * minor(m, i, 0);
                    }
                } else if (h >= 2 * TT_Y) {
                    const int h2 = h - 2 * TT_Y;
                    const int side = h2 / TPX, col = 2 * (h2 % TPX);
                    const int r = side ? TT_Y + 1 : 0;
                    const int cx = col + TMA_HX, cy = r - 1 + TMA_HY;
                    if constexpr (sizeof(T) == 4) {
                        float2 M[3][3];
                        mat_pair2(cx, cy, M);
                        const float2 ep = ld_pair(e0 + cy * TMA_PX + cx);
#pragma unroll
                        for (int i = 0; i < 3; ++i) st2(PT(ps, 3 + i, r, col + 2), p_mul(ep, minor2(M, i, 1)));
                    } else {
                        T m0[3][3], m1[3][3];
                        mat_pair(cx, cy, m0, m1);
                        const auto ep = ld_pair(e0 + cy * TMA_PX + cx);
#pragma unroll
                        for (int i = 0; i < 3; ++i)
                            st_pair(PT(ps, 3 + i, r, col + 2), ep.x * minor(m0, i, 1), ep.y * minor(m1, i, 1));
                    }
                }
            }
            __syncthreads();
            if (s_fault) {
                failed = true;
                fail_it = it;
                break;
            }
            if (tid == 0 && it >= 2 && it - 2 + L::S < n_it) issue(it - 2 + L::S);
            const int z = q - 2;  // gradient plane: P(z-1), P(z), P(z+1) ready
            if (own && it >= 3 && z >= z0 && z < z1 && z >= 1 && z < g.nz - 1 && x < g.nx - 1 && x + 1 >= 1) {
                const int ps = ring_slot(z, L::NP);
                const bool in0 = x >= 1, in1 = x + 1 < g.nx - 1;
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    const int y = y0 + ty + r * TYT;
                    if (y < 1 || y >= g.ny - 1) continue;
                    const int rp = ty + r * TYT + 1;
                    T gv[2][3];
                    if constexpr (sizeof(T) == 4) {
                        // Pairs; every rounding stated: t = ih (P(-) - P(+)),
                        // g = (t_a - t_b) + t_c with the reference's signs.
                        float2 t[3][3];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const float2 a = ld_pair(PT(ps, i, rp, cp - 2)), b = ld_pair(PT(ps, i, rp, cp)),
                                         c = ld_pair(PT(ps, i, rp, cp + 2));
                            t[i][0] = p_mul(p_splat(ihx), make_float2(__fsub_rn(a.y, b.y), __fsub_rn(b.x, c.x)));
                            const float2 ym = ld_pair(PT(ps, 3 + i, rp - 1, cp)),
                                         yp = ld_pair(PT(ps, 3 + i, rp + 1, cp));
                            t[i][1] = p_mul(p_splat(ihy), p_sub(ym, yp));
                            t[i][2] = p_mul(p_splat(ihz), p_sub(pz_m2[r][i], pz_new[r][i]));
                        }
                        const float2 g0 = p_add(p_sub(t[0][0], t[0][1]), t[0][2]);
                        const float2 g1 = p_sub(p_sub(t[1][1], t[1][0]), t[1][2]);
                        const float2 g2 = p_add(p_sub(t[2][0], t[2][1]), t[2][2]);
                        gv[0][0] = g0.x, gv[0][1] = g1.x, gv[0][2] = g2.x;
                        gv[1][0] = g0.y, gv[1][1] = g1.y, gv[1][2] = g2.y;
                    } else {
                        T t[2][3][3];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const auto a = ld_pair(PT(ps, i, rp, cp - 2)), b = ld_pair(PT(ps, i, rp, cp)),
                                       c = ld_pair(PT(ps, i, rp, cp + 2));
                            t[0][i][0] = ihx * (a.y - b.y);
                            t[1][i][0] = ihx * (b.x - c.x);
                            const auto ym = ld_pair(PT(ps, 3 + i, rp - 1, cp)),
                                       yp = ld_pair(PT(ps, 3 + i, rp + 1, cp));
                            t[0][i][1] = ihy * (ym.x - yp.x);
                            t[1][i][1] = ihy * (ym.y - yp.y);
                            t[0][i][2] = ihz * (pz_m2[r][i].x - pz_new[r][i].x);
                            t[1][i][2] = ihz * (pz_m2[r][i].y - pz_new[r][i].y);
                        }
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            gv[v][0] = t[v][0][0] - t[v][0][1] + t[v][0][2];
                            gv[v][1] = -t[v][1][0] + t[v][1][1] - t[v][1][2];
                            gv[v][2] = t[v][2][0] - t[v][2][1] + t[v][2][2];
                        }
                    }
                    // |g|^2 of a voxel, summed in the element type, then in FP64.
                    auto sq = [](const T (&w)[3]) -> double {
                        if constexpr (sizeof(T) == 4)
                            return (double) __fmaf_rn(w[2], w[2], __fmaf_rn(w[1], w[1], __fmul_rn(w[0], w[0])));
                        else return (double) (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
                    };
                    T *o = V.grad + zoff + (long long) y * g.ys + x;
                    if (in0 && in1) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) st_pair(o + c * g.cs, gv[0][c], gv[1][c]);
                        acc += sq(gv[0]);
                        acc += sq(gv[1]);
                    } else {
                        // one voxel of the pair is on the boundary (x = 0 or nx - 1)
                        T w[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            w[c] = in0 ? gv[0][c] : gv[1][c];
                            o[(in0 ? 0 : 1) + c * g.cs] = w[c];
                        }
                        acc += sq(w);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RYT; ++r)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    pz_m2[r][i] = pz_m1[r][i];
                    pz_m1[r][i] = pz_new[r][i];
                }
        }
        if (failed) {
            if (tid == 0) tma_fault<L::S>(st, bars, kbase, fail_it + 1, issued_n);
            __syncthreads();
            return;
        }
        kbase += n_it;

        const double2 rr = block_reduce_n<NTH, TPX>(acc, 0.0, red);
        if (tid == 0) V.part_g[lt] = rr.x;
        if (publish_partial_n<TPX>(&st->ticket_g, V.ntiles, &s_flag)) {
            double ssum = 0.0;
            for (int i = tid; i < V.ntiles; i += NTH) ssum += __ldcg(&V.part_g[i]);
            const double2 tot = block_reduce_n<NTH, TPX>(ssum, 0.0, red);
            if (tid == 0) {
                st->ticket_g = 0;
                st->gn2 = tot.x;
                st->need_gradient = 0;
                st->gradients++;
                if (work_flag) *work_flag = 1;
                __threadfence();
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------
// Trial of the gradient method without a per-plane block barrier
// (k_trial_rel): the work and results of k_trial_tma<T, TXW, TYT, false>
// with another schedule.
//
// Stage j of a tile holds the field and gradient boxes of plane
// q = z0 - 2 + j (tile + 4 voxels in x, 2 rows in y) and the target and mask
// tiles of that plane.  A stage stays resident until its plane has been the
// stencil's centre plane, two iterations after it arrived, so no candidate
// plane is formed in shared memory: each stencil tap's candidate value
// u - eta g is formed where it is read (the expression of the formed plane,
// so FP64 results keep their bits), and each thread forms its own two
// columns of plane q for its register z-queue and for the store into the
// other field buffer.
//
// There is no block barrier in the plane loop.  A warp that has read a stage
// for the last time counts itself out of it (a shared counter); the warp that
// counts out last issues the stage's next load, the plane S iterations
// later, into the same slot.  So a warp waits only for data, and a slow warp
// delays only the refill of the stages it still reads.  A wait that runs out
// sets a block-wide fault flag that the other warps see at their next plane
// (or their own waits run out); one block barrier per tile, after the loop,
// agrees on it before the block reports the fault, waits (bounded) for its
// loads in flight and leaves.
// ------------------------------------------------------------------------
template <typename T, int TXW>
struct TrialRelLayout {
    static constexpr int TMA_PX = Box<TXW>::PX;
    static constexpr int TMA_PLANE = Box<TXW>::PLANE;
    static constexpr int S = 5;  // planes in use (centre, centre + 1, centre + 2) and two in flight
    static constexpr int U_BYTES = 3 * TMA_PLANE * (int) sizeof(T);
    static constexpr int G_OFF = U_BYTES;
    static constexpr int JT_BYTES = TXW * TT_Y * (int) sizeof(T);
    static constexpr int MASK_BYTES = TXW * TT_Y;
    static constexpr int JT_OFF = 2 * U_BYTES;
    static constexpr int MASK_OFF = JT_OFF + JT_BYTES;
    static constexpr int STAGE_BYTES = MASK_OFF + MASK_BYTES;  // u, g, Jt, mask
    static_assert(STAGE_BYTES % 128 == 0, "stages stay 128-byte aligned");
    static constexpr int BAR_OFF = S * STAGE_BYTES;
    static constexpr int CNT_OFF = BAR_OFF + S * 8;
    static constexpr int BYTES = CNT_OFF + S * 4;
};

// Orders this thread's earlier shared-memory accesses (and those ordered
// before them) before its later async-proxy (TMA) writes to shared memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Candidate pair u - eta g of two adjacent x voxels (box offset o).
template <typename T>
__device__ __forceinline__ typename PairOf<T>::type cand_pair(const T *u, const T *g, int o, T eta) {
    const auto a = ld_pair(u + o), b = ld_pair(g + o);
    typename PairOf<T>::type c;
    c.x = a.x - eta * b.x;
    c.y = a.y - eta * b.y;
    return c;
}

template <typename T, int TXW, int TYT>
__global__ void __launch_bounds__(TXW / 2 * TYT, (TXW / 2 * TYT <= 256 && sizeof(T) == 4) ? 2 : 1)
    k_trial_rel(const VolumeDesc<T> *__restrict__ vols, const int *__restrict__ tile_vol, int total_tiles,
                unsigned char *__restrict__ work_flag, TileQueue *queue) {
    using L = TrialRelLayout<T, TXW>;
    constexpr int TPX = TXW / 2, NTH = TPX * TYT, RYT = TT_Y / TYT, NW = NTH / 32, S = L::S;
    constexpr int TMA_PX = L::TMA_PX, TMA_PLANE = L::TMA_PLANE;
    static_assert(TPX <= 32 && 32 % TPX == 0, "a warp spans whole tile rows");
    static_assert(NTH % 32 == 0, "whole warps");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    unsigned *cnt = reinterpret_cast<unsigned *>(smem + L::CNT_OFF);
    __shared__ double red[2 * NW];
    __shared__ int s_flag, s_tile;
    __shared__ int s_issued;  // loads issued for the current tile (iterations 0 .. s_issued - 1)
    __shared__ volatile int s_fault;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars[s], 1);
            cnt[s] = 0;
        }
        fence_mbar_init();
        s_fault = 0;
    }
    __syncthreads();
    uint32_t kbase = 0;  // iterations consumed by this block (mbarrier phases)

    // The current tile's load parameters: any warp may issue a refill, so
    // they sit in shared memory rather than in every thread's registers.
    __shared__ const CUtensorMap *s_tm[4];  // field, gradient, target, mask
    __shared__ int s_box[4];                // x0, y0, z0, z1
    __shared__ int s_drop;                  // iteration whose loads are dropped (failure-path test), or -1
    __shared__ int s_done, s_phase, s_old;
    __shared__ double s_eta;
    // Per-tile constants read outside the voxel arithmetic (kept out of the
    // registers, which the plane loop needs): inverse spacing, the wait bound.
    __shared__ T s_ih[3];
    __shared__ unsigned s_wait;
    for (int tile = take_tile<TPX>(queue, total_tiles, &s_tile); tile >= 0;
         tile = take_tile<TPX>(queue, total_tiles, &s_tile)) {
        const VolumeDesc<T> &V = vols[tile_vol[tile]];
        SolverState *st = V.st;
        const Geom g = V.g;
        const int lt = tile - V.tile_begin;
        const int txi = lt % V.tiles_x, tyi = (lt / V.tiles_x) % V.tiles_y, tzi = lt / (V.tiles_x * V.tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * V.bz;
        const int z1 = min(z0 + V.bz, g.nz);
        const int n_it = z1 - z0 + 4;  // planes z0-2 .. z1+1
        // The volume's state, read once for the whole block: every warp takes
        // the same path through the tile.
        if (tid == 0) {
            s_done = ldcg_int(&st->done);
            s_phase = ldcg_int(&st->phase);
            s_old = ldcg_int(&st->old_buf);
            s_eta = __ldcg(&st->eta);
            s_tm[0] = V.tm_field[s_old];
            s_tm[1] = V.tm_grad;
            s_tm[2] = V.tm_Jt;
            s_tm[3] = V.tm_mask;
            s_box[0] = x0;
            s_box[1] = y0;
            s_box[2] = z0;
            s_box[3] = z1;
            s_drop = (s_phase != PH_EVAL0 && tile == V.drop_tile) ? V.drop_it : -1;
            s_issued = 0;
            for (int a = 0; a < 3; ++a) s_ih[a] = (T) g.ih[a];
            s_wait = V.wait_limit ? V.wait_limit : (1u << 22);
        }
        __syncthreads();
        if (s_done) continue;
        const int phase = s_phase;
        const int old_b = s_old;
        const double eta = s_eta;
        const bool trial = phase != PH_EVAL0;
        // The launch that evaluates the initial field takes it as it is:
        // eta 0 over the gradient buffer, which the set-up zeroed.
        const T eta_t = trial ? (T) eta : T(0);
        const T tol = (T) st->tolerance, delta = (T) st->delta, zeta = (T) st->zeta;

        // Issues the loads of iteration j (plane z0-2+j) into its slot (one
        // thread; the tile's parameters come from shared memory).
        auto issue = [&](int j) {
            atomicMax(&s_issued, j + 1);
            if (j == s_drop) return;  // failure-path test only
            const uint32_t k = kbase + j;
            const int s = k % S;
            unsigned char *sb = smem + s * L::STAGE_BYTES;
            const int bx = s_box[0], by = s_box[1], bz0 = s_box[2], q = bz0 - 2 + j;
            const bool with_target = q >= bz0 && q < s_box[3];
            mbar_arrive_expect_tx(&bars[s], 2 * L::U_BYTES + (with_target ? L::JT_BYTES + L::MASK_BYTES : 0));
            tma_load_4d(sb, s_tm[0], &bars[s], bx - TMA_HX, by - TMA_HY, q, 0);
            tma_load_4d(sb + L::G_OFF, s_tm[1], &bars[s], bx - TMA_HX, by - TMA_HY, q, 0);
            if (with_target) {
                tma_load_3d(sb + L::JT_OFF, s_tm[2], &bars[s], bx, by, q);
                tma_load_3d(sb + L::MASK_OFF, s_tm[3], &bars[s], bx, by, q);
            }
        };
        // This warp has read iteration j's stage for the last time; the last
        // warp to say so issues the loads of iteration j + S into the slot.
        auto release = [&](int j) {
            __syncwarp();
            if (lane == 0) {
                const int s = (kbase + j) % S;
                __threadfence_block();
                if (atomicAdd(&cnt[s], 1u) == (unsigned) (NW - 1)) {
                    cnt[s] = 0;
                    __threadfence_block();
                    fence_proxy_async_smem();
                    issue(j + S);
                }
            }
        };
        if (tid == 0) {
            for (int m = 0; m < 4; ++m) tmap_acquire(s_tm[m]);
            for (int j = 0; j < min(S, n_it); ++j) issue(j);
        }

        const int x = x0 + 2 * tx;       // this thread's columns: x, x + 1
        const int lx = 2 * tx + TMA_HX;  // their box column
        const bool pair_in = x + 1 < g.nx;
        const bool tile_x_in = x0 >= 2 && x0 + TXW - 1 <= g.nx - 3;
        // Own columns: candidate values of planes q-4 .. q (z differences).
        T zq[RYT][2][3][5];
#pragma unroll
        for (int r = 0; r < RYT; ++r)
#pragma unroll
            for (int v = 0; v < 2; ++v)
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int k = 0; k < 5; ++k) zq[r][v][c][k] = T(0);
        double acc_s = 0.0;
        T acc_mt = T(0);
        // Running pointers at the thread's first row: the candidate of plane
        // q in the other field buffer, e' of plane q - 2.
        const long long row0 = (long long) (y0 + ty) * g.ys + x;
        T *dq = V.field[old_b ^ 1] + (long long) (z0 - 2) * g.zs + row0;
        T *eq = V.ep[trial ? old_b ^ 1 : old_b] + (long long) (z0 - 4) * g.zs + row0;  // e' of the evaluated field
        for (int it = 0; it < n_it; ++it, dq += g.zs, eq += g.zs) {
            if (s_fault) break;
            const uint32_t k = kbase + it;
            if (!mbar_wait_bounded(&bars[k % S], (k / S) & 1u, s_wait)) {
                s_fault = 1;
                break;
            }
            const T *su = reinterpret_cast<const T *>(smem + (k % S) * L::STAGE_BYTES);
            const T *sg = su + L::G_OFF / (int) sizeof(T);
            const int q = z0 - 2 + it, ze = q - 2;
            // Own columns of plane q: shift the z-queues, store the candidate.
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                const int ly = ty + r * TYT + TMA_HY;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const auto nv = cand_pair(su, sg, c * TMA_PLANE + ly * TMA_PX + lx, eta_t);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        zq[r][0][c][kk] = zq[r][0][c][kk + 1];
                        zq[r][1][c][kk] = zq[r][1][c][kk + 1];
                    }
                    zq[r][0][c][4] = nv.x;
                    zq[r][1][c][4] = nv.y;
                }
                const int y = y0 + ty + r * TYT;
                if (trial && x < g.nx && y < g.ny && q >= z0 && q < z1) {
                    T *o = dq + (long long) (r * TYT) * g.ys;
                    if (pair_in) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) st_pair(o + c * g.cs, zq[r][0][c][4], zq[r][1][c][4]);
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; ++c) o[c * g.cs] = zq[r][0][c][4];
                    }
                }
            }
            if (ze >= z0 && ze < z1) {
                // Plane ze is iteration it - 2's stage.
                const unsigned char *se = smem + ((k - 2) % S) * L::STAGE_BYTES;
                const T *eu = reinterpret_cast<const T *>(se);
                const T *eg = eu + L::G_OFF / (int) sizeof(T);
                const bool plane_in = ze >= 2 && ze <= g.nz - 3;
                // Fourth-order weights with the spacing folded in (FP32); the
                // FP64 path keeps the reference's operation order.
                const T ih[3] = {s_ih[0], s_ih[1], s_ih[2]};
                const T k1[3] = {FD<T>::two_thirds * ih[0], FD<T>::two_thirds * ih[1], FD<T>::two_thirds * ih[2]};
                const T k2n[3] = {-FD<T>::one_twelfth * ih[0], -FD<T>::one_twelfth * ih[1],
                                  -FD<T>::one_twelfth * ih[2]};
                auto c4 = [&](T p1, T m1, T p2, T m2, int ax) -> T {
                    if constexpr (sizeof(T) == 4) return c4_folded(p1, m1, p2, m2, k1[ax], k2n[ax]);
                    return fd_c4<T>(p1, m1, p2, m2, ih[ax]);
                };
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    const int y = y0 + ty + r * TYT;
                    const bool row_in = plane_in && y >= 2 && y <= g.ny - 3;
                    const int ly = ty + r * TYT + TMA_HY;
                    if (x >= g.nx || y >= g.ny) continue;
                    const int ot = (ty + r * TYT) * TXW + 2 * tx;
                    const auto j2 = ld_pair(reinterpret_cast<const T *>(se + L::JT_OFF) + ot);
                    const unsigned short m2 = *reinterpret_cast<const unsigned short *>(se + L::MASK_OFF + ot);
                    const T jt[2] = {j2.x, j2.y};
                    const bool msk[2] = {(m2 & 0xffu) != 0, (m2 >> 8) != 0};
                    T epv[2];
                    // Error terms of voxel v from its Jacobian determinant.
                    auto finish_j = [&](int v, const T J) {
                        const T vv = voxel_error<T>(J, jt[v], msk[v], tol);
                        acc_s += (double) vv * (double) vv;
                        const T av = fabs(vv);  // the maximum is exact in the element type
                        if (msk[v] && av > acc_mt) acc_mt = av;
                        T ep = vv;
                        if (J < delta) ep += zeta * (J - delta);  // src/displacement_field_gradient.c:71-88
                        epv[v] = ep;
                    };
                    auto finish = [&](int v, const T (&a)[3][3]) { finish_j(v, det_i_plus<T>(a)); };
                    if (row_in && tile_x_in) {
                        // Row c of both voxels' matrices (fourth order throughout).
                        auto row = [&](int c, T (&m)[2][3]) {
                            const int o = c * TMA_PLANE + ly * TMA_PX + lx;
                            const T *zc0 = zq[r][0][c], *zc1 = zq[r][1][c];  // own values: planes ze-2 .. ze+2
                            const auto xm = cand_pair(eu, eg, o - 2, eta_t), xp = cand_pair(eu, eg, o + 2, eta_t);
                            m[0][0] = c4(zc1[2], xm.y, xp.x, xm.x, 0);
                            m[1][0] = c4(xp.x, zc0[2], xp.y, xm.y, 0);
                            const auto ym1 = cand_pair(eu, eg, o - TMA_PX, eta_t);
                            const auto yp1 = cand_pair(eu, eg, o + TMA_PX, eta_t);
                            const auto ym2 = cand_pair(eu, eg, o - 2 * TMA_PX, eta_t);
                            const auto yp2 = cand_pair(eu, eg, o + 2 * TMA_PX, eta_t);
                            m[0][1] = c4(yp1.x, ym1.x, yp2.x, ym2.x, 1);
                            m[1][1] = c4(yp1.y, ym1.y, yp2.y, ym2.y, 1);
                            m[0][2] = c4(zc0[3], zc0[1], zc0[4], zc0[0], 2);
                            m[1][2] = c4(zc1[3], zc1[1], zc1[4], zc1[0], 2);
                        };
                        // det_i_plus's operations in its order, rows 1 and 2
                        // folded into the cofactors of row 0 before row 0 is
                        // formed, so fewer values are live at once.
                        T cf[2][3];
                        {
                            T m1[2][3], m2[2][3];
                            row(1, m1);
                            row(2, m2);
#pragma unroll
                            for (int v = 0; v < 2; ++v) {
                                const T a21 = m1[v][0], a22 = m1[v][1] + T(1.0), a23 = m1[v][2];
                                const T a31 = m2[v][0], a32 = m2[v][1], a33 = m2[v][2] + T(1.0);
                                cf[v][0] = a22 * a33 - a23 * a32;
                                cf[v][1] = a21 * a33 - a23 * a31;
                                cf[v][2] = a21 * a32 - a22 * a31;
                            }
                        }
                        T m0[2][3];
                        row(0, m0);
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            const T a11 = m0[v][0] + T(1.0), a12 = m0[v][1], a13 = m0[v][2];
                            finish_j(v, a11 * cf[v][0] - a12 * cf[v][1] + a13 * cf[v][2]);
                        }
                    } else {
                        // Interior rows of a tile that reaches an x end, and the
                        // two outer layers: the case analysis per voxel
                        // (src/jacobian.c:113-241), taps formed one by one.
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            const int xv = x + v;
                            if (xv >= g.nx) continue;
                            auto tap = [&](int c, int d) -> T {
                                const int o = c * TMA_PLANE + ly * TMA_PX + lx + v + d;
                                return eu[o] - eta_t * eg[o];
                            };
                            T a[3][3];
                            if (row_in) {
                                const bool xo_lo = xv == 0, xo_hi = xv == g.nx - 1;
                                const bool second = xo_lo || xo_hi || xv == 1 || xv == g.nx - 2;
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    const T p0 = zq[r][v][c][2];
                                    const T pm1 = tap(c, -1), pp1 = tap(c, 1), pm2 = tap(c, -2), pp2 = tap(c, 2);
                                    const T fx = xo_lo ? fd_fwd<T>(p0, pp1, pp2, ih[0])
                                                       : (xo_hi ? fd_bwd<T>(p0, pm1, pm2, ih[0])
                                                                : fd_c2<T>(pp1, pm1, ih[0]));
                                    const T cx4 = c4(pp1, pm1, pp2, pm2, 0);
                                    a[c][0] = second ? fx : cx4;
                                    const T ym1 = tap(c, -TMA_PX), yp1 = tap(c, TMA_PX);
                                    const T ym2 = tap(c, -2 * TMA_PX), yp2 = tap(c, 2 * TMA_PX);
                                    const T cy4 = c4(yp1, ym1, yp2, ym2, 1);
                                    const T cy2 = fd_c2<T>(yp1, ym1, ih[1]);
                                    a[c][1] = second ? cy2 : cy4;
                                    const T *zv = zq[r][v][c];
                                    const T cz4 = c4(zv[3], zv[1], zv[4], zv[0], 2);
                                    const T cz2 = fd_c2<T>(zv[3], zv[1], ih[2]);
                                    a[c][2] = second ? cz2 : cz4;
                                }
                            } else {
                                int kk[3];
                                schemes_at(xv, y, ze, g, kk);
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    const T p0 = zq[r][v][c][2];
                                    const T vx[5] = {tap(c, -2), tap(c, -1), p0, tap(c, 1), tap(c, 2)};
                                    const T vy[5] = {tap(c, -2 * TMA_PX), tap(c, -TMA_PX), p0, tap(c, TMA_PX),
                                                     tap(c, 2 * TMA_PX)};
#pragma unroll
                                    for (int ax = 0; ax < 3; ++ax) {
                                        const T *w = ax == 0 ? vx : (ax == 1 ? vy : zq[r][v][c]);
                                        T d;
                                        switch (kk[ax]) {
                                        case S_FWD: d = fd_fwd<T>(w[2], w[3], w[4], ih[ax]); break;
                                        case S_BWD: d = fd_bwd<T>(w[2], w[1], w[0], ih[ax]); break;
                                        case S_C2: d = fd_c2<T>(w[3], w[1], ih[ax]); break;
                                        default: d = c4(w[3], w[1], w[4], w[0], ax); break;
                                        }
                                        a[c][ax] = d;
                                    }
                                }
                            }
                            finish(v, a);
                        }
                    }
                    T *o = eq + (long long) (r * TYT) * g.ys;
                    if (pair_in)
                        st_pair(o, epv[0], epv[1]);
                    else
                        o[0] = epv[0];
                }
            }
            // Iteration it - 2's stage is not read again; count out of it
            // when its slot has a later plane of this tile to take.
            if (it >= 2 && it - 2 + S < n_it) release(it - 2);
        }
        __syncthreads();  // every warp has left the plane loop
        if (s_fault) {
            if (tid == 0) {
                atomicExch(&st->fault, 1);
                atomicExch(&st->done, 1);
                // The last load issued into each slot: wait (bounded) until it
                // has landed, so nothing arrives after the block has left.
                const int to = s_issued;
                for (int j = max(0, to - S); j < to; ++j) {
                    const uint32_t kk = kbase + j;
                    mbar_wait_bounded(&bars[kk % S], (kk / S) & 1u, 1u << 16);
                }
            }
            __syncthreads();
            return;
        }
        kbase += n_it;

        const double2 rr = block_reduce_n<NTH, TPX>(acc_s, (double) acc_mt, red);
        if (tid == 0) V.part_t[lt] = rr;
        if (publish_partial_n<TPX>(&st->ticket_t, V.ntiles, &s_flag)) {
            // Each thread folds a fixed subset of the tile partials, so the
            // total does not depend on timing.
            double ssum = 0.0, smax = 0.0;
            for (int i = tid; i < V.ntiles; i += NTH) {
                const double2 pp = __ldcg(&V.part_t[i]);
                ssum += pp.x;
                smax = fmax(smax, pp.y);
            }
            const double2 tot = block_reduce_n<NTH, TPX>(ssum, smax, red);
            if (tid == 0) {
                st->ticket_t = 0;
                control_after_trial(st, tot.x, tot.y);
                if (work_flag) *work_flag = 1;
                __threadfence();
            }
        }
        __syncthreads();
    }
}

template <typename T, int TXW, int TYT>
cudaError_t launch_trial_rel_v(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                               cudaStream_t s, unsigned char *work_flag, TileQueue *queue) {
    constexpr int smem = TrialRelLayout<T, TXW>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_trial_rel<T, TXW, TYT>, smem, devs);
    if (attr != cudaSuccess) return attr;
    k_trial_rel<T, TXW, TYT><<<grid, dim3(TXW / 2, TYT), smem, s>>>(vols, tile_vol, total_tiles, work_flag, queue);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int TXW, int TYT>
int trial_rel_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_trial_rel<T, TXW, TYT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TrialRelLayout<T, TXW>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_trial_rel<T, TXW, TYT>, TXW / 2 * TYT,
                                                      TrialRelLayout<T, TXW>::BYTES + 128);
        return v;
    }();
    return n;
}

template <typename T, int TXW, int TYT>
cudaError_t launch_trial_tma_v(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                               cudaStream_t s, unsigned char *work_flag, TileQueue *queue, int pf) {
    constexpr int smem = TrialTmaLayout<T, TXW>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_trial_tma<T, TXW, TYT>, smem, devs);
    if (attr != cudaSuccess) return attr;
    k_trial_tma<T, TXW, TYT><<<grid, dim3(TXW / 2, TYT), smem, s>>>(vols, tile_vol, total_tiles, work_flag, queue,
                                                                     pf);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int TXW, int TYT>
cudaError_t launch_greedy_tma_v(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                                cudaStream_t s, unsigned char *work_flag, TileQueue *queue) {
    constexpr int smem = TrialTmaLayout<T, TXW, true>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_trial_tma<T, TXW, TYT, true>, smem, devs);
    if (attr != cudaSuccess) return attr;
    k_trial_tma<T, TXW, TYT, true><<<grid, dim3(TXW / 2, TYT), smem, s>>>(vols, tile_vol, total_tiles, work_flag,
                                                                           queue, 0);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int TXW, int TYT>
cudaError_t launch_gradient_tma_v(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                                  cudaStream_t s, unsigned char *work_flag, TileQueue *queue, int pf) {
    constexpr int smem = GradTmaLayout<T, TXW>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_gradient_tma<T, TXW, TYT>, smem, devs);
    if (attr != cudaSuccess) return attr;
    k_gradient_tma<T, TXW, TYT><<<grid, dim3(TXW / 2, TYT + grad_halo_rows<TXW>()), smem, s>>>(
        vols, tile_vol, total_tiles, work_flag, queue, pf);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int TXW, int TYT>
int trial_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_trial_tma<T, TXW, TYT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TrialTmaLayout<T, TXW>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_trial_tma<T, TXW, TYT>, TXW / 2 * TYT,
                                                      TrialTmaLayout<T, TXW>::BYTES + 128);
        return v;
    }();
    return n;
}
template <typename T, int TXW, int TYT>
int greedy_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_trial_tma<T, TXW, TYT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TrialTmaLayout<T, TXW, true>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_trial_tma<T, TXW, TYT, true>, TXW / 2 * TYT,
                                                      TrialTmaLayout<T, TXW, true>::BYTES + 128);
        return v;
    }();
    return n;
}
template <typename T, int TXW, int TYT>
int gradient_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_gradient_tma<T, TXW, TYT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GradTmaLayout<T, TXW>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_gradient_tma<T, TXW, TYT>,
                                                      TXW / 2 * (TYT + grad_halo_rows<TXW>()),
                                                      GradTmaLayout<T, TXW>::BYTES + 128);
        return v;
    }();
    return n;
}

// Tile shapes (tile_x x TT_Y voxels).  Trial kernel: tile_x / 2 x threads_y
// threads of TT_Y / threads_y rows and two columns each:
//   tile_x 32, threads_y 16  default, 256 threads (two blocks per SM for FP32)
//   tile_x 32, threads_y 8   128 threads of two rows (four voxels) each
//   tile_x 64, threads_y 16  FP32 only, 512 threads, one block per SM
// Gradient kernel: tile_x / 2 x threads_y threads of TT_Y / threads_y rows
// and two columns each:
//   tile_x 32, threads_y 16  default, 256 threads of one row
//   tile_x 32, threads_y 8   128 threads of two rows
//   tile_x 64, threads_y 8   FP32 only, 256 threads of two rows
template <typename T>
cudaError_t launch_trial_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                             cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y, TileQueue *q,
                             int pf) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64)
            return launch_trial_tma_v<T, 64, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
    if (threads_y == 8) return launch_trial_tma_v<T, 32, 8>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
    return launch_trial_tma_v<T, 32, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
}

// Trial kernel without the per-plane barrier (same tile shapes as
// launch_trial_tma, no L2 prefetch option).
template <typename T>
cudaError_t launch_trial_rel(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                             cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y, TileQueue *q) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64) return launch_trial_rel_v<T, 64, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q);
    if (threads_y == 8) return launch_trial_rel_v<T, 32, 8>(vols, tile_vol, total_tiles, grid, s, work_flag, q);
    return launch_trial_rel_v<T, 32, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q);
}

template <typename T>
int trial_rel_blocks_per_sm(int tile_x, int threads_y) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64) return trial_rel_blocks_v<T, 64, 16>();
    return threads_y == 8 ? trial_rel_blocks_v<T, 32, 8>() : trial_rel_blocks_v<T, 32, 16>();
}

template <typename T>
cudaError_t launch_gradient_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                                cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y, TileQueue *q,
                                int pf) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64)
            return launch_gradient_tma_v<T, 64, 8>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
    if (threads_y == 16)
        return launch_gradient_tma_v<T, 32, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
    return launch_gradient_tma_v<T, 32, 8>(vols, tile_vol, total_tiles, grid, s, work_flag, q, pf);
}

// Greedy trial: tile 32 x TT_Y, 16 x 16 threads.
template <typename T>
cudaError_t launch_greedy_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                              cudaStream_t s, unsigned char *work_flag, TileQueue *q) {
    return launch_greedy_tma_v<T, 32, 16>(vols, tile_vol, total_tiles, grid, s, work_flag, q);
}
template <typename T>
int greedy_tma_blocks_per_sm() {
    return greedy_blocks_v<T, 32, 16>();
}

template <typename T>
int trial_tma_blocks_per_sm(int tile_x, int threads_y) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64) return trial_blocks_v<T, 64, 16>();
    return threads_y == 8 ? trial_blocks_v<T, 32, 8>() : trial_blocks_v<T, 32, 16>();
}
template <typename T>
int gradient_tma_blocks_per_sm(int tile_x, int threads_y) {
    if constexpr (sizeof(T) == 4)
        if (tile_x == 64) return gradient_blocks_v<T, 64, 8>();
    return threads_y == 16 ? gradient_blocks_v<T, 32, 16>() : gradient_blocks_v<T, 32, 8>();
}

// ------------------------------------------------------------------------
// Jacobian map of one field with the TMA pipeline (src/jacobian.c:70-242,
// fourth-order interior): J = det(I + grad u) into jout.
//
// A block of TXW / 2 x TYT threads marches a TXW x TT_Y tile through bz
// planes.  Field boxes (tile + 4 voxels in x, 2 rows in y, three components)
// go straight into S shared-memory stages and stay there until their plane
// has been the stencil's centre plane, so no candidate plane is formed.
// Threads wait for each stage's mbarrier themselves; the block barrier only
// guards stage reuse and is taken every B planes.  At the barrier of
// iteration it every warp has finished iteration it-1, so the loads of
// iterations it+LA .. it+LA+B-1 (LA + B = S - 2) go into stages whose planes
// were last read, as a stencil's centre plane, by iteration it-1.  Each
// thread keeps its two columns of planes ze-2 .. ze+2 in registers for the
// z differences.  The tensor map is a kernel parameter and tiles are dealt
// round-robin (one volume, uniform tiles), so a launch needs no device
// memory of its own.  A load that does not arrive within the bound leaves
// NaN in the rest of the block's tile (no endless wait).
// ------------------------------------------------------------------------
template <typename T, int TXW>
struct JacTmaLayout {
    static constexpr int TMA_PX = Box<TXW>::PX;
    static constexpr int TMA_PLANE = Box<TXW>::PLANE;
    static constexpr int S = 10;   // stages: 96 KB (FP32, two blocks per SM), 192 KB (FP64, one)
    static constexpr int B = 4;    // planes between block barriers
    static constexpr int LA = S - 2 - B;  // first load distance: loads of it+LA .. it+LA+B-1 at a barrier
    static constexpr int U_BYTES = 3 * TMA_PLANE * (int) sizeof(T);
    static constexpr int BAR_OFF = S * U_BYTES;
    static constexpr int BYTES = BAR_OFF + S * 8;
    static_assert(U_BYTES % 128 == 0, "stages stay 128-byte aligned");
};

//
// ADJ instantiates the weight pass of the Jacobian's adjoint instead: with
// w = gJ(p), W[c][a](p) = w * cof_ca(I + A(p)) * ih_a for the stencil matrix
// A(p), W dense with component stride wn (the gather pass follows).
// COF (the differentiable Jacobian's forward) writes the map and, into W,
// C[c][a](p) = cof_ca(I + A(p)) * ih_a, so that the backward needs only the
// gather, with W = gJ * C formed there.
template <typename T, int TXW, int TYT, bool ADJ = false, bool COF = false>
__global__ void __launch_bounds__(TXW / 2 * TYT, sizeof(T) == 4 ? 2 : 1)
    k_jacobian_tma(const __grid_constant__ CUtensorMap tm_u, const Geom g, T *__restrict__ jout, long long jys,
                   long long jzs, int tiles_x, int tiles_y, int ntiles, int bz, const T *__restrict__ gJ,
                   T *__restrict__ W, long long wn) {
    using L = JacTmaLayout<T, TXW>;
    constexpr int TPX = TXW / 2, RYT = TT_Y / TYT;
    constexpr int TMA_PX = L::TMA_PX, TMA_PLANE = L::TMA_PLANE, S = L::S, LA = L::LA;
    static_assert(TPX <= 32 && 32 % TPX == 0, "a warp spans whole tile rows");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    __shared__ int s_fault;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx;
    if (tid == 0) {
        for (int k = 0; k < S; ++k) mbar_init(&bars[k], 1);
        fence_mbar_init();
        tmap_prefetch(&tm_u);
        s_fault = 0;
    }
    __syncthreads();
    const T ih[3] = {(T) g.ih[0], (T) g.ih[1], (T) g.ih[2]};
    uint32_t kbase = 0;  // iterations consumed by this block (mbarrier phases)

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int txi = tile % tiles_x, tyi = (tile / tiles_x) % tiles_y, tzi = tile / (tiles_x * tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * bz;
        const int z1 = min(z0 + bz, g.nz);
        const int n_it = z1 - z0 + 4;  // planes z0-2 .. z1+1
        // Every warp has finished the previous tile, whose stages the first
        // loads below overwrite.
        __syncthreads();
        int issued_n = 0;
        auto issue = [&](int j) {
            issued_n = j + 1;
            const uint32_t k = kbase + j;
            uint64_t *bar = &bars[k % S];
            mbar_arrive_expect_tx(bar, L::U_BYTES);
            tma_load_4d(smem + (k % S) * L::U_BYTES, &tm_u, bar, x0 - TMA_HX, y0 - TMA_HY, z0 - 2 + j, 0);
        };
        if (tid == 0)
            for (int j = 0; j < min(LA, n_it); ++j) issue(j);

        const int x = x0 + 2 * tx;       // this thread's columns: x, x + 1
        const int lx = 2 * tx + TMA_HX;  // their box column
        const bool pair_in = x + 1 < g.nx;
        // Own columns (x, x + 1 as one pair): field values of planes ze-2 .. ze+2.
        using P2 = typename PairOf<T>::type;
        P2 zq[RYT][3][5];
#pragma unroll
        for (int r = 0; r < RYT; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 5; ++k) zq[r][c][k] = P2{T(0), T(0)};
        const bool tile_x_in = x0 >= 2 && x0 + TXW - 1 <= g.nx - 3;
        T wnext[RYT][2];  // adjoint weights: gJ of the next plane
#pragma unroll
        for (int r = 0; r < RYT; ++r) wnext[r][0] = wnext[r][1] = T(0);
        bool failed = false;
        int fail_it = 0;
        for (int it = 0; it < n_it; ++it) {
            const uint32_t k = kbase + it;
            if (it % L::B == 0) {
                __syncthreads();
                if (s_fault) {
                    failed = true;
                    fail_it = it;
                    break;
                }
                if (tid == 0)
                    for (int j = it + LA; j < min(it + LA + L::B, n_it); ++j) issue(j);
            }
            // A load that does not arrive stops the block at the next barrier
            // (this plane's values are not used then).
            if (!mbar_wait_bounded(&bars[k % S], (k / S) & 1u)) s_fault = 1;
            const T *sb = reinterpret_cast<const T *>(smem + (k % S) * L::U_BYTES);
            const int q = z0 - 2 + it, ze = q - 2;
            // Adjoint weights: this plane's gJ, loaded an iteration ahead,
            // and the load of the next plane's.
            T wcur[RYT][2];
            if (ADJ) {
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    wcur[r][0] = wnext[r][0];
                    wcur[r][1] = wnext[r][1];
                    const int y = y0 + ty + r * TYT;
                    if (ze + 1 >= z0 && ze + 1 < z1 && x < g.nx && y < g.ny) {
                        const long long off = (ze + 1) * jzs + y * jys + x;
                        if (pair_in) {
                            const auto w2 = ld_pair(gJ + off);
                            wnext[r][0] = w2.x;
                            wnext[r][1] = w2.y;
                        } else {
                            wnext[r][0] = gJ[off];
                            wnext[r][1] = T(0);
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                const int ly = ty + r * TYT + TMA_HY;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) zq[r][c][kk] = zq[r][c][kk + 1];
                    zq[r][c][4] = ld_pair(sb + c * TMA_PLANE + ly * TMA_PX + lx);
                }
            }
            if (ze < z0 || ze >= z1) continue;
            const T *jp = reinterpret_cast<const T *>(smem + ((k - 2) % S) * L::U_BYTES);  // plane ze
            const bool plane_in = ze >= 2 && ze <= g.nz - 3;
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                const int y = y0 + ty + r * TYT;
                if (x >= g.nx || y >= g.ny) continue;
                const bool row_in = plane_in && y >= 2 && y <= g.ny - 3;
                const long long off = ze * jzs + y * jys + x;
                if (ADJ) {
                    const T w[2] = {wcur[r][0], wcur[r][1]};
                    T wv[9][2];
                    // FP32 states every rounding (the scalar and the paired
                    // epilogues give the same bits): a minor is a difference
                    // of two products, and w * cof * ih is (w * minor) * (+-ih).
                    auto weights = [&](int v, const T (&a)[3][3]) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const int c0 = b == 0 ? 1 : 0, c1 = b == 2 ? 1 : 2;
                                if constexpr (sizeof(T) == 4) {
                                    auto m = [&](int i, int j) { return i == j ? __fadd_rn(a[i][j], 1.f) : a[i][j]; };
                                    const float minor =
                                        __fsub_rn(__fmul_rn(m(r0, c0), m(r1, c1)), __fmul_rn(m(r0, c1), m(r1, c0)));
                                    wv[c * 3 + b][v] = __fmul_rn(__fmul_rn(w[v], minor), ((c + b) & 1) ? -ih[b] : ih[b]);
                                } else {
                                    const T m00 = a[r0][c0] + (r0 == c0 ? T(1) : T(0));
                                    const T m11 = a[r1][c1] + (r1 == c1 ? T(1) : T(0));
                                    const T m01 = a[r0][c1] + (r0 == c1 ? T(1) : T(0));
                                    const T m10 = a[r1][c0] + (r1 == c0 ? T(1) : T(0));
                                    const T minor = m00 * m11 - m01 * m10;
                                    const T cof = ((c + b) & 1) ? -minor : minor;
                                    wv[c * 3 + b][v] = w[v] * cof * ih[b];
                                }
                            }
                        }
                    };
                    auto weights2 = [&](const auto &a) {
                        const float2 w2 = make_float2(w[0], w[1]);
                        auto m = [&](int i, int j) { return i == j ? p_add(a[i][j], p_splat(1.f)) : a[i][j]; };
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const int c0 = b == 0 ? 1 : 0, c1 = b == 2 ? 1 : 2;
                                const float2 minor = p_sub(p_mul(m(r0, c0), m(r1, c1)), p_mul(m(r0, c1), m(r1, c0)));
                                const float2 wq2 =
                                    p_mul(p_mul(w2, minor), p_splat(((c + b) & 1) ? -ih[b] : ih[b]));
                                wv[c * 3 + b][0] = wq2.x;
                                wv[c * 3 + b][1] = wq2.y;
                            }
                        }
                    };
                    stencil_pair<T, TMA_PX, TMA_PLANE>(zq[r], jp, lx, ty + r * TYT + TMA_HY, x, y, ze, g, ih, row_in,
                                                       tile_x_in, weights, weights2);
#pragma unroll
                    for (int k = 0; k < 9; ++k) {
                        if (pair_in)
                            st_pair(W + k * wn + off, wv[k][0], wv[k][1]);
                        else
                            W[k * wn + off] = wv[k][0];
                    }
                } else {
                    T jv[2];
                    T cv[COF ? 9 : 1][2];
                    // C[c][b] = cof_cb(I + a) * ih_b: a minor (difference of
                    // two products) times +-ih_b, as the weight epilogue
                    // rounds it before its factor w.
                    auto det2 = [&](const auto &a) {
                        const auto J = det_i_plus2(a);
                        jv[0] = J.x;
                        jv[1] = J.y;
                        if constexpr (COF) {
                            auto m = [&](int i, int j) { return i == j ? p_add(a[i][j], p_splat(1.f)) : a[i][j]; };
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
#pragma unroll
                                for (int b = 0; b < 3; ++b) {
                                    const int c0 = b == 0 ? 1 : 0, c1 = b == 2 ? 1 : 2;
                                    const float2 minor =
                                        p_sub(p_mul(m(r0, c0), m(r1, c1)), p_mul(m(r0, c1), m(r1, c0)));
                                    const float2 q = p_mul(minor, p_splat(((c + b) & 1) ? -ih[b] : ih[b]));
                                    cv[c * 3 + b][0] = q.x;
                                    cv[c * 3 + b][1] = q.y;
                                }
                            }
                        }
                    };
                    auto det1 = [&](int v, const T (&a)[3][3]) {
                        jv[v] = det_i_plus<T>(a);
                        if constexpr (COF) {
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
#pragma unroll
                                for (int b = 0; b < 3; ++b) {
                                    const int c0 = b == 0 ? 1 : 0, c1 = b == 2 ? 1 : 2;
                                    const T m00 = a[r0][c0] + (r0 == c0 ? T(1) : T(0));
                                    const T m11 = a[r1][c1] + (r1 == c1 ? T(1) : T(0));
                                    const T m01 = a[r0][c1] + (r0 == c1 ? T(1) : T(0));
                                    const T m10 = a[r1][c0] + (r1 == c0 ? T(1) : T(0));
                                    const T ihs = ((c + b) & 1) ? -ih[b] : ih[b];
                                    if constexpr (sizeof(T) == 4)
                                        cv[c * 3 + b][v] =
                                            __fmul_rn(__fsub_rn(__fmul_rn(m00, m11), __fmul_rn(m01, m10)), ihs);
                                    else cv[c * 3 + b][v] = (m00 * m11 - m01 * m10) * ihs;
                                }
                            }
                        }
                    };
                    stencil_pair<T, TMA_PX, TMA_PLANE>(zq[r], jp, lx, ty + r * TYT + TMA_HY, x, y, ze, g, ih,
                                                       row_in, tile_x_in, det1, det2);
                    T *o = jout + off;
                    if (pair_in)
                        st_pair(o, jv[0], jv[1]);
                    else
                        o[0] = jv[0];
                    if constexpr (COF) {
#pragma unroll
                        for (int k = 0; k < 9; ++k) {
                            if (pair_in)
                                st_pair(W + k * wn + off, cv[k][0], cv[k][1]);
                            else
                                W[k * wn + off] = cv[k][0];
                        }
                    }
                }
            }
        }
        if (failed) {
            // Wait (bounded) for the loads still in flight, mark the tile's
            // planes NaN and leave.
            if (tid == 0)
                for (int j = max(0, fail_it - L::B); j < issued_n; ++j) {
                    const uint32_t kk = kbase + j;
                    mbar_wait_bounded(&bars[kk % S], (kk / S) & 1u, 1u << 16);
                }
            const T nan = T(NAN);
            for (int ze = z0; ze < z1; ++ze)
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    const int y = y0 + ty + r * TYT;
                    if (y >= g.ny) continue;
                    for (int v = 0; v < 2; ++v) {
                        if (x + v >= g.nx) continue;
                        const long long off = ze * jzs + y * jys + x + v;
                        if (ADJ || COF)
                            for (int k = 0; k < 9; ++k) W[k * wn + off] = nan;
                        if (!ADJ) jout[off] = nan;
                    }
                }
            __syncthreads();
            return;
        }
        kbase += n_it;
    }
}

template <typename T, int TXW, int TYT, bool ADJ, bool COF>
int jacobian_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_jacobian_tma<T, TXW, TYT, ADJ, COF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             JacTmaLayout<T, TXW>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_jacobian_tma<T, TXW, TYT, ADJ, COF>, TXW / 2 * TYT,
                                                      JacTmaLayout<T, TXW>::BYTES + 128);
        return v;
    }();
    return n;
}

// Jacobian map (or adjoint weights) of the field `tm_u` describes (geometry
// g, order 4) into jout (strides jys, jzs): tiles of 32 x TT_Y voxels, 16 x 16 threads, as many
// blocks as fit on the device.  Tiles are dealt round-robin, so the z split
// is chosen to fill whole waves of the grid: about 32 planes a tile, then as
// many z tiles per column as fit in that many waves (at least 8 planes a
// tile, since each tile also loads 4 halo planes).
template <typename T, bool ADJ, bool COF>
cudaError_t launch_jacobian_tma_v(const CUtensorMap &tm_u, const Geom &g, T *jout, long long jys, long long jzs,
                                  int num_sms, cudaStream_t s, const T *gJ, T *W, long long wn) {
    constexpr int TXW = 32, TYT = 16, BZ = 32;
    constexpr int smem = JacTmaLayout<T, TXW>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_jacobian_tma<T, TXW, TYT, ADJ, COF>, smem, devs);
    if (attr != cudaSuccess) return attr;
    const int tiles_x = (g.nx + TXW - 1) / TXW, tiles_y = (g.ny + TT_Y - 1) / TT_Y;
    const int cols = tiles_x * tiles_y;
    const int slots = std::max(1, jacobian_blocks_v<T, TXW, TYT, ADJ, COF>()) * num_sms;  // resident blocks
    int nzt = (g.nz + BZ - 1) / BZ;                                             // z tiles per column
    const int waves = (cols * nzt + slots - 1) / slots;
    nzt = std::min((g.nz + 7) / 8, std::max(nzt, waves * slots / cols));  // at least 8 planes a tile
    const int bz = (g.nz + nzt - 1) / nzt;
    const int ntiles = cols * ((g.nz + bz - 1) / bz);
    const int grid = std::min(ntiles, slots);
    k_jacobian_tma<T, TXW, TYT, ADJ, COF><<<grid, dim3(TXW / 2, TYT), smem, s>>>(tm_u, g, jout, jys, jzs, tiles_x,
                                                                                tiles_y, ntiles, bz, gJ, W, wn);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_jacobian_tma(const CUtensorMap &tm_u, const Geom &g, T *jout, long long jys, long long jzs,
                                int num_sms, cudaStream_t s, const T *gJ, T *W, long long wn) {
    if (W && gJ) return launch_jacobian_tma_v<T, true, false>(tm_u, g, jout, jys, jzs, num_sms, s, gJ, W, wn);
    if (W) return launch_jacobian_tma_v<T, false, true>(tm_u, g, jout, jys, jzs, num_sms, s, gJ, W, wn);
    return launch_jacobian_tma_v<T, false, false>(tm_u, g, jout, jys, jzs, num_sms, s, gJ, W, wn);
}

// ------------------------------------------------------------------------
// k_gather_tma: the gather pass of the adjoint,
//   grad_c(q) = sum_a sum_t W[c][a](q - t e_a) * kappa(k_a(q - t e_a), t)
// (the same taps, coefficients and summation order as k_adjoint_gather), on
// weights streamed by TMA.  W is [c][a][wn] with the field's row and plane
// strides.  A 32 x TT_Y tile marches through its z range; the stage of plane
// q holds W[.][z] of the tile at plane q and, for the gradient plane
// ze = q - 2, W[.][x] of the tile's rows with four columns each side and
// W[.][y] of its columns with two rows each side.  Each thread keeps its
// pair's W[.][z] of planes ze-2 .. ze+2 in registers.  A stage is consumed
// in its own iteration, so a block barrier every B planes is all that
// guards reuse (loads run LA = S - B iterations ahead).  Warps whose pairs
// all have their taps at fourth-order voxels (four or more voxels from
// every face) take constant coefficients; warps near an x face take
// per-lane coefficients for the x taps (both as FP32 pairs); the others
// choose each tap's coefficient by the tap voxel's scheme.
// ------------------------------------------------------------------------
// GJ: the stages hold C (the weights without their factor gJ) and two boxes
// of gJ (TXW + 8 columns, TT_Y + 4 rows) at planes ze and q, and each weight
// is formed as gJ * C where it is read.
template <typename T, int TXW, bool GJ = false>
struct GatherTmaLayout {
    static constexpr int XPX = TXW + 2 * TMA_HX;  // W[.][x] box: TXW + 8 columns, TT_Y rows
    static constexpr int X_ELEMS = 3 * TT_Y * XPX;
    static constexpr int YPY = TT_Y + 2 * TMA_HY;  // W[.][y] box: TXW columns, TT_Y + 4 rows
    static constexpr int Y_ELEMS = 3 * YPY * TXW;
    static constexpr int Z_ELEMS = 3 * TT_Y * TXW;  // W[.][z] box: the tile
    static constexpr int G_ELEMS = YPY * XPX;       // a gJ box
    static constexpr int X_OFF = 0;
    static constexpr int Y_OFF = X_ELEMS * (int) sizeof(T);
    static constexpr int Z_OFF = Y_OFF + Y_ELEMS * (int) sizeof(T);
    static constexpr int G_BYTES = (G_ELEMS * (int) sizeof(T) + 127) / 128 * 128;
    static constexpr int GE_OFF = (Z_OFF + Z_ELEMS * (int) sizeof(T) + 127) / 128 * 128;  // gJ at ze
    static constexpr int GQ_OFF = GE_OFF + G_BYTES;                                        // gJ at q
    static constexpr int STAGE_BYTES = GJ ? GQ_OFF + G_BYTES : GE_OFF;
    // 63 KB (FP32, three blocks per SM; GJ: two stages, 56 KB), 168 KB (FP64)
    static constexpr int S = sizeof(T) == 4 ? (GJ ? 2 : 3) : 4;
    static constexpr int B = sizeof(T) == 4 ? 1 : 2;  // planes between block barriers
    static constexpr int LA = S - B;                  // load distance
    static constexpr int BAR_OFF = S * STAGE_BYTES;
    static constexpr int BYTES = BAR_OFF + S * 8;
    static_assert(Y_OFF % 128 == 0 && Z_OFF % 128 == 0, "boxes start 128-byte aligned");
};

template <typename T, int TXW, int TYT, bool GJ = false>
__global__ void __launch_bounds__(TXW / 2 * TYT, sizeof(T) == 4 ? 3 : 1)
    k_gather_tma(const __grid_constant__ CUtensorMap tm_wx, const __grid_constant__ CUtensorMap tm_wy,
                 const __grid_constant__ CUtensorMap tm_wz, const __grid_constant__ CUtensorMap tm_gj, const Geom g,
                 T *__restrict__ gout, int tiles_x, int tiles_y, int ntiles, int bz) {
    using L = GatherTmaLayout<T, TXW, GJ>;
    using P2 = typename PairOf<T>::type;
    constexpr int TPX = TXW / 2, RYT = TT_Y / TYT, S = L::S, LA = L::LA, XPX = L::XPX, YPY = L::YPY;
    static_assert(TPX <= 32 && 32 % TPX == 0, "a warp spans whole tile rows");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    __shared__ int s_fault;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx;
    if (tid == 0) {
        for (int k = 0; k < S; ++k) mbar_init(&bars[k], 1);
        fence_mbar_init();
        tmap_prefetch(&tm_wx);
        tmap_prefetch(&tm_wy);
        tmap_prefetch(&tm_wz);
        if (GJ) tmap_prefetch(&tm_gj);
        s_fault = 0;
    }
    __syncthreads();
    const int n[3] = {g.nx, g.ny, g.nz};
    // Fourth-order coefficients kappa(S_C4, t) by tap, t = -2, -1, 1, 2.
    const T kc[4] = {FD<T>::one_twelfth, -FD<T>::two_thirds, FD<T>::two_thirds, -FD<T>::one_twelfth};
    uint32_t kbase = 0;  // iterations consumed by this block (mbarrier phases)

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int txi = tile % tiles_x, tyi = (tile / tiles_x) % tiles_y, tzi = tile / (tiles_x * tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * bz;
        const int z1 = min(z0 + bz, g.nz);
        const int n_it = z1 - z0 + 4;  // W[.][z] planes z0-2 .. z1+1
        __syncthreads();  // every warp has left the previous tile's stages
        int issued_n = 0;
        auto issue = [&](int j) {
            issued_n = j + 1;
            const uint32_t k = kbase + j;
            uint64_t *bar = &bars[k % S];
            unsigned char *sb = smem + (k % S) * L::STAGE_BYTES;
            const int q = z0 - 2 + j, ze = q - 2;
            const bool with_xy = ze >= z0 && ze < z1;
            const int elems = L::Z_ELEMS + (with_xy ? L::X_ELEMS + L::Y_ELEMS : 0) +
                              (GJ ? L::G_ELEMS * (with_xy ? 2 : 1) : 0);
            mbar_arrive_expect_tx(bar, (uint32_t) (elems * sizeof(T)));
            tma_load_5d(sb + L::Z_OFF, &tm_wz, bar, x0, y0, q, 2, 0);
            if (GJ) tma_load_3d(sb + L::GQ_OFF, &tm_gj, bar, x0 - TMA_HX, y0 - TMA_HY, q);
            if (with_xy) {
                tma_load_5d(sb + L::X_OFF, &tm_wx, bar, x0 - TMA_HX, y0, ze, 0, 0);
                tma_load_5d(sb + L::Y_OFF, &tm_wy, bar, x0, y0 - TMA_HY, ze, 1, 0);
                if (GJ) tma_load_3d(sb + L::GE_OFF, &tm_gj, bar, x0 - TMA_HX, y0 - TMA_HY, ze);
            }
        };
        if (tid == 0)
            for (int j = 0; j < min(LA, n_it); ++j) issue(j);

        const int x = x0 + 2 * tx;  // this thread's columns: x, x + 1
        const bool pair_in = x + 1 < g.nx;
        // Own pair's W[c][z] of planes q-4 .. q (index 2 - t holds plane ze - t).
        P2 wq[RYT][3][5];
#pragma unroll
        for (int r = 0; r < RYT; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 5; ++k) wq[r][c][k] = P2{T(0), T(0)};
        bool failed = false;
        int fail_it = 0;
        for (int it = 0; it < n_it; ++it) {
            const uint32_t k = kbase + it;
            if (it % L::B == 0) {
                __syncthreads();
                if (s_fault) {
                    failed = true;
                    fail_it = it;
                    break;
                }
                if (tid == 0)
                    for (int j = it + LA; j < min(it + LA + L::B, n_it); ++j) issue(j);
            }
            // A load that does not arrive stops the block at the next barrier.
            if (!mbar_wait_bounded(&bars[k % S], (k / S) & 1u)) s_fault = 1;
            const unsigned char *sb = smem + (k % S) * L::STAGE_BYTES;
            const T *wx = reinterpret_cast<const T *>(sb + L::X_OFF);
            const T *wy = reinterpret_cast<const T *>(sb + L::Y_OFF);
            const T *wz = reinterpret_cast<const T *>(sb + L::Z_OFF);
            // GJ: gJ at planes ze (x and y taps) and q (z queue), boxes
            // starting at column x0-4 and row y0-2.
            const T *gje = reinterpret_cast<const T *>(sb + L::GE_OFF);
            const T *gjq = reinterpret_cast<const T *>(sb + L::GQ_OFF);
            // A weight pair gJ * C (GJ) or W as stored.
            auto wmul = [&](P2 w, const T *gp) -> P2 {
                if constexpr (GJ) {
                    const P2 gv = ld_pair(gp);
                    if constexpr (sizeof(T) == 4) return p_mul(w, gv);
                    else return P2{w.x * gv.x, w.y * gv.y};
                } else {
                    return w;
                }
            };
            auto wmul1 = [&](T w, const T *gp) -> T {
                if constexpr (GJ) {
                    if constexpr (sizeof(T) == 4) return __fmul_rn(w, *gp);
                    else return w * *gp;
                } else {
                    return w;
                }
            };
            const int q = z0 - 2 + it, ze = q - 2;
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                const int ly = ty + r * TYT;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) wq[r][c][kk] = wq[r][c][kk + 1];
                    wq[r][c][4] = wmul(ld_pair(wz + (c * TT_Y + ly) * TXW + 2 * tx),
                                       gjq + (ly + TMA_HY) * XPX + 2 * tx + TMA_HX);
                }
            }
#pragma unroll
            for (int r = 0; r < RYT; ++r) {
                if (ze < z0 || ze >= z1) break;
                const int ly = ty + r * TYT, y = y0 + ly;
                const bool valid = x < g.nx && y < g.ny;
                T acc[2][3];
                // Three paths, chosen per warp (a warp is two rows of the
                // tile, so a voxel's path depends on where it lies, not on the
                // launch): every pair of the warp with all its taps at
                // fourth-order voxels (four or more voxels from every face);
                // y and z that deep but x near a face (only the x taps choose
                // a scheme); the rest.  In FP32 the first two run on pairs.
                const bool yz_deep = y >= 4 && y <= g.ny - 5 && ze >= 4 && ze <= g.nz - 5;
                const bool deep = yz_deep && x >= 4 && x + 1 <= g.nx - 5;
                const bool w_deep = __all_sync(0xffffffffu, deep || !valid);
                const bool w_yz = __all_sync(0xffffffffu, yz_deep || !valid);
                auto acc_op = [](T a, T w, T kp) -> T {
                    if constexpr (sizeof(T) == 4) return __fmaf_rn(w, kp, a);
                    else return a + w * kp;
                };
                bool done = false;
                if constexpr (sizeof(T) == 4) {
                    if (w_deep) {
                        // sum over the axes of (W(+2) - W(-2)) / 12 + (W(-1) - W(+1)) 2/3,
                        // W(+t) the weight t voxels up the axis: the fourth-order
                        // taps with the differences formed first, per axis
                        // independent, for instruction-level parallelism.
                        const float2 k12 = p_splat(FD<float>::one_twelfth), k23 = p_splat(FD<float>::two_thirds);
#pragma unroll
                        const T *gp = gje + (ly + TMA_HY) * XPX + 2 * tx + TMA_HX;  // gJ at (x, y, ze)
                        for (int c = 0; c < 3; ++c) {
                            const T *px = wx + (c * TT_Y + ly) * XPX + 2 * tx + TMA_HX;
                            const float2 xm = wmul(ld_pair(px - 2), gp - 2), xc = wmul(ld_pair(px), gp),
                                         xp = wmul(ld_pair(px + 2), gp + 2);
                            const T *py = wy + (c * YPY + ly + TMA_HY) * TXW + 2 * tx;
                            const float2 ym2 = wmul(ld_pair(py - 2 * TXW), gp - 2 * XPX),
                                         ym1 = wmul(ld_pair(py - TXW), gp - XPX);
                            const float2 yp1 = wmul(ld_pair(py + TXW), gp + XPX),
                                         yp2 = wmul(ld_pair(py + 2 * TXW), gp + 2 * XPX);
                            const float2 d1x = make_float2(__fsub_rn(xm.y, xc.y), __fsub_rn(xc.x, xp.x));
                            const float2 sx = p_fma(d1x, k23, p_mul(p_sub(xp, xm), k12));
                            const float2 sy = p_fma(p_sub(ym1, yp1), k23, p_mul(p_sub(yp2, ym2), k12));
                            const float2 sz = p_fma(p_sub(wq[r][c][1], wq[r][c][3]), k23,
                                                    p_mul(p_sub(wq[r][c][4], wq[r][c][0]), k12));
                            const float2 a2 = p_add(p_add(sx, sy), sz);
                            acc[0][c] = a2.x;
                            acc[1][c] = a2.y;
                        }
                        done = true;
                    } else if (w_yz) {
                        // x near a face: per-lane coefficients of the x taps
                        // (the tap voxel's scheme along x) and of the y and z
                        // taps (second order when the voxel's x is on the two
                        // outer layers), in the general path's tap order.
                        float2 kx[5], kyz[4];
#pragma unroll
                        for (int i = 0; i < 5; ++i) {
                            const int t = i - 2;
                            float kv[2];
#pragma unroll
                            for (int v = 0; v < 2; ++v) {
                                const int pa = x + v - t;
                                const int kk = pa == 0 ? S_FWD
                                             : pa == g.nx - 1 ? S_BWD
                                             : (pa == 1 || pa == g.nx - 2) ? S_C2 : S_C4;
                                kv[v] = pa < 0 || pa >= g.nx ? 0.f : kappa<float>(kk, t);
                            }
                            kx[i] = make_float2(kv[0], kv[1]);
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int t = i < 2 ? i - 2 : i - 1;
                            float kv[2];
#pragma unroll
                            for (int v = 0; v < 2; ++v) {
                                const bool x_c2 = x + v <= 1 || x + v >= g.nx - 2;
                                kv[v] = x_c2 ? kappa<float>(S_C2, t) : kc[i];
                            }
                            kyz[i] = make_float2(kv[0], kv[1]);
                        }
                        const T *gp = gje + (ly + TMA_HY) * XPX + 2 * tx + TMA_HX;  // gJ at (x, y, ze)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const T *px = wx + (c * TT_Y + ly) * XPX + 2 * tx + TMA_HX;
                            const float2 xm = wmul(ld_pair(px - 2), gp - 2), xc = wmul(ld_pair(px), gp),
                                         xp = wmul(ld_pair(px + 2), gp + 2);
                            const T *py = wy + (c * YPY + ly + TMA_HY) * TXW + 2 * tx;
                            float2 a2 = p_mul(xp, kx[0]);
                            a2 = p_fma(make_float2(xc.y, xp.x), kx[1], a2);
                            a2 = p_fma(xc, kx[2], a2);
                            a2 = p_fma(make_float2(xm.y, xc.x), kx[3], a2);
                            a2 = p_fma(xm, kx[4], a2);
                            a2 = p_fma(wmul(ld_pair(py + 2 * TXW), gp + 2 * XPX), kyz[0], a2);
                            a2 = p_fma(wmul(ld_pair(py + TXW), gp + XPX), kyz[1], a2);
                            a2 = p_fma(wmul(ld_pair(py - TXW), gp - XPX), kyz[2], a2);
                            a2 = p_fma(wmul(ld_pair(py - 2 * TXW), gp - 2 * XPX), kyz[3], a2);
                            a2 = p_fma(wq[r][c][4], kyz[0], a2);
                            a2 = p_fma(wq[r][c][3], kyz[1], a2);
                            a2 = p_fma(wq[r][c][1], kyz[2], a2);
                            a2 = p_fma(wq[r][c][0], kyz[3], a2);
                            acc[0][c] = a2.x;
                            acc[1][c] = a2.y;
                        }
                        done = true;
                    }
                }
                if (!done) {
#pragma unroll
                    for (int v = 0; v < 2; ++v) {
                        T a3[3] = {T(0), T(0), T(0)};
                        if (w_yz) {
                            // Only x can be outer or penultimate: the x taps
                            // choose their schemes; the y and z taps are
                            // fourth order, or second order when the voxel's
                            // x is on the two outer layers (its tap voxels
                            // share that x).  Same order as below.
                            const int xv = x + v;
                            const bool x_c2 = xv <= 1 || xv >= g.nx - 2;
#pragma unroll
                            for (int t = -2; t <= 2; ++t) {
                                const int pa = xv - t;
                                if (pa < 0 || pa >= g.nx) continue;
                                const int kk = pa == 0 ? S_FWD
                                             : pa == g.nx - 1 ? S_BWD
                                             : (pa == 1 || pa == g.nx - 2) ? S_C2 : S_C4;
                                const T kp = kappa<T>(kk, t);
                                if (kp == T(0)) continue;
#pragma unroll
                                for (int c = 0; c < 3; ++c)
                                    a3[c] = acc_op(a3[c],
                                                   wmul1(wx[(c * TT_Y + ly) * XPX + 2 * tx + v - t + TMA_HX],
                                                         gje + (ly + TMA_HY) * XPX + 2 * tx + v - t + TMA_HX),
                                                   kp);
                            }
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const int t = i < 2 ? i - 2 : i - 1;
                                if (x_c2 && (t == -2 || t == 2)) continue;
                                const T kp = x_c2 ? kappa<T>(S_C2, t) : kc[i];
#pragma unroll
                                for (int c = 0; c < 3; ++c)
                                    a3[c] = acc_op(a3[c],
                                                   wmul1(wy[(c * YPY + ly + TMA_HY - t) * TXW + 2 * tx + v],
                                                         gje + (ly + TMA_HY - t) * XPX + 2 * tx + v + TMA_HX),
                                                   kp);
                            }
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const int t = i < 2 ? i - 2 : i - 1;
                                if (x_c2 && (t == -2 || t == 2)) continue;
                                const T kp = x_c2 ? kappa<T>(S_C2, t) : kc[i];
#pragma unroll
                                for (int c = 0; c < 3; ++c)
                                    a3[c] = acc_op(a3[c], v ? wq[r][c][2 - t].y : wq[r][c][2 - t].x, kp);
                            }
                        } else {
                            // Per tap: the tap voxel p = q - t e_a differs
                            // from q only along a, so the outer / penultimate
                            // flags of the other axes come from q
                            // (src/jacobian.c:70-242).
                            const int q3[3] = {x + v, y, ze};
                            bool ob[3], pb[3];
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                ob[b] = q3[b] == 0 || q3[b] == n[b] - 1;
                                pb[b] = q3[b] == 1 || q3[b] == n[b] - 2;
                            }
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                const bool o_other = (a != 0 && ob[0]) || (a != 1 && ob[1]) || (a != 2 && ob[2]);
                                const bool p_other = (a != 0 && pb[0]) || (a != 1 && pb[1]) || (a != 2 && pb[2]);
#pragma unroll
                                for (int t = -2; t <= 2; ++t) {
                                    const int pa = q3[a] - t;
                                    if (pa < 0 || pa >= n[a]) continue;
                                    const bool outer = o_other || pa == 0 || pa == n[a] - 1;
                                    const bool pen = p_other || pa == 1 || pa == n[a] - 2;
                                    const int kk = outer ? (pa == 0 ? S_FWD : (pa == n[a] - 1 ? S_BWD : S_C2))
                                                         : (pen ? S_C2 : S_C4);
                                    const T kp = kappa<T>(kk, t);
                                    if (kp == T(0)) continue;
#pragma unroll
                                    for (int c = 0; c < 3; ++c) {
                                        T w;
                                        if (a == 0)
                                            w = wmul1(wx[(c * TT_Y + ly) * XPX + 2 * tx + v - t + TMA_HX],
                                                      gje + (ly + TMA_HY) * XPX + 2 * tx + v - t + TMA_HX);
                                        else if (a == 1)
                                            w = wmul1(wy[(c * YPY + ly + TMA_HY - t) * TXW + 2 * tx + v],
                                                      gje + (ly + TMA_HY - t) * XPX + 2 * tx + v + TMA_HX);
                                        else
                                            w = v ? wq[r][c][2 - t].y : wq[r][c][2 - t].x;
                                        a3[c] = acc_op(a3[c], w, kp);
                                    }
                                }
                            }
                        }
#pragma unroll
                        for (int c = 0; c < 3; ++c) acc[v][c] = a3[c];
                    }
                }
                if (!valid) continue;
                T *o = gout + (long long) ze * g.zs + (long long) y * g.ys + x;
                if (pair_in) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) st_pair(o + c * g.cs, acc[0][c], acc[1][c]);
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) o[c * g.cs] = acc[0][c];
                }
            }
        }
        if (failed) {
            // Wait (bounded) for the loads still in flight, mark the tile's
            // gradient NaN and leave.
            if (tid == 0)
                for (int j = max(0, fail_it - L::B); j < issued_n; ++j) {
                    const uint32_t kk = kbase + j;
                    mbar_wait_bounded(&bars[kk % S], (kk / S) & 1u, 1u << 16);
                }
            const T nan = T(NAN);
            for (int ze = z0; ze < z1; ++ze)
#pragma unroll
                for (int r = 0; r < RYT; ++r) {
                    const int y = y0 + ty + r * TYT;
                    if (y >= g.ny) continue;
                    for (int v = 0; v < 2; ++v) {
                        if (x + v >= g.nx) continue;
                        for (int c = 0; c < 3; ++c)
                            gout[c * g.cs + (long long) ze * g.zs + (long long) y * g.ys + x + v] = nan;
                    }
                }
            __syncthreads();
            return;
        }
        kbase += n_it;
    }
}

template <typename T, int TXW, int TYT, bool GJ>
int gather_blocks_v() {
    static const int n = [] {
        int v = 0;
        cudaFuncSetAttribute(k_gather_tma<T, TXW, TYT, GJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GatherTmaLayout<T, TXW, GJ>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_gather_tma<T, TXW, TYT, GJ>, TXW / 2 * TYT,
                                                      GatherTmaLayout<T, TXW, GJ>::BYTES + 128);
        return v;
    }();
    return n;
}

// Gather pass on TMA-staged weights: tiles of 32 x TT_Y voxels, 16 x 16
// threads, the z split as in launch_jacobian_tma_v.  With `tm_gj` (a map over
// gJ with box 40 x (TT_Y + 4)), the three weight maps cover C and each weight
// is gJ * C.
template <typename T, bool GJ>
cudaError_t launch_gather_tma_v(const CUtensorMap &tm_wx, const CUtensorMap &tm_wy, const CUtensorMap &tm_wz,
                                const CUtensorMap &tm_gj, const Geom &g, T *gout, int num_sms, cudaStream_t s) {
    constexpr int TXW = 32, TYT = 16, BZ = 32;
    constexpr int smem = GatherTmaLayout<T, TXW, GJ>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_gather_tma<T, TXW, TYT, GJ>, smem, devs);
    if (attr != cudaSuccess) return attr;
    const int tiles_x = (g.nx + TXW - 1) / TXW, tiles_y = (g.ny + TT_Y - 1) / TT_Y;
    const int cols = tiles_x * tiles_y;
    const int slots = std::max(1, gather_blocks_v<T, TXW, TYT, GJ>()) * num_sms;  // resident blocks
    int nzt = (g.nz + BZ - 1) / BZ;                                          // z tiles per column
    const int waves = (cols * nzt + slots - 1) / slots;
    nzt = std::min((g.nz + 7) / 8, std::max(nzt, waves * slots / cols));  // at least 8 planes a tile
    const int bz = (g.nz + nzt - 1) / nzt;
    const int ntiles = cols * ((g.nz + bz - 1) / bz);
    const int grid = std::min(ntiles, slots);
    k_gather_tma<T, TXW, TYT, GJ><<<grid, dim3(TXW / 2, TYT), smem, s>>>(tm_wx, tm_wy, tm_wz, tm_gj, g, gout, tiles_x,
                                                                          tiles_y, ntiles, bz);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gather_tma(const CUtensorMap &tm_wx, const CUtensorMap &tm_wy, const CUtensorMap &tm_wz,
                              const Geom &g, T *gout, int num_sms, cudaStream_t s, const CUtensorMap *tm_gj) {
    if (tm_gj) return launch_gather_tma_v<T, true>(tm_wx, tm_wy, tm_wz, *tm_gj, g, gout, num_sms, s);
    return launch_gather_tma_v<T, false>(tm_wx, tm_wy, tm_wz, tm_wz, g, gout, num_sms, s);
}

// ------------------------------------------------------------------------
// Fused adjoint of the Jacobian map (autograd backward) with the TMA
// pipeline: grad_c(q) = sum_a sum_t W[c][a](q - t e_a) kappa(k_a(q - t e_a), t)
// with W[c][a](p) = gJ(p) cof_ca(I + A(p)) ih_a, A(p) the stencil matrix of
// the Jacobian map at p (the two-pass path's k_adjoint_w / k_adjoint_gather),
// without writing W to memory.
//
// A block of TXW / 2 x TYT threads marches a TXW x TT_Y tile through its z
// range.  Field boxes of the tile plus 4 voxels on every x-y side arrive by
// TMA in S stages; plane m's stage stays until the weights of plane m + 2
// have been formed (their z differences read planes m .. m + 4).  Per plane:
// * the z weights W[c][2] of the newest plane at the thread's own two
//   voxels go into a register queue (they need only in-plane differences);
// * the x weights W[c][0] of the centre plane on the tile plus two columns
//   each side, and its y weights W[c][1] on the tile plus two rows each
//   side, go into shared memory (the halo cells on the last threads);
// * after the block barrier each thread gathers its two voxels' gradient
//   from the x and y weights in shared memory and the z weights in its
//   queue, in the two-pass gather's tap order, and stores it.
// The weights are those of the two-pass path, formed in the same operation
// order, so FP64 results agree with it bit for bit.  Tiles, planes and halo
// cells away from the faces take a fourth-order-only path; near the faces
// every cell and every tap takes its scheme from schemes_at.
// ------------------------------------------------------------------------
template <typename T, int TXW>
struct AdjTmaLayout {
    static constexpr int PX = TXW + 8;      // columns x0-4 .. x0+TXW+3
    static constexpr int PY = TT_Y + 8;     // rows y0-4 .. y0+TT_Y+3
    static constexpr int PLANE = PX * PY;   // elements of one component plane
    static constexpr int S = 7;             // planes m-2 .. m+2 in use, two in flight
    static constexpr int U_BYTES = 3 * PLANE * (int) sizeof(T);
    static_assert(U_BYTES % 128 == 0, "stages stay 128-byte aligned");
    static constexpr int WXC = TXW + 4, WXR = TT_Y;  // x weights: columns x0-2 .. x0+TXW+1, tile rows
    static constexpr int WYC = TXW, WYR = TT_Y + 4;  // y weights: tile columns, rows y0-2 .. y0+TT_Y+1
    static constexpr int WX_ELEMS = 3 * WXR * WXC;
    static constexpr int W_ELEMS = WX_ELEMS + 3 * WYR * WYC;  // one plane's x and y weights
    static constexpr int W_OFF = S * U_BYTES;
    static constexpr int W_BYTES = 2 * W_ELEMS * (int) sizeof(T);  // two planes (double buffer)
    static constexpr int BAR_OFF = (W_OFF + W_BYTES + 7) / 8 * 8;
    static constexpr int BYTES = BAR_OFF + S * 8;
};

// The stages of planes m-2 .. m+2 (the cell's plane is c0).
template <typename T>
struct Planes5 {
    const T *m2, *m1, *c0, *p1, *p2;
    __device__ __forceinline__ const T *at(int d) const {
        return d == -2 ? m2 : (d == -1 ? m1 : (d == 0 ? c0 : (d == 1 ? p1 : p2)));
    }
};

// Derivative of component c along `ax` by scheme k at the box cell whose
// offset in a component plane is `o`, in plane sp.c0 (sp.at(d) the plane d
// away).  The arithmetic of stencil_pair (the Jacobian map's evaluator):
// fourth order with the spacing folded into the weights in FP32, the
// reference's operation order in FP64.
template <typename T, int PX, int PLANE>
__device__ __forceinline__ T adj_deriv(const Planes5<T> &sp, int c, int o, int ax, int k, const T (&ih)[3],
                                       const T (&k1)[3], const T (&k2n)[3]) {
    const int oc = c * PLANE + o;
    auto v = [&](int d) -> T {
        if (ax == 0) return sp.c0[oc + d];
        if (ax == 1) return sp.c0[oc + d * PX];
        return sp.at(d)[oc];
    };
    switch (k) {
    case S_FWD: return fd_fwd<T>(v(0), v(1), v(2), ih[ax]);
    case S_BWD: return fd_bwd<T>(v(0), v(-1), v(-2), ih[ax]);
    case S_C2: return fd_c2<T>(v(1), v(-1), ih[ax]);
    default:
        if constexpr (sizeof(T) == 4) return c4_folded(v(1), v(-1), v(2), v(-2), k1[ax], k2n[ax]);
        return fd_c4<T>(v(1), v(-1), v(2), v(-2), ih[ax]);
    }
}

// W[c][b] = w * cof_cb(I + a) * ih_b for the three components c (the weight
// epilogue's expression and order).
template <typename T>
__device__ __forceinline__ void adj_weights(const T (&a)[3][3], T w, int b, T ihb, T (&out)[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int r0 = c == 0 ? 1 : 0, r1 = c == 2 ? 1 : 2;
        const int c0 = b == 0 ? 1 : 0, c1 = b == 2 ? 1 : 2;
        const T m00 = a[r0][c0] + (r0 == c0 ? T(1) : T(0));
        const T m11 = a[r1][c1] + (r1 == c1 ? T(1) : T(0));
        const T m01 = a[r0][c1] + (r0 == c1 ? T(1) : T(0));
        const T m10 = a[r1][c0] + (r1 == c0 ? T(1) : T(0));
        const T minor = m00 * m11 - m01 * m10;
        const T cof = ((c + b) & 1) ? -minor : minor;
        out[c] = w * cof * ihb;
    }
}

template <typename T, int TXW, int TYT>
__global__ void __launch_bounds__(TXW / 2 * TYT, sizeof(T) == 4 ? 2 : 1)
    k_adjoint_tma(const __grid_constant__ CUtensorMap tm_u, const Geom g, const T *__restrict__ gJ,
                  T *__restrict__ gout, int tiles_x, int tiles_y, int ntiles, int bz) {
    using L = AdjTmaLayout<T, TXW>;
    constexpr int TPX = TXW / 2, NTH = TPX * TYT, S = L::S, PX = L::PX, PLANE = L::PLANE;
    constexpr int WXC = L::WXC, WYC = L::WYC;
    constexpr int NHX = TT_Y * 2, NHY = 4 * TPX, NH = NHX + NHY;  // halo pair tasks: x sides, y sides
    static_assert(TYT == TT_Y && TPX == 16, "one tile row per thread row, two rows per warp");
    static_assert(NH <= NTH - 64, "halo tasks on threads other than the first two warps");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char *smem = align_smem_128(smem_dyn);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::BAR_OFF);
    __shared__ int s_fault;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TPX + tx;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        tmap_prefetch(&tm_u);
        s_fault = 0;
    }
    __syncthreads();
    const T ih[3] = {(T) g.ih[0], (T) g.ih[1], (T) g.ih[2]};
    const T k1[3] = {FD<T>::two_thirds * ih[0], FD<T>::two_thirds * ih[1], FD<T>::two_thirds * ih[2]};
    const T k2n[3] = {-FD<T>::one_twelfth * ih[0], -FD<T>::one_twelfth * ih[1], -FD<T>::one_twelfth * ih[2]};
    const int n[3] = {g.nx, g.ny, g.nz};
    // Fourth-order difference (the generic path's arithmetic for S_C4).
    auto c4 = [&](T p1, T m1, T p2, T m2, int ax) -> T {
        if constexpr (sizeof(T) == 4) return c4_folded(p1, m1, p2, m2, k1[ax], k2n[ax]);
        return fd_c4<T>(p1, m1, p2, m2, ih[ax]);
    };
    // Differences of the cell pair (xf, xf + 1) at box offset o (row and
    // plane at least two cells inside the volume): along x, y and z as
    // requested, with each cell's scheme chosen by its x position
    // (src/jacobian.c:113-241): outer column -> one-sided in x and second
    // order in y and z; penultimate column -> second order; else fourth
    // order.  With all_c4 every cell is fourth order (no selects).  Rows a0
    // of the first cell, a1 of the second.
    auto pair_diffs = [&](const Planes5<T> &sp, int c, int o, int xf, bool all_c4, bool wx, bool wy, bool wz,
                          T (&a0)[3][3], T (&a1)[3][3]) {
        const T *q = sp.c0 + c * PLANE + o;
        const int oc = c * PLANE + o;
        if (all_c4) {
            if (wx) {
                const auto xm = ld_pair(q - 2), xc = ld_pair(q), xp = ld_pair(q + 2);
                a0[c][0] = c4(xc.y, xm.y, xp.x, xm.x, 0);
                a1[c][0] = c4(xp.x, xc.x, xp.y, xm.y, 0);
            }
            if (wy) {
                const auto ym1 = ld_pair(q - PX), yp1 = ld_pair(q + PX), ym2 = ld_pair(q - 2 * PX),
                           yp2 = ld_pair(q + 2 * PX);
                a0[c][1] = c4(yp1.x, ym1.x, yp2.x, ym2.x, 1);
                a1[c][1] = c4(yp1.y, ym1.y, yp2.y, ym2.y, 1);
            }
            if (wz) {
                const auto zm2 = ld_pair(sp.m2 + oc), zm1 = ld_pair(sp.m1 + oc);
                const auto zp1 = ld_pair(sp.p1 + oc), zp2 = ld_pair(sp.p2 + oc);
                a0[c][2] = c4(zp1.x, zm1.x, zp2.x, zm2.x, 2);
                a1[c][2] = c4(zp1.y, zm1.y, zp2.y, zm2.y, 2);
            }
            return;
        }
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            T(&a)[3][3] = v ? a1 : a0;
            const int xv = xf + v;
            const bool xo_lo = xv == 0, xo_hi = xv == g.nx - 1;
            const bool second = xo_lo || xo_hi || xv == 1 || xv == g.nx - 2;
            const T *p = q + v;
            if (wx) {
                const T fx = xo_lo ? fd_fwd<T>(p[0], p[1], p[2], ih[0])
                                   : (xo_hi ? fd_bwd<T>(p[0], p[-1], p[-2], ih[0]) : fd_c2<T>(p[1], p[-1], ih[0]));
                const T cx4 = c4(p[1], p[-1], p[2], p[-2], 0);
                a[c][0] = second ? fx : cx4;
            }
            if (wy) {
                const T cy4 = c4(p[PX], p[-PX], p[2 * PX], p[-2 * PX], 1);
                const T cy2 = fd_c2<T>(p[PX], p[-PX], ih[1]);
                a[c][1] = second ? cy2 : cy4;
            }
            if (wz) {
                const T zp1 = sp.p1[oc + v], zm1 = sp.m1[oc + v], zp2 = sp.p2[oc + v], zm2 = sp.m2[oc + v];
                const T cz4 = c4(zp1, zm1, zp2, zm2, 2);
                const T cz2 = fd_c2<T>(zp1, zm1, ih[2]);
                a[c][2] = second ? cz2 : cz4;
            }
        }
    };
    // Differences of one cell by the schemes schemes_at gives it (any
    // position in the volume).
    auto cell_diffs = [&](const Planes5<T> &sp, int x, int y, int z, int o, bool wx, bool wy, bool wz,
                          T (&a)[3][3]) {
        int ks[3];
        schemes_at(x, y, z, g, ks);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a[c][0] = wx ? adj_deriv<T, PX, PLANE>(sp, c, o, 0, ks[0], ih, k1, k2n) : T(0);
            a[c][1] = wy ? adj_deriv<T, PX, PLANE>(sp, c, o, 1, ks[1], ih, k1, k2n) : T(0);
            a[c][2] = wz ? adj_deriv<T, PX, PLANE>(sp, c, o, 2, ks[2], ih, k1, k2n) : T(0);
        }
    };
    uint32_t kbase = 0;

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int txi = tile % tiles_x, tyi = (tile / tiles_x) % tiles_y, tzi = tile / (tiles_x * tiles_y);
        const int x0 = txi * TXW, y0 = tyi * TT_Y, z0 = tzi * bz;
        const int z1 = min(z0 + bz, g.nz);
        const int n_it = z1 - z0 + 4;  // newest planes z0-2 .. z1+1
        __syncthreads();  // every warp has finished the previous tile's stages
        int issued_n = 0;
        auto issue = [&](int j) {
            issued_n = j + 1;
            const uint32_t k = kbase + j;
            uint64_t *bar = &bars[k % S];
            mbar_arrive_expect_tx(bar, L::U_BYTES);
            tma_load_4d(smem + (k % S) * L::U_BYTES, &tm_u, bar, x0 - 4, y0 - 4, z0 - 2 + j, 0);
        };
        if (tid == 0)
            for (int j = 0; j < min(S, n_it); ++j) issue(j);
        auto stage = [&](int j) -> const T * {
            return reinterpret_cast<const T *>(smem + ((kbase + j) % S) * L::U_BYTES);
        };

        const int x = x0 + 2 * tx, y = y0 + ty;  // own voxels (x, y), (x + 1, y)
        const int bxo = 2 * tx + 4, byo = ty + 4;  // their box cell
        const bool row_vol = y < g.ny;
        const bool x0_vol = x < g.nx, x1_vol = x + 1 < g.nx;
        // Rows of this thread's warp (two tile rows) at least two cells
        // inside the volume; tile columns likewise (fourth order in x).
        const int yw = y0 + (ty & ~1);
        const bool warp_rows_in = yw >= 2 && yw + 1 <= g.ny - 3;
        const bool cols_c4 = x0 >= 2 && x0 + TXW - 1 <= g.nx - 3;
        const bool warp_rows_deep = yw >= 4 && yw + 1 <= g.ny - 5;
        const bool cols_deep = x0 >= 4 && x0 + TXW - 1 <= g.nx - 5;
        // Own z weights W[c][2] of planes m-2 .. m+2 (queue index 2 + d for
        // plane m + d), and own gJ of planes p-2 .. p (index 0 .. 2).
        T zw[2][3][5];
        T gq[2][3];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 5; ++k) zw[v][c][k] = T(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) gq[v][k] = T(0);
        }
        auto own_gj = [&](int z, int v) -> T {
            const bool in = z >= 0 && z < g.nz && row_vol && (v ? x1_vol : x0_vol);
            return in ? gJ[(long long) z * g.zs + (long long) y * g.ys + x + v] : T(0);
        };
        T gnext[2] = {own_gj(z0 - 2, 0), own_gj(z0 - 2, 1)};  // gJ of the next newest plane
        bool failed = false;
        for (int it = 0; it < n_it; ++it) {
            const uint32_t k = kbase + it;
            if (!mbar_wait_bounded(&bars[k % S], (k / S) & 1u)) s_fault = 1;
            const int p = z0 - 2 + it;  // newest plane
            const int m = p - 2;        // centre plane of this iteration's x and y weights and gradient
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                gq[v][0] = gq[v][1];
                gq[v][1] = gq[v][2];
                gq[v][2] = gnext[v];
                gnext[v] = own_gj(p + 1, v);  // used next iteration
            }
            const bool centre = m >= z0 && m < z1;
            // Halo task of this thread (x sides: pairs of columns x0-2, x0-1
            // or x0+TXW, x0+TXW+1 on a tile row; y sides: pairs of tile
            // columns on rows y0-2, y0-1, y0+TT_Y, y0+TT_Y+1), and its gJ,
            // loaded before the weights are formed.
            const int h = tid - (NTH - NH);
            const bool xside = h < NHX;
            int cx = 0, cy = 0;
            if (h >= 0) {
                if (xside) {
                    cx = (h / TT_Y) ? x0 + TXW : x0 - 2;
                    cy = y0 + h % TT_Y;
                } else {
                    const int h2 = h - NHX, r = h2 / TPX;
                    cx = x0 + 2 * (h2 % TPX);
                    cy = r < 2 ? y0 - 2 + r : y0 + TT_Y - 2 + r;
                }
            }
            T hw[2] = {T(0), T(0)};
            if (h >= 0 && centre) {
#pragma unroll
                for (int v = 0; v < 2; ++v) {
                    const int xv = cx + v;
                    if (xv >= 0 && xv < g.nx && cy >= 0 && cy < g.ny)
                        hw[v] = gJ[(long long) m * g.zs + (long long) cy * g.ys + xv];
                }
            }
            // (a) z weights of plane p at the own voxels (in-plane differences only).
            {
                const Planes5<T> sp{nullptr, nullptr, stage(it), nullptr, nullptr};
                T wz0[3] = {T(0), T(0), T(0)}, wz1[3] = {T(0), T(0), T(0)};
                if (p >= 2 && p <= g.nz - 3 && warp_rows_in) {
                    T a0[3][3], a1[3][3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        pair_diffs(sp, c, byo * PX + bxo, x, cols_c4, true, true, false, a0, a1);
                        a0[c][2] = a1[c][2] = T(0);  // not used by the z weights
                    }
                    adj_weights<T>(a0, gq[0][2], 2, ih[2], wz0);
                    adj_weights<T>(a1, gq[1][2], 2, ih[2], wz1);
                } else if (p >= 0 && p < g.nz && row_vol) {
#pragma unroll
                    for (int v = 0; v < 2; ++v) {
                        if (x + v >= g.nx) continue;
                        T a[3][3];
                        cell_diffs(sp, x + v, y, p, byo * PX + bxo + v, true, true, false, a);
                        adj_weights<T>(a, gq[v][2], 2, ih[2], v ? wz1 : wz0);
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        zw[0][c][kk] = zw[0][c][kk + 1];
                        zw[1][c][kk] = zw[1][c][kk + 1];
                    }
                    zw[0][c][4] = wz0[c];
                    zw[1][c][4] = wz1[c];
                }
            }
            T *wb = reinterpret_cast<T *>(smem + L::W_OFF) + (it & 1) * L::W_ELEMS;
            T *WX = wb, *WY = wb + L::WX_ELEMS;
            if (centre && !s_fault) {
                const Planes5<T> sp{stage(it - 4), stage(it - 3), stage(it - 2), stage(it - 1), stage(it)};
                const bool plane_in = m >= 2 && m <= g.nz - 3;
                // (b) own voxels: x and y weights of plane m.
                {
                    T wx0[3] = {T(0), T(0), T(0)}, wx1[3] = {T(0), T(0), T(0)};
                    T wy0[3] = {T(0), T(0), T(0)}, wy1[3] = {T(0), T(0), T(0)};
                    if (plane_in && warp_rows_in) {
                        T a0[3][3], a1[3][3];
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            pair_diffs(sp, c, byo * PX + bxo, x, cols_c4, true, true, true, a0, a1);
                        adj_weights<T>(a0, gq[0][0], 0, ih[0], wx0);
                        adj_weights<T>(a1, gq[1][0], 0, ih[0], wx1);
                        adj_weights<T>(a0, gq[0][0], 1, ih[1], wy0);
                        adj_weights<T>(a1, gq[1][0], 1, ih[1], wy1);
                    } else if (row_vol) {
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            if (x + v >= g.nx) continue;
                            T a[3][3];
                            cell_diffs(sp, x + v, y, m, byo * PX + bxo + v, true, true, true, a);
                            adj_weights<T>(a, gq[v][0], 0, ih[0], v ? wx1 : wx0);
                            adj_weights<T>(a, gq[v][0], 1, ih[1], v ? wy1 : wy0);
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        st_pair(WX + (c * TT_Y + ty) * WXC + 2 * tx + 2, wx0[c], wx1[c]);
                        st_pair(WY + (c * (TT_Y + 4) + ty + 2) * WYC + 2 * tx, wy0[c], wy1[c]);
                    }
                }
                // (c) halo pairs: the x weights use columns 1 and 2 of I + A
                // (differences along y and z), the y weights 0 and 2.
                if (h >= 0) {
                    const int o = (cy - y0 + 4) * PX + (cx - x0 + 4);
                    T wv0[3] = {T(0), T(0), T(0)}, wv1[3] = {T(0), T(0), T(0)};
                    const bool cells_in = cx >= 0 && cx + 1 < g.nx && cy >= 0 && cy < g.ny;
                    const bool row_in = cy >= 2 && cy <= g.ny - 3;
                    // x sides: two columns at least two inside the volume;
                    // y sides: any columns, selects at the x ends.
                    const bool pair_ok = plane_in && row_in && cells_in && (!xside || (cx >= 2 && cx + 1 <= g.nx - 3));
                    const bool pair_c4 = cx >= 2 && cx + 1 <= g.nx - 3;
                    if (pair_ok) {
                        T a0[3][3], a1[3][3];
                        if (xside) {
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                a0[c][0] = a1[c][0] = T(0);
                                pair_diffs(sp, c, o, cx, true, false, true, true, a0, a1);
                            }
                            adj_weights<T>(a0, hw[0], 0, ih[0], wv0);
                            adj_weights<T>(a1, hw[1], 0, ih[0], wv1);
                        } else {
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                a0[c][1] = a1[c][1] = T(0);
                                pair_diffs(sp, c, o, cx, pair_c4, true, false, true, a0, a1);
                            }
                            adj_weights<T>(a0, hw[0], 1, ih[1], wv0);
                            adj_weights<T>(a1, hw[1], 1, ih[1], wv1);
                        }
                    } else {
#pragma unroll
                        for (int v = 0; v < 2; ++v) {
                            const int xv = cx + v;
                            if (!(xv >= 0 && xv < g.nx && cy >= 0 && cy < g.ny)) continue;
                            T a[3][3];
                            if (xside) {
                                cell_diffs(sp, xv, cy, m, o + v, false, true, true, a);
                                adj_weights<T>(a, hw[v], 0, ih[0], v ? wv1 : wv0);
                            } else {
                                cell_diffs(sp, xv, cy, m, o + v, true, false, true, a);
                                adj_weights<T>(a, hw[v], 1, ih[1], v ? wv1 : wv0);
                            }
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        if (xside)
                            st_pair(WX + (c * TT_Y + (cy - y0)) * WXC + (cx - x0 + 2), wv0[c], wv1[c]);
                        else
                            st_pair(WY + (c * (TT_Y + 4) + (cy - y0 + 2)) * WYC + (cx - x0), wv0[c], wv1[c]);
                    }
                }
            }
            __syncthreads();
            if (s_fault) {
                failed = true;
                break;
            }
            // Iteration it - 4's stage (plane m - 2) is not read again.
            if (tid == 0 && it >= 4 && it + 3 < n_it) issue(it + 3);
            // (d) gradient of the own voxels at plane m.
            if (!centre || !row_vol) continue;
            if (cols_deep && warp_rows_deep && m >= 4 && m <= g.nz - 5) {
                // Every tap is fourth order: constant weights, the general
                // path's tap and summation order.
                T acc0[3] = {T(0), T(0), T(0)}, acc1[3] = {T(0), T(0), T(0)};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const T *wxr = WX + (c * TT_Y + ty) * WXC + 2 * tx;  // columns x-2 .. x+3
                    const auto xa = ld_pair(wxr), xb = ld_pair(wxr + 2), xc = ld_pair(wxr + 4);
                    const T wxv[6] = {xa.x, xa.y, xb.x, xb.y, xc.x, xc.y};
#pragma unroll
                    for (int t = -2; t <= 2; ++t) {
                        if (t == 0) continue;
                        const T kp = kappa<T>(S_C4, t);
                        acc0[c] += wxv[2 - t] * kp;
                        acc1[c] += wxv[3 - t] * kp;
                    }
                    const T *wyc = WY + (c * (TT_Y + 4) + ty + 2) * WYC + 2 * tx;
#pragma unroll
                    for (int t = -2; t <= 2; ++t) {
                        if (t == 0) continue;
                        const T kp = kappa<T>(S_C4, t);
                        const auto wy = ld_pair(wyc - t * WYC);
                        acc0[c] += wy.x * kp;
                        acc1[c] += wy.y * kp;
                    }
#pragma unroll
                    for (int t = -2; t <= 2; ++t) {
                        if (t == 0) continue;
                        const T kp = kappa<T>(S_C4, t);
                        acc0[c] += zw[0][c][2 - t] * kp;
                        acc1[c] += zw[1][c][2 - t] * kp;
                    }
                }
                const long long off = (long long) m * g.zs + (long long) y * g.ys + x;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    gout[c * g.cs + off] = acc0[c];
                    gout[c * g.cs + off + 1] = acc1[c];
                }
                continue;
            }
            // Taps with their schemes (the two-pass gather's general path),
            // out-of-volume and zero-weight taps predicated off.
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const int xv = x + v;
                if (xv >= g.nx) continue;
                T acc[3] = {T(0), T(0), T(0)};
                const int q[3] = {xv, y, m};
                bool ob[3], pb[3];
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    ob[bb] = q[bb] == 0 || q[bb] == n[bb] - 1;
                    pb[bb] = q[bb] == 1 || q[bb] == n[bb] - 2;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const bool o_other = (a != 0 && ob[0]) || (a != 1 && ob[1]) || (a != 2 && ob[2]);
                    const bool p_other = (a != 0 && pb[0]) || (a != 1 && pb[1]) || (a != 2 && pb[2]);
#pragma unroll
                    for (int t = -2; t <= 2; ++t) {
                        const int pa = q[a] - t;
                        const bool outer = o_other || pa == 0 || pa == n[a] - 1;
                        const bool pen = p_other || pa == 1 || pa == n[a] - 2;
                        const int kk = outer ? (pa == 0 ? S_FWD : (pa == n[a] - 1 ? S_BWD : S_C2))
                                             : ((g.order == 2 || pen) ? S_C2 : S_C4);
                        const T kp = (pa >= 0 && pa < n[a]) ? kappa<T>(kk, t) : T(0);
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            T wt;
                            if (a == 0)
                                wt = WX[(c * TT_Y + ty) * WXC + 2 * tx + v - t + 2];
                            else if (a == 1)
                                wt = WY[(c * (TT_Y + 4) + ty - t + 2) * WYC + 2 * tx + v];
                            else
                                wt = zw[v][c][2 - t];
                            if (kp != T(0)) acc[c] += wt * kp;
                        }
                    }
                }
                const long long off = (long long) m * g.zs + (long long) y * g.ys + xv;
#pragma unroll
                for (int c = 0; c < 3; ++c) gout[c * g.cs + off] = acc[c];
            }
        }
        if (failed) {
            // Wait (bounded) for the loads still in flight, mark the tile's
            // voxels NaN and leave.
            if (tid == 0)  // the last load issued into each slot
                for (int j = max(0, issued_n - S); j < issued_n; ++j) {
                    const uint32_t kk = kbase + j;
                    mbar_wait_bounded(&bars[kk % S], (kk / S) & 1u, 1u << 16);
                }
            const T nan = T(NAN);
            for (int ze = z0; ze < z1; ++ze)
                for (int v = 0; v < 2; ++v) {
                    if (x + v >= g.nx || !row_vol) continue;
                    const long long off = (long long) ze * g.zs + (long long) y * g.ys + x + v;
                    for (int c = 0; c < 3; ++c) gout[c * g.cs + off] = nan;
                }
            __syncthreads();
            return;
        }
        kbase += n_it;
    }
}

template <typename T, int TXW, int TYT>
int adjoint_tma_blocks_v() {
    static const int nb = [] {
        int v = 0;
        cudaFuncSetAttribute(k_adjoint_tma<T, TXW, TYT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             AdjTmaLayout<T, TXW>::BYTES + 128);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_adjoint_tma<T, TXW, TYT>, TXW / 2 * TYT,
                                                      AdjTmaLayout<T, TXW>::BYTES + 128);
        return v;
    }();
    return nb;
}

// Fused adjoint of the field `tm_u` describes (box 40 x 24 x 1 x 3, order 4),
// gJ and gout in the field's dense layout (geometry g).  Tiles of 32 x TT_Y,
// dealt round-robin, z split as the Jacobian map's.
template <typename T>
cudaError_t launch_adjoint_tma(const CUtensorMap &tm_u, const Geom &g, const T *gJ, T *gout, int num_sms,
                               cudaStream_t s) {
    constexpr int TXW = 32, TYT = 16, BZ = 32;
    constexpr int smem = AdjTmaLayout<T, TXW>::BYTES + 128;
    static std::atomic<unsigned long long> devs{0};
    const cudaError_t attr = opt_in_smem(k_adjoint_tma<T, TXW, TYT>, smem, devs);
    if (attr != cudaSuccess) return attr;
    const int tiles_x = (g.nx + TXW - 1) / TXW, tiles_y = (g.ny + TT_Y - 1) / TT_Y;
    const int cols = tiles_x * tiles_y;
    const int slots = std::max(1, adjoint_tma_blocks_v<T, TXW, TYT>()) * num_sms;
    int nzt = (g.nz + BZ - 1) / BZ;
    const int waves = (cols * nzt + slots - 1) / slots;
    nzt = std::min((g.nz + 7) / 8, std::max(nzt, waves * slots / cols));
    const int bz = (g.nz + nzt - 1) / nzt;
    const int ntiles = cols * ((g.nz + bz - 1) / bz);
    const int grid = std::min(ntiles, slots);
    k_adjoint_tma<T, TXW, TYT><<<grid, dim3(TXW / 2, TYT), smem, s>>>(tm_u, g, gJ, gout, tiles_x, tiles_y, ntiles,
                                                                       bz);
    count_launch();
    return cudaGetLastError();
}

#define DTB_INSTANTIATE_TMA(T)                                                                              \
    template cudaError_t launch_trial_tma<T>(const VolumeDesc<T> *, const int *, int, int, cudaStream_t,    \
                                             unsigned char *, int, int, TileQueue *, int);                  \
    template cudaError_t launch_gradient_tma<T>(const VolumeDesc<T> *, const int *, int, int, cudaStream_t, \
                                                unsigned char *, int, int, TileQueue *, int);               \
    template int trial_tma_blocks_per_sm<T>(int, int);                                                      \
    template cudaError_t launch_greedy_tma<T>(const VolumeDesc<T> *, const int *, int, int, cudaStream_t,   \
                                              unsigned char *, TileQueue *);                                \
    template int greedy_tma_blocks_per_sm<T>();                                                             \
    template cudaError_t launch_jacobian_tma<T>(const CUtensorMap &, const Geom &, T *, long long, long long, int, \
                                                cudaStream_t, const T *, T *, long long);                   \
    template cudaError_t launch_gather_tma<T>(const CUtensorMap &, const CUtensorMap &, const CUtensorMap &,   \
                                              const Geom &, T *, int, cudaStream_t, const CUtensorMap *);   \
    template int gradient_tma_blocks_per_sm<T>(int, int);                                                   \
    template cudaError_t launch_trial_rel<T>(const VolumeDesc<T> *, const int *, int, int, cudaStream_t,    \
                                             unsigned char *, int, int, TileQueue *);                       \
    template int trial_rel_blocks_per_sm<T>(int, int);                                                     \
    template cudaError_t launch_adjoint_tma<T>(const CUtensorMap &, const Geom &, const T *, T *, int,       \
                                               cudaStream_t);

}  // namespace dtb
