// Internal declarations shared by the host driver and the kernel files.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "disptools_b200.h"

namespace dtb {

// Thread-block shape of every stencil kernel: BX threads along x (one warp,
// coalesced rows), BY along y; each block marches a z-range of one tile.
constexpr int BX = 32;
constexpr int BY = 8;
constexpr int NT = BX * BY;
// Tile height of the TMA kernels of the gradient method (two rows per thread).
constexpr int TT_Y = 2 * BY;

// Phases of the per-volume step-control state machine.
enum Phase {
    PH_EVAL0 = 0,   // evaluate the initial field
    PH_SEARCH = 1,  // initial step-length search (gradient method)
    PH_MAIN = 2,    // backtracking line search (gradient method)
    PH_GREEDY = 3,  // greedy iterations
};

// Per-volume solver state, resident in device memory.  The last block of each
// trial launch runs the step control on it (one thread, FP64), so no host
// round trip is needed between trials.
// One line of the verbose output: the reference prints "Iteration ..."
// after every line search (kind 0) and the greedy method "reducing step
// size" after a rejected step (kind 1), src/displacement_field_gradient.c:377-383,
// src/displacement_field_greedy.c:184-212.
struct IterLog {
    long long it;
    int kind;
    int pad;
    double E, M, eta;
};

struct SolverState {
    // parameters (reference signature order)
    double epsilon, tolerance, eta_max, alpha, beta, gamma, delta, zeta, theta, iota;
    long long it_max;
    int strict;
    int algorithm;
    // control
    double eta;
    double E_last, M_last;   // error of the last accepted field; M_last for `strict`
    double E0, M0;           // error of the initial field
    double gn2;              // squared norm of the current gradient
    double E, M;             // last evaluated candidate
    double ret_E, ret_M;     // error of the field that would be returned
    long long it, trials, gradients;
    int phase;
    int done;
    int reason;
    int old_buf;             // which field buffer holds the accepted field
    int need_gradient;
    // Greedy method: some boundary voxel of the initial field (buffer 0) is
    // not +0 (bitwise).  Buffer 1 starts zeroed, and no buffer's boundary
    // voxels are ever changed, so otherwise every boundary value is +0.
    int b0_nonzero;
    int v_cur;               // greedy: which error map is the current one
    unsigned int ticket_t;   // block counters of the trial / gradient launches
    unsigned int ticket_g;
    int fault;               // a bounded wait gave up (reported as an error)
    IterLog *log;            // verbose output (null when off)
    long long log_cap, log_n;
};

// Dynamic tile queue of one persistent launch: blocks take tiles with an
// atomic counter; the last block to leave resets the queue for the next
// launch (every block increments `exited` exactly once, after its last take).
struct TileQueue {
    unsigned int next;
    unsigned int exited;
};

// Geometry of one volume on the device.
struct Geom {
    int nx, ny, nz;
    int order;               // interior finite-difference order: 4 or 2
    long long ys, zs, cs;    // element strides of y, z and the component
    double ih[3];            // inverse spacing
    double sp[3];            // spacing
};

// One volume of a launch (single solves use one).
template <typename T>
struct VolumeDesc {
    Geom g;
    T *field[2];             // ping-pong fields [3][nz][ny][nx]
    T *grad;                 // gradient [3][nz][ny][nx], zero on the boundary
    const T *Jt;             // target Jacobian
    const uint8_t *mask;     // body mask
    T *v[2];                 // greedy: error maps
    T *jout;                 // jacobian-only launches: output map
    T *ep[2];                // gradient method: regularised error e' of field[i]
    // TMA descriptors (device memory) of field[0..1], grad, ep[0..1] or
    // v[0..1] (three-plane boxes), Jt, mask
    const CUtensorMap *tm_field[2];
    const CUtensorMap *tm_grad;
    const CUtensorMap *tm_ep[2];
    const CUtensorMap *tm_v[2];
    const CUtensorMap *tm_Jt;
    const CUtensorMap *tm_mask;
    SolverState *st;
    double2 *part_t;         // per-tile partials of the trial launch (sum, max)
    double *part_g;          // per-tile partials of the gradient launch
    int tiles_x, tiles_y, tiles_z;
    int tile_begin;          // first global tile index of this volume
    int ntiles;
    int bz;                  // planes per tile
    // Failure-path test (dtb_test_drop_tma_load): the trial launch's tile
    // `drop_tile` (global index, -1: none) does not issue the loads of its
    // iteration `drop_it`; bounded waits poll at most `wait_limit` times
    // (0: the default bound).
    int drop_tile, drop_it;
    unsigned wait_limit;
};

// Dynamic shared memory of the Jacobian map kernel (bytes): a five-plane ring.
template <typename T> constexpr int jacobian_smem_bytes() {
    return 5 * 3 * (BY + 4) * (BX + 4) * (int) sizeof(T);
}

// Launch wrappers, instantiated for float and double in dt_kernels_*.cu.
// `work_flag` (may be null) is set to 1 by a launch that did work for at
// least one volume (profiling separates real launches from no-op ones).
// Jacobian map of field[0] of each volume into its jout (tiles BX x BY).
template <typename T>
cudaError_t launch_jacobian(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                            cudaStream_t s);
// TMA kernels of the gradient method; tiles are tile_x (64 or 32) by TT_Y
// voxels; threads_y rows of threads (8 or 16).  `pf` > 0 prefetches into L2
// the boxes of the plane pf iterations ahead of each load.
template <typename T>
cudaError_t launch_trial_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                             cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y, TileQueue *queue,
                             int pf);
template <typename T>
cudaError_t launch_gradient_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                                cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y,
                                TileQueue *queue, int pf);
template <typename T>
int trial_tma_blocks_per_sm(int tile_x, int threads_y);
// The trial kernel without a per-plane block barrier: stages stay resident
// until their plane was the stencil's centre, candidate taps are formed where
// they are read, and the last warp out of a stage issues its refill.
template <typename T>
cudaError_t launch_trial_rel(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                             cudaStream_t s, unsigned char *work_flag, int tile_x, int threads_y, TileQueue *queue);
template <typename T>
int trial_rel_blocks_per_sm(int tile_x, int threads_y);
template <typename T>
int gradient_tma_blocks_per_sm(int tile_x, int threads_y);
// TMA trial kernel of the greedy method (tiles 32 x TT_Y).
template <typename T>
cudaError_t launch_greedy_tma(const VolumeDesc<T> *vols, const int *tile_vol, int total_tiles, int grid,
                              cudaStream_t s, unsigned char *work_flag, TileQueue *queue);
template <typename T>
int greedy_tma_blocks_per_sm();
// TMA stencil of one field of order 4 (the map `tm_u` over the field with
// box 40 x 20 x 1 x 3), with element strides jys, jzs for the scalar maps:
// the Jacobian map into jout; with gJ and W, (adjoint weights) W[c][a] = gJ *
// cof_ca(I + grad u) * ih_a into W with component stride wn (no map); with W
// and no gJ, the map and C[c][a] = cof_ca(I + grad u) * ih_a into W.
template <typename T>
cudaError_t launch_jacobian_tma(const CUtensorMap &tm_u, const Geom &g, T *jout, long long jys, long long jzs,
                                int num_sms, cudaStream_t s, const T *gJ = nullptr, T *W = nullptr,
                                long long wn = 0);
// Gather pass of the adjoint on TMA-staged weights W[c][a][wn]: maps over W
// with boxes 40 x TT_Y (axis x), 32 x (TT_Y + 4) (axis y) and 32 x TT_Y
// (axis z), one plane, three components.  With `tm_gj` (a map over gJ, box
// 40 x (TT_Y + 4)), the maps cover C[c][a] = cof_ca * ih_a instead and each
// weight is formed as gJ * C.
template <typename T>
cudaError_t launch_gather_tma(const CUtensorMap &tm_wx, const CUtensorMap &tm_wy, const CUtensorMap &tm_wz,
                              const Geom &g, T *gout, int num_sms, cudaStream_t s,
                              const CUtensorMap *tm_gj = nullptr);
// Fused adjoint of the Jacobian stencil of order 4 (one TMA kernel, no
// weight buffer): `tm_u` maps the field with box 40 x 24 x 1 x 3; gJ and gout
// in the field's dense layout.
template <typename T>
cudaError_t launch_adjoint_tma(const CUtensorMap &tm_u, const Geom &g, const T *gJ, T *gout, int num_sms,
                               cudaStream_t s);
// Adjoint of the Jacobian stencil: the weight pass (unless w_done: W already
// holds the weights) and the gather pass; W is [9][N] with component stride wn.
template <typename T>
cudaError_t launch_adjoint(const Geom &g, const T *field, const T *gJ, T *W, long long wn, T *gout, bool w_done,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_convert(const void *src, int src_is_double, T *dst, long long n, cudaStream_t s);
template <typename T>
cudaError_t launch_to_double(const T *src, double *dst, long long n, cudaStream_t s);
template <typename T>
cudaError_t launch_regularise(T *J, long long n, double eps, cudaStream_t s);
// Sets *flag = 1 if a boundary voxel of the field [3][nz][ny][nx] (strides
// of g) is not +0 bitwise; leaves it otherwise.
template <typename T>
cudaError_t launch_boundary_nonzero(const T *field, const Geom &g, int *flag, cudaStream_t s);

// Kernel profiling (dtb_set_profiling): whether it is on, and one timed
// launch of a matching-solver kernel (PROF_MATCH_GRAD or PROF_MATCH_COST).
enum { PROF_MATCH_GRAD = 0, PROF_MATCH_COST = 1, PROF_MATCH_KINDS = 2 };
bool profiling_on();
void profile_match(int kind, double ms);

// Kernel-launch counter (host side).  Launches issued while a stream is being
// captured are not counted; each replay of a graph counts its kernels.
void count_launch(unsigned n = 1);
void set_capturing(bool on);

// Opts kernel `fn` in to `bytes` of dynamic shared memory on the current
// device.  The attribute belongs to one device, so it is set once per device
// ordinal (bit d of `devs`, one word per kernel at the call site); ordinals
// from 64 up set it on every call.
template <typename K>
inline cudaError_t opt_in_smem(K *fn, int bytes, std::atomic<unsigned long long> &devs) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
    if (bit && (devs.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) devs.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

}  // namespace dtb
