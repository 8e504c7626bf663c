/*
 * disptools_b200 — C ABI of the B200 (sm_100a) displacement-field generator.
 *
 * Drop-in for the CUDA entry points of disptools v0.4.1 and the C99 calls
 * its `_disptools` NumPy extension binds, plus explicit-precision,
 * statistics-returning and device-pointer entry points.
 *
 * All functions are `extern "C"` with plain pointers and sizes.  Arrays use
 * the reference layout (src/headers/disptools.h:30-36 of the reference):
 * vector fields are [3][nz][ny][nx] (component-major, x fastest), scalar maps
 * [nz][ny][nx], masks `bool` (one byte per voxel).
 *
 * FLOATING at this ABI is `double` (the reference built with FLOAT_SIZE=64,
 * which is the correctness oracle for this library).  The device arithmetic
 * is selected separately (DTB_PRECISION_*): the default mixed path stores
 * the field in FP32 and evaluates the stencils in FP32 while every cost
 * reduction and every step-control decision is FP64.
 *
 * Errors follow the reference convention: the reference-named functions
 * return void and set a process-wide error state that callers poll with
 * disptools_has_error() (src/headers/disptools.h:202-264); the dtb_*
 * functions also return 0 on success and a negative code on failure.
 */
#ifndef DISPTOOLS_B200_H
#define DISPTOOLS_B200_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Error state                                                         */
/* ------------------------------------------------------------------ */

/* Same fields and sizes as the reference's disptools_error_state
 * (src/headers/disptools.h:204-211). */
typedef struct disptools_error_state {
    bool error;
    int line;
    char file[512];
    char function[512];
    char message[1024];
    char trace[4096];
} disptools_error_state;

/* Replaces disptools_get_error (src/headers/disptools.h:250, src/disptools.c:26-29). */
disptools_error_state *disptools_get_error(void);
/* Replaces disptools_has_error (src/headers/disptools.h:257, src/disptools.c:31-34). */
bool disptools_has_error(void);
/* Replaces disptools_clear_error (src/headers/disptools.h:264, src/disptools.c:36-43). */
void disptools_clear_error(void);
/* Replaces get_float_type_size (src/headers/disptools.h:289, src/disptools.c:45-48).
 * Returns 64: FLOATING is double at this ABI. */
int get_float_type_size(void);

/* ------------------------------------------------------------------ */
/* Reference-named entry points (FLOATING = double)                    */
/* ------------------------------------------------------------------ */

/* Replaces set_device (cuda/headers/generate_displacement.cuh:11,
 * cuda/device.cu:4-15): false when `id` is not a valid device. */
bool set_device(const int id);

/* Replaces generate_displacement_gradient_cuda
 * (cuda/headers/generate_displacement.cuh:39-62) with the semantics of the
 * C library's generate_displacement_gradient
 * (src/displacement_field_gradient.c:191-431): one-sided Jacobian at the
 * boundary, mask-restricted maximum error, last accepted field returned.
 * `field` is the initial guess on entry and the result on exit.  The device
 * precision is the process default (dtb_set_default_precision). */
void generate_displacement_gradient_cuda(
    const size_t nx, const size_t ny, const size_t nz,
    const double dx, const double dy, const double dz,
    const double *J, const bool *mask,
    const double epsilon, const double tolerance, double eta, const double eta_max,
    const double alpha, const double beta, const double gamma, const double delta,
    const double zeta, const double theta, const double iota,
    const bool strict, const size_t it_max, double *field);

/* Replaces generate_displacement_greedy_cuda
 * (cuda/headers/generate_displacement.cuh:14-37) with the semantics of
 * generate_displacement_greedy (src/displacement_field_greedy.c:85-247):
 * the step length shrinks with eta on every rejection. */
void generate_displacement_greedy_cuda(
    const size_t nx, const size_t ny, const size_t nz,
    const double dx, const double dy, const double dz,
    const double *J, const bool *mask,
    const double epsilon, const double tolerance, double eta, const double eta_max,
    const double alpha, const double beta, const double gamma, const double delta,
    const double zeta, const double theta, const double iota,
    const bool strict, const size_t it_max, double *field);

/* Replaces volume_matching_3d (src/headers/VolumeMatching3D.h,
 * src/VolumeMatching3D.c:689-796), the `matching` algorithm, on the current
 * device.  As in the reference, only epsilon (stop when the maximum voxel
 * error of the last cost evaluation is below it), delta and zeta (the
 * Jacobian barrier) and it_max are used, the arithmetic is FP32, and the
 * mask is not used. */
void volume_matching_3d(
    const size_t nx, const size_t ny, const size_t nz,
    const double dx, const double dy, const double dz,
    const double *J, const bool *mask,
    const double epsilon, const double tolerance, double eta, const double eta_max,
    const double alpha, const double beta, const double gamma, const double delta,
    const double zeta, const double theta, const double iota,
    const bool strict, const size_t it_max, double *field);

/* Replaces jacobian_dynamic (src/headers/jacobian.h:24-33,
 * src/jacobian.c:7-21), computed on the current device in FP64. */
void jacobian_dynamic(
    const size_t nx, const size_t ny, const size_t nz,
    const double dx, const double dy, const double dz,
    const double *f, double *J);

/* Replaces regularise (src/headers/jacobian.h:13-19, src/jacobian.c:29-55):
 * J[i] = max(J[i], epsilon) in place, on the current device. */
void regularise(const size_t nx, const size_t ny, const size_t nz,
                double *J, double epsilon);

/* ------------------------------------------------------------------ */
/* Explicit entry points                                               */
/* ------------------------------------------------------------------ */

enum {
    DTB_PRECISION_MIXED = 0, /* FP32 field and stencils, FP64 reductions/control */
    DTB_PRECISION_FP64 = 1   /* FP64 everywhere */
};

enum {
    DTB_ALGORITHM_GRADIENT = 0,
    DTB_ALGORITHM_GREEDY = 1,
    DTB_ALGORITHM_MATCHING = 2 /* single volumes, FP32 (dtb_volume_matching) */
};

enum {
    DTB_OK = 0,
    DTB_ERR_ARGUMENT = -1,
    DTB_ERR_CUDA = -2,
    DTB_ERR_ALLOC = -3,
    DTB_ERR_DEVICE = -4,
    DTB_ERR_IO = -5 /* a file could not be opened, read, written or parsed */
};

/* Why a solve stopped; the stopping conditions of
 * src/displacement_field_gradient.c:387-410 and
 * src/displacement_field_greedy.c:193-228. */
enum {
    DTB_STOP_IT_MAX = 0,
    DTB_STOP_ERROR_EXPLODED = 1,
    DTB_STOP_ETA = 2,
    DTB_STOP_THETA = 3,
    DTB_STOP_MAX_EXPLODED = 4,
    DTB_STOP_EPSILON = 5
};

/* The 13 scalar solver parameters of the reference signature, in order
 * (DisplacementFunction, python_c_extension/_disptools.c:62-85). */
typedef struct dtb_params {
    double epsilon, tolerance, eta, eta_max, alpha, beta, gamma, delta, zeta,
        theta, iota;
    int strict;
    long long it_max;
} dtb_params;

/* Statistics of one solve (the reference prints these only when verbose). */
typedef struct dtb_solve_stats {
    long long iterations; /* loop counter when the loop ended */
    long long trials;     /* candidate fields evaluated */
    long long gradients;  /* gradient evaluations */
    int reason;           /* DTB_STOP_* */
    int precision;        /* DTB_PRECISION_* used */
    double error;         /* total error of the returned field (FP64 sum) */
    double max_error;     /* masked max |J - J_t| of the returned field */
    double cand_error;    /* total error of the last evaluated candidate */
    double cand_max_error;
    double eta;           /* final step length */
    double device_ms;     /* device time of the solve loop (CUDA events) */
} dtb_solve_stats;

/* Process-wide precision of the reference-named solver entry points.
 * The initial value is DTB_PRECISION_MIXED, or DTB_PRECISION_FP64 when the
 * environment variable DISPTOOLS_B200_PRECISION is "fp64" at load time. */
int dtb_set_default_precision(int precision);
int dtb_get_default_precision(void);

/* One solve on the current device from host arrays, with statistics
 * (`stats` may be NULL).  Returns DTB_OK or a DTB_ERR_* code; the error
 * state is set as well. */
int dtb_generate_displacement(
    int algorithm, int precision,
    size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const double *J, const bool *mask, const dtb_params *params,
    double *field, dtb_solve_stats *stats);

/* One volume of a batched solve (host arrays). */
typedef struct dtb_volume {
    size_t nx, ny, nz;
    double dx, dy, dz;
    const double *J;
    const bool *mask;
    double *field; /* in: initial guess, out: result */
} dtb_volume;

/* Solve `count` independent volumes of any sizes together: every device
 * launch covers the tiles of all volumes still running, each volume keeps
 * its own step-control state.  `stats` (may be NULL) has `count` entries. */
int dtb_generate_displacement_batched(
    int algorithm, int precision, int count, const dtb_volume *volumes,
    const dtb_params *params, dtb_solve_stats *stats);

/* One volume of a device-resident solve: `J` and `field` are device
 * pointers of the element type of the precision (float for MIXED, double for
 * FP64), `mask` a device array of one byte per voxel. */
typedef struct dtb_device_volume {
    size_t nx, ny, nz;
    double dx, dy, dz;
    const void *J;
    const void *mask;
    void *field; /* in: initial guess, out: result (device) */
} dtb_device_volume;

/* Batched solve of device-resident volumes on `stream` (a cudaStream_t or
 * NULL).  Scratch memory comes from the library's device workspace. */
int dtb_generate_displacement_batched_device(
    int algorithm, int precision, int count, const dtb_device_volume *volumes,
    const dtb_params *params, dtb_solve_stats *stats, void *stream);

/* The matching solver (volume_matching_3d) with statistics: iterations,
 * final cost (error), maximum voxel error of the last cost evaluation
 * (max_error), final step (eta), stop reason.  Host arrays, current
 * device; needs at least 2 voxels per axis. */
int dtb_volume_matching(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                        const double *J, const bool *mask, const dtb_params *params,
                        double *field, dtb_solve_stats *stats);

/* The matching solver on device arrays: `J` [nz][ny][nx] and `field`
 * [3][nz][ny][nx] (in: initial guess, out: result) are device pointers of
 * doubles; the work runs on `stream` (a cudaStream_t or NULL).  Its step
 * control reads every cost evaluation on the host, so the call returns once
 * the solve is complete.  dtb_generate_displacement_batched_device with
 * DTB_ALGORITHM_MATCHING and DTB_PRECISION_FP64 runs this per volume. */
int dtb_volume_matching_device(size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
                               const double *J, const dtb_params *params, double *field,
                               dtb_solve_stats *stats, void *stream);

/* Jacobian determinant of a device-resident field (reference stencil and
 * boundary rules, src/jacobian.c:70-242).  `field` is [3][nz][ny][nx] and
 * `J` [nz][ny][nx], both device pointers of the element type of
 * `precision` (float for MIXED, double for FP64); `order` is the interior
 * finite-difference order, 4 (the reference default ORDER_PD) or 2;
 * `stream` is a cudaStream_t or NULL.  The work is enqueued on `stream`:
 * with order 4, rows a multiple of 16 bytes long, `field` 16-byte aligned
 * and `J` aligned to two elements, the call returns without waiting for the
 * device; otherwise it returns once the map is complete. */
int dtb_jacobian_device(
    int precision, int order, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const void *field, void *J, void *stream);

/* Adjoint of dtb_jacobian_device: grad_field = (dJ/dfield)^T grad_J, the
 * exact transpose of the position-dependent stencil (fourth order inside,
 * second order on the penultimate and outer layers).  Device pointers as
 * above; grad_field is overwritten.  The work is enqueued on `stream` and
 * the call returns without waiting for the device; calls on different
 * streams are ordered on the device (they share one weight buffer). */
int dtb_jacobian_adjoint_device(
    int precision, int order, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const void *field, const void *grad_J, void *grad_field, void *stream);

/* The differentiable Jacobian split differently from the pair above: the
 * forward also writes C[c][a] = cof_ca(I + A) * ih_a, the cofactors of the
 * stencil matrix times the inverse spacing ([9][nz][ny][nx], c major), and
 * the adjoint then needs only C and grad_J (grad_field = the gather of
 * grad_J * C over the stencil's taps), so no pass re-reads the field.  No
 * counterpart in the reference.  Fourth order only; rows a multiple of 16
 * bytes long, `field`, `C` and `grad_J` 16-byte aligned, `J` and
 * `grad_field` aligned to two elements; other layouts return
 * DTB_ERR_ARGUMENT (use dtb_jacobian_device / dtb_jacobian_adjoint_device).
 * The gradient equals dtb_jacobian_adjoint_device's up to the rounding of
 * grad_J * (cof * ih) against (grad_J * cof) * ih.  Enqueued on `stream`, no
 * wait, no device memory of their own. */
int dtb_jacobian_cof_device(
    int precision, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const void *field, void *J, void *C, void *stream);
int dtb_jacobian_adjoint_cof_device(
    int precision, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const void *C, const void *grad_J, void *grad_field, void *stream);

/* Jacobian determinant of a device-resident field, like dtb_jacobian_device,
 * but without allocating any memory.  No counterpart in the reference.  It
 * is for callers that cannot let the library allocate device memory: hosts
 * that fix their memory budget at start-up (a later cudaMalloc may fail, and
 * cudaMalloc / cudaFree can synchronise the device and stall a loop with a
 * deadline), processes whose device memory another allocator has already
 * reserved, and runtimes that hand the library pointers into memory they
 * manage.  Its launch descriptor and tile table live in a 65 KiB array in
 * device memory that belongs to the library and is held by every GPU that
 * loads it until the process exits.  The first call on a device looks up
 * that array's address (cudaGetSymbolAddress), so make it before any stream
 * capture.  Volumes up to 16384 tiles of 32 x 8 x 32 voxels (512^3) are
 * accepted; larger ones return DTB_ERR_ARGUMENT before any device work.
 * All calls on a device share the array and it keeps the last call's
 * contents: calls whose work overlaps on the GPU race, so consecutive calls
 * on one device must use one stream or be ordered by an event. */
int dtb_jacobian_device_noalloc(
    int precision, int order, size_t nx, size_t ny, size_t nz, double dx, double dy, double dz,
    const void *field, void *J, void *stream);

/* ------------------------------------------------------------------ */
/* Multi-resolution pyramid: smoothing and resampling                  */
/* ------------------------------------------------------------------ */

enum {
    DTB_RESAMPLE_LINEAR = 0,
    DTB_RESAMPLE_NEAREST = 1
};

/* Gaussian smoothing of `comps` device volumes [comps][nz][ny][nx] (the
 * anti-aliasing step of scale_image, disptools/drawing.py:62-66, which
 * smooths by 2.0 physical units: sigma = 2.0 / spacing voxels per axis),
 * as a sampled Gaussian: weights exp(-k^2 / (2 sigma^2)) for
 * |k| <= ceil(4 sigma) normalised to sum 1, zero-flux border; sigma <= 0
 * leaves an axis alone, sigma is at most 32 voxels.  Sums are formed in
 * double.  `in`, `out` and `scratch` are device arrays of the precision's
 * element type that must not overlap.  Enqueued on `stream` (a cudaStream_t
 * or NULL).  The pyramid uses dtb_smooth_recursive_device unless asked for
 * this filter. */
int dtb_smooth_device(int precision, int comps, size_t nx, size_t ny, size_t nz,
                      double sigma_x, double sigma_y, double sigma_z,
                      const void *in, void *out, void *scratch, void *stream);

/* The same smoothing as the recursive Gaussian that scale_image's
 * sitk.SmoothingRecursiveGaussian (disptools/drawing.py:67) is built on:
 * R. Deriche, "Recursively implementing the Gaussian and its derivatives",
 * INRIA RR-1893 (1993), fourth-order causal and anticausal recursions per
 * axis with Deriche's coefficients, unit DC gain, each recursion started in
 * the steady state of the border value (zero flux).  sigma <= 0 leaves an
 * axis alone, sigma is at most 256 voxels; arguments as dtb_smooth_device.
 * Arithmetic in double with a fixed operation order. */
int dtb_smooth_recursive_device(int precision, int comps, size_t nx, size_t ny, size_t nz,
                                double sigma_x, double sigma_y, double sigma_z,
                                const void *in, void *out, void *scratch, void *stream);

/* Resampling of `comps` device volumes onto an nx2 x ny2 x nz2 grid that
 * spans the same physical extent (the resampler of scale_image,
 * disptools/drawing.py:54-68: output spacing s * n / n2, same origin):
 * output voxel i samples the input at continuous index i * n / n2 per axis;
 * points outside [-0.5, n - 0.5) on any axis get 0.  DTB_RESAMPLE_LINEAR
 * interpolates (x, then y, then z, neighbour indices clamped into the
 * volume), DTB_RESAMPLE_NEAREST takes floor(p + 0.5). */
int dtb_resample_device(int precision, int mode, int comps, size_t nx, size_t ny, size_t nz,
                        size_t nx2, size_t ny2, size_t nz2,
                        const void *in, void *out, void *stream);

/* ------------------------------------------------------------------ */
/* Jacobian-map utilities (device)                                     */
/* ------------------------------------------------------------------ */

enum {
    DTB_CLAMP_THRESHOLD = 0, /* values outside [epsilon, 1e9] become epsilon */
    DTB_CLAMP_REGULARISE = 1 /* values below epsilon become epsilon */
};

/* Volume-change map of a Jacobian map (jacobian_to_volume_change,
 * disptools/displacements.py:628-668): J <= epsilon is replaced by epsilon,
 * then out = J - 1 where J >= 1 and 1 - 1/J where J < 1.  `J` and `out` are
 * n device values of the precision's element type. */
int dtb_volume_change_device(int precision, size_t n, double epsilon, const void *J, void *out,
                             void *stream);

/* acc[i] += log(clamp(J[i])) over n values, acc in FP64: one map of the
 * geometric means of average_jacobian (mode DTB_CLAMP_THRESHOLD,
 * disptools/displacements.py:571-625) and
 * average_jacobian_from_displacements (DTB_CLAMP_REGULARISE, :486-568). */
int dtb_log_jacobian_accumulate_device(int precision, int mode, size_t n, double epsilon,
                                       const void *J, double *acc, void *stream);

/* out[i] = exp(scale * acc[i]): the geometric mean, scale = 1 / maps. */
int dtb_exp_mean_device(int precision, size_t n, double scale, const double *acc, void *out,
                        void *stream);

/* ------------------------------------------------------------------ */
/* Field files (host)                                                  */
/* ------------------------------------------------------------------ */

/* Replaces write_rvf (src/headers/rvf_io.h:9-12, src/rvf_io.c:11-50): the
 * header lines "nx ny nz" and "dx dy dz" (%f), then 3 native-endian doubles
 * per voxel (x fastest, components together).  `field` is [3][nz][ny][nx].
 * The file functions return DTB_OK, DTB_ERR_ARGUMENT (invalid arguments, an
 * output array too small) or DTB_ERR_IO (the file cannot be opened, read or
 * written, is too short or malformed), with the error state set. */
int dtb_write_rvf(const char *filename, size_t nx, size_t ny, size_t nz,
                  double dx, double dy, double dz, const double *field);

/* Size and spacing of an RVF file (the spacing is parsed as float, as the
 * reference's read_rvf does, src/rvf_io.c:57-90). */
int dtb_read_rvf_header(const char *filename, size_t *nx, size_t *ny, size_t *nz,
                        double *dx, double *dy, double *dz);

/* Replaces read_rvf (src/headers/rvf_io.h:17-21, src/rvf_io.c:57-125):
 * reads the field into `field` [3][nz][ny][nx]; `capacity` is its length in
 * elements. */
int dtb_read_rvf(const char *filename, double *field, size_t capacity);

/* Replaces write_vtk (src/headers/vtk_io.h, src/vtk_io.c:74-133): legacy VTK,
 * BINARY, STRUCTURED_POINTS, origin 0, spacing (%f), SCALARS image_data
 * double nd, big-endian doubles, nd components per voxel (x fastest).
 * `data` is [nd][nz][ny][nx]. */
int dtb_write_vtk(const char *filename, int nd, size_t nx, size_t ny, size_t nz,
                  double dx, double dy, double dz, const double *data);

/* Components, size and spacing of a legacy VTK file written as above. */
int dtb_read_vtk_header(const char *filename, int *nd, size_t *nx, size_t *ny, size_t *nz,
                        double *dx, double *dy, double *dz);

/* Replaces read_vtk (src/vtk_io.c:138-215): reads the data into `data`
 * [nd][nz][ny][nx]; `capacity` is its length in elements.  Float data is
 * rejected, as by the reference. */
int dtb_read_vtk(const char *filename, double *data, size_t capacity);

/* Upper bound, in bytes, on each of the two device-memory areas the library
 * keeps (the solver workspace and the staging area of host-array calls);
 * 0 removes the bound.  A solve that needs more fails with DTB_ERR_ALLOC and
 * the error state set, before touching the device.  For hosts with a fixed
 * memory budget; the tests use it to make an allocation fail. */
int dtb_set_device_memory_limit(size_t bytes);

/* Test hook of the failure path of both solvers' trial kernel: in the
 * following solves, tile `tile` (global tile index, -1 turns the hook off)
 * of every launch that evaluates a candidate (not the evaluation of the
 * initial field) does not issue the TMA loads of its plane iteration
 * `iteration`, and every bounded wait of the trial kernel polls at most
 * `wait_limit` times.  The block's wait for the missing plane then runs
 * out: the volume is stopped with its fault flag, the block waits (bounded)
 * for the loads it did issue, which complete normally, and the solve
 * returns DTB_ERR_CUDA with the error state set; the device stays usable.
 * No fault, trap or endless wait is involved. */
int dtb_test_drop_tma_load(long long tile, int iteration, unsigned wait_limit);

/* Verbose solver output on stdout, in the reference's format: one
 * "Iteration %5ld:  total error %6e  max voxel error %6e  eta %6e" line per
 * line search (per trial for the greedy method, with its "reducing step
 * size" lines) and the termination message
 * (src/displacement_field_gradient.c:377-410,
 * src/displacement_field_greedy.c:184-228, printed there when built with
 * DISPTOOLS_VERBOSE).  The lines are collected on the device and printed
 * after each solve.  Off by default, or on when DISPTOOLS_B200_VERBOSE is
 * set (and not "0") at first use.  Returns the previous setting. */
int dtb_set_verbose(int on);

/* Tile-shape autotuner of the gradient method.  When on (the default, or
 * DISPTOOLS_B200_AUTOTUNE=0 in the environment at first use for off), the
 * first solve of a problem shape on a device (shape = element type, volume
 * count, total voxels, largest extent per axis) with at least 2^21 voxels
 * times each candidate tile shape on the solve's own geometry, one gradient
 * and one trial launch on zeroed inputs each, and keeps the fastest for
 * that shape for the rest of the process.  Shapes set in the environment
 * (DISPTOOLS_B200_TILE_X, _TRIAL_THREADS_Y, _THREADS_Y, _BZ) take
 * precedence.  Returns the previous setting (0 or 1). */
int dtb_set_autotune(int on);

/* Tile shape of the last solve on the current device: shape[0] tile width
 * in voxels, shape[1] thread rows of the trial kernel, shape[2] thread rows
 * of the gradient kernel, shape[3] planes per tile along z.  Returns
 * DTB_ERR_ARGUMENT before the first solve on the device. */
int dtb_get_tile_config(int shape[4]);

/* Trial kernel of the last gradient-method solve on the current device: 0
 * for the kernel that forms each candidate plane in a shared ring (one
 * block barrier per plane), 1 for the kernel that keeps each stage until its
 * plane was the stencil's centre, forms the candidate's taps where it reads
 * them and has no barrier in its plane loop.  The autotuner uses the first
 * (the second measured slower); DISPTOOLS_B200_TRIAL_KERNEL = formed |
 * release forces one.  Returns
 * DTB_ERR_ARGUMENT before the first solve on the device.  No counterpart in
 * the reference. */
int dtb_get_trial_kernel(void);

/* Frees the device memory the library keeps on the current device between
 * calls: the solver's workspace (pitched field buffers, descriptors, tile
 * partials) and the staging area of host-array calls, both of which grow to
 * the largest solve seen and are otherwise kept until the process exits.  No
 * counterpart in the reference, whose CUDA path allocates and frees its
 * buffers in every call (cuda/displacement_field_gradient.cu:213-236,
 * 458-467).  Returns DTB_OK; must not overlap a running call on the device. */
int dtb_release_device_memory(void);

/* Number of kernels this library has launched in the process (a counter
 * kept by the host code, for benchmarks that report launch counts; each
 * replay of a captured step graph counts the kernels it contains). */
unsigned long long dtb_kernel_launch_count(void);

/* Per-kernel profile of the solvers: launches that did work and their summed
 * device time, measured with CUDA events recorded between the kernels of the
 * step graph (gradient and greedy solvers) or around each launch (matching
 * solver) while profiling is on. */
typedef struct dtb_kernel_profile {
    char name[32];        /* "trial", "gradient" (gradient and greedy
                             solvers), "match_gradient", "match_cost"
                             (matching solver; the cost kernel includes the
                             trial move) */
    long long launches;
    double total_ms;
} dtb_kernel_profile;

/* Turns profiling on or off and clears the counters. */
int dtb_set_profiling(int on);
/* Copies up to `max` entries into `out`; returns the number written. */
int dtb_get_profile(dtb_kernel_profile *out, int max);

#ifdef __cplusplus
}
#endif

#endif /* DISPTOOLS_B200_H */
