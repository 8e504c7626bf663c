// Element-wise Jacobian-map utilities on the device.
//
// * Volume change (jacobian_to_volume_change,
//   disptools/displacements.py:628-668): J <= epsilon is first replaced by
//   epsilon; then VC = J - 1 where J >= 1 and VC = 1 - 1/J where J < 1
//   (both tests on the original J).  A NaN stays NaN.
// * Geometric mean of several maps (average_jacobian, :571-625, and
//   average_jacobian_from_displacements, :486-568): each map is clamped,
//   its log added to an FP64 accumulator, and the mean is
//   exp((1 / n) * sum).  The clamp of average_jacobian is SimpleITK's
//   Threshold(lower = epsilon, upper = 1e9, outside = epsilon): values
//   outside [epsilon, 1e9] become epsilon.  The clamp of
//   average_jacobian_from_displacements is `regularise` (src/jacobian.c:29-55):
//   values below epsilon become epsilon.
// Divisions are IEEE (no fast math); log and exp are CUDA's.
#include <cuda_runtime.h>

#include <cstdio>

#include "dt_internal.h"

using namespace dtb;

namespace {

int grid_for(long long n) {
    const long long blocks = (n + 255) / 256;
    return (int) (blocks < 148 * 32 ? (blocks > 0 ? blocks : 1) : 148 * 32);
}

template <typename T>
__global__ void k_volume_change(const T *__restrict__ J, T *__restrict__ out, long long n, T eps) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        const T j = J[i];
        const T js = j <= eps ? eps : j;
        T v = j;  // NaN: neither branch of the reference applies
        if (j >= T(1)) v = js - T(1);
        else if (j < T(1)) v = T(1) - T(1) / js;
        out[i] = v;
    }
}

template <typename T>
__global__ void k_log_accumulate(const T *__restrict__ J, double *__restrict__ acc, long long n, double eps,
                                 int mode) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x) {
        double j = (double) J[i];
        if (mode == DTB_CLAMP_THRESHOLD)
            j = (j >= eps && j <= 1e9) ? j : eps;
        else
            j = j < eps ? eps : j;
        acc[i] += log(j);
    }
}

template <typename T>
__global__ void k_exp_mean(const double *__restrict__ acc, T *__restrict__ out, long long n, double scale) {
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n;
         i += (long long) gridDim.x * blockDim.x)
        out[i] = (T) exp(scale * acc[i]);
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

int finish(const char *function, int line) {
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        report(line, function, cudaGetErrorString(e));
        return DTB_ERR_CUDA;
    }
    return DTB_OK;
}

}  // namespace

extern "C" int dtb_volume_change_device(int precision, size_t n, double epsilon, const void *J, void *out,
                                        void *stream) {
    disptools_clear_error();
    if (!J || !out || n == 0) {
        report(__LINE__, __func__, "null array or empty map");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = grid_for((long long) n);
    if (precision == DTB_PRECISION_FP64)
        k_volume_change<double><<<grid, 256, 0, s>>>(static_cast<const double *>(J), static_cast<double *>(out),
                                                     (long long) n, epsilon);
    else if (precision == DTB_PRECISION_MIXED)
        k_volume_change<float><<<grid, 256, 0, s>>>(static_cast<const float *>(J), static_cast<float *>(out),
                                                    (long long) n, (float) epsilon);
    else {
        report(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    return finish(__func__, __LINE__);
}

extern "C" int dtb_log_jacobian_accumulate_device(int precision, int mode, size_t n, double epsilon, const void *J,
                                                  double *acc, void *stream) {
    disptools_clear_error();
    if (!J || !acc || n == 0) {
        report(__LINE__, __func__, "null array or empty map");
        return DTB_ERR_ARGUMENT;
    }
    if (mode != DTB_CLAMP_THRESHOLD && mode != DTB_CLAMP_REGULARISE) {
        report(__LINE__, __func__, "invalid clamp mode");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = grid_for((long long) n);
    if (precision == DTB_PRECISION_FP64)
        k_log_accumulate<double><<<grid, 256, 0, s>>>(static_cast<const double *>(J), acc, (long long) n, epsilon,
                                                      mode);
    else if (precision == DTB_PRECISION_MIXED)
        k_log_accumulate<float><<<grid, 256, 0, s>>>(static_cast<const float *>(J), acc, (long long) n, epsilon,
                                                     mode);
    else {
        report(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    return finish(__func__, __LINE__);
}

extern "C" int dtb_exp_mean_device(int precision, size_t n, double scale, const double *acc, void *out,
                                   void *stream) {
    disptools_clear_error();
    if (!acc || !out || n == 0) {
        report(__LINE__, __func__, "null array or empty map");
        return DTB_ERR_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = grid_for((long long) n);
    if (precision == DTB_PRECISION_FP64)
        k_exp_mean<double><<<grid, 256, 0, s>>>(acc, static_cast<double *>(out), (long long) n, scale);
    else if (precision == DTB_PRECISION_MIXED)
        k_exp_mean<float><<<grid, 256, 0, s>>>(acc, static_cast<float *>(out), (long long) n, scale);
    else {
        report(__LINE__, __func__, "invalid precision");
        return DTB_ERR_ARGUMENT;
    }
    return finish(__func__, __LINE__);
}
