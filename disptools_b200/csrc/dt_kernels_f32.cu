// FP32 instantiation of the stencil kernels (mixed path: FP32 field and
// stencil arithmetic, FP64 reductions and step control).
#include "dt_kernels_tma.cuh"

namespace dtb {
DTB_INSTANTIATE(float)
DTB_INSTANTIATE_TMA(float)
}
