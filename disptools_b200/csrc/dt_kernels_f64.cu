// FP64 instantiation of the stencil kernels.  This file is compiled with
// -fmad=false: no multiply-add contraction, so every per-voxel expression
// rounds exactly as the reference C library computes it.
#include "dt_kernels_tma.cuh"

namespace dtb {
DTB_INSTANTIATE(double)
DTB_INSTANTIATE_TMA(double)
}
