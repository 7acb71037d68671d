// kp_launch.h -- internal launch interface between the C-ABI host code
// (kp_capi.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "kp_common.cuh"

namespace kp {

struct CameraFrame;

// Plain FP64 kernel, one thread per pixel, one image (kp_kernels_fp64.cu).
cudaError_t launch_image_fp64(const ImageConsts& c, const ImageOutPtrs& out, cudaStream_t stream);

}  // namespace kp
