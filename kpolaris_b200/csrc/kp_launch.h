// kp_launch.h -- internal launch interface between the C-ABI host code
// (kp_capi.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "kp_common.cuh"

namespace kp {

struct CameraFrame;

// Plain FP64 kernel, one thread per pixel, one image (kp_kernels_fp64.cu).
cudaError_t launch_image_fp64(const ImageConsts& c, const ImageOutPtrs& out, cudaStream_t stream);

struct LaunchDesc;
struct JobDesc;

// Camera tetrad of an image, evaluated on the host (bit-identical to the
// reference's CPU evaluation).
void host_camera_frame(const ImageConsts& c, double frame[5][4]);

// Persistent engine.  `L` is a host copy whose pointers are device pointers.
// precision: 0 FP64 (bit-exact arithmetic), 1 mixed.  nf_max: the largest
// frequency count of the launch's jobs.
cudaError_t launch_persistent_fp64(const LaunchDesc& L, int nf_max, int blocks, int threads,
                                   cudaStream_t stream);
cudaError_t launch_persistent_mixed(const LaunchDesc& L, int nf_max, int blocks, int threads,
                                    cudaStream_t stream);
// Resident CTAs per SM of the persistent kernels at `threads` per CTA.
int persistent_occupancy_fp64(int nf_max, int threads);
int persistent_occupancy_mixed(int nf_max, int threads);

}  // namespace kp
