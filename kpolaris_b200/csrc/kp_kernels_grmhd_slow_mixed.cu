// kp_kernels_grmhd_slow_mixed.cu -- slow-light GRMHD images (FMKS metric, grid plasma interpolated
// in time between resident snapshots) on the wavefront engine with
// the mixed policy (FP64 geodesic and grid sample, FP32 fits and transfer).  Compiled with FMA contraction.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

namespace kp {

template<int NF>
__global__ void __launch_bounds__(kFarThreads, 2) wave_far_grmhd_slow_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseFar, SceneFarCks<SceneGrmhdSlow>>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_a_grmhd_slow_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearA, SceneGrmhdSlow>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_b_grmhd_slow_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearB, SceneGrmhdSlow>(W);
}

template<int NF>
static const void* wave_kernel_grmhd_slow_mixed(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_far_grmhd_slow_mixed<NF>);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_grmhd_slow_mixed<NF>);
    return reinterpret_cast<const void*>(wave_near_b_grmhd_slow_mixed<NF>);
}

cudaError_t launch_wave_grmhd_slow_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                              cudaStream_t stream) {
    if (nf_max < 1 || nf_max > kMaxFreq || phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd_slow_mixed<1>(phase) : wave_kernel_grmhd_slow_mixed<kMaxFreq>(phase);
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, 0, stream);
}

int wave_occupancy_grmhd_slow_mixed(int phase, int nf_max, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd_slow_mixed<1>(phase) : wave_kernel_grmhd_slow_mixed<kMaxFreq>(phase);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0);
    return n;
}

}  // namespace kp
