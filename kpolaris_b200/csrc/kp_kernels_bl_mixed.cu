// kp_kernels_bl_mixed.cu -- the RIAF in Boyer-Lindquist coordinates (SceneRiafBL)
// on the wavefront engine with the mixed policy (FP64 BL geodesic, FP32 fits and compensated transfer), compiled with FMA contraction.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

namespace kp {

template<int NF>
__global__ void __launch_bounds__(kFarThreads, 2) wave_bl_mixed_far(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseFar, SceneRiafBL>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_bl_mixed_near_a(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearA, SceneRiafBL>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_bl_mixed_near_b(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearB, SceneRiafBL>(W);
}

template<int NF>
static const void* wave_bl_mixed_kernel(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_bl_mixed_far<NF>);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_bl_mixed_near_a<NF>);
    return reinterpret_cast<const void*>(wave_bl_mixed_near_b<NF>);
}

cudaError_t launch_wave_bl_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads, cudaStream_t stream) {
    if (nf_max < 1 || nf_max > kMaxFreq || phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    const void* fn = nf_max == 1 ? wave_bl_mixed_kernel<1>(phase) : wave_bl_mixed_kernel<kMaxFreq>(phase);
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, 0, stream);
}

int wave_occupancy_bl_mixed(int phase, int nf_max, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    const void* fn = nf_max == 1 ? wave_bl_mixed_kernel<1>(phase) : wave_bl_mixed_kernel<kMaxFreq>(phase);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0);
    return n;
}

}  // namespace kp
