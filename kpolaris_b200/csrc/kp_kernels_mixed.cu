// kp_kernels_mixed.cu -- the mixed-precision wavefront kernels.  FP64 ray
// state, stage combination and step control everywhere; the far kernel
// (rays beyond ImageConsts::fp32_radius) contracts the connection in FP32,
// the near kernels in FP64; radiative transfer (near-B) in FP32.  Compiled with FMA
// contraction enabled.  Both always carry four frequency channels, so the
// same compiled code traces a ray whatever the rest of the batch is.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

// resident CTAs per SM the wavefront kernels are compiled for
#ifndef KP_FAR_MIN_BLOCKS
#define KP_FAR_MIN_BLOCKS 3
#endif
#ifndef KP_NEAR_MIN_BLOCKS
#define KP_NEAR_MIN_BLOCKS 1
#endif

namespace kp {

__global__ void __launch_bounds__(kFarThreads, KP_FAR_MIN_BLOCKS) wave_far_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseFar>(W);
}

__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_a_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseNearA>(W);
}

__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_b_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseNearB>(W);
}

static const void* wave_kernel_mixed(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_far_mixed);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_mixed);
    return reinterpret_cast<const void*>(wave_near_b_mixed);
}

cudaError_t launch_wave_mixed(int phase, const WaveDesc& W, int blocks, int threads, cudaStream_t stream) {
    if (phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(wave_kernel_mixed(phase), dim3(blocks), dim3(threads), args, 0, stream);
}

__global__ void __launch_bounds__(128) seed_mixed(const JobDesc* jobs, const SeedEntry* entries,
                                                 const long long* prefix, int nentries, RayRecord* pool,
                                                 unsigned* far_ids, unsigned* far_count) {
    seed_body<SceneRiaf>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
}

cudaError_t launch_seed_mixed(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                              long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                              cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    const int grid = int((total + 127) / 128);
    seed_mixed<<<grid, 128, 0, stream>>>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
    return cudaGetLastError();
}

int wave_occupancy_mixed(int phase, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_kernel_mixed(phase), threads, 0);
    return n;
}

}  // namespace kp
