// kp_kernels_grmhd_mixed.cu -- the GRMHD scene (FMKS metric, grid plasma) of
// the wavefront engine with the mixed policy: FP64 geodesic and grid sample,
// FP32 thermal fits and Stokes transfer with compensated accumulation.
// Compiled with FMA contraction (the mixed path is held to a flux/EVPA
// budget, not to the reference's rounding).
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

namespace kp {

template<int NF>
__global__ void __launch_bounds__(kFarThreads, 2) wave_far_grmhd_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseFar, SceneFarCks<SceneGrmhd>>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_a_grmhd_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearA, SceneGrmhd>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_b_grmhd_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, NF, kPhaseNearB, SceneGrmhd>(W);
}

template<int NF>
static const void* wave_kernel_grmhd_mixed(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_far_grmhd_mixed<NF>);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_grmhd_mixed<NF>);
    return reinterpret_cast<const void*>(wave_near_b_grmhd_mixed<NF>);
}

cudaError_t launch_wave_grmhd_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                                    cudaStream_t stream) {
    if (nf_max < 1 || nf_max > kMaxFreq || phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd_mixed<1>(phase) : wave_kernel_grmhd_mixed<kMaxFreq>(phase);
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, 0, stream);
}

int wave_occupancy_grmhd_mixed(int phase, int nf_max, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd_mixed<1>(phase) : wave_kernel_grmhd_mixed<kMaxFreq>(phase);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0);
    return n;
}

// Initial records of newly admitted GRMHD jobs' rays for the serving loop,
// compiled with this file's contraction so a served image starts from the
// same camera rays as kp_image_grmhd's mixed far kernel.
__global__ void __launch_bounds__(128) seed_grmhd_mixed(const JobDesc* jobs, const SeedEntry* entries,
                                                       const long long* prefix, int nentries, RayRecord* pool,
                                                       unsigned* far_ids, unsigned* far_count) {
    seed_body<SceneGrmhd>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
}

cudaError_t launch_seed_grmhd_mixed(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix,
                                    int nentries, long long total, RayRecord* pool, unsigned* far_ids,
                                    unsigned* far_count, cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    const int grid = int((total + 127) / 128);
    seed_grmhd_mixed<<<grid, 128, 0, stream>>>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
    return cudaGetLastError();
}

}  // namespace kp
