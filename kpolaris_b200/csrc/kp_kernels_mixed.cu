// kp_kernels_mixed.cu -- the mixed-precision wavefront kernels.  FP64 ray
// state, stage combination and step control everywhere; the far kernel
// (rays beyond ImageConsts::fp32_radius) contracts the connection in FP32,
// the near kernels in FP64; radiative transfer (near-B) in FP32.  Compiled with FMA
// contraction enabled.  Both always carry four frequency channels, so the
// same compiled code traces a ray whatever the rest of the batch is.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "kp_far.cuh"
#include "kp_launch.h"
#include "kp_persistent.cuh"

// resident CTAs per SM the wavefront kernels are compiled for
#ifndef KP_FAR_MIN_BLOCKS
#define KP_FAR_MIN_BLOCKS 4
#endif
#ifndef KP_NEAR_MIN_BLOCKS
#define KP_NEAR_MIN_BLOCKS 1
#endif

namespace kp {

// The far phase: the stage-loop kernel of kp_far.cuh (dynamic shared memory
// kFarSmemBytes per CTA).
__global__ void __launch_bounds__(kFarThreads, KP_FAR_MIN_BLOCKS) wave_far_mixed(const WaveDesc W) {
    far_body<SceneRiaf, kMaxFreq, false>(W);
}

__global__ void __launch_bounds__(kFarThreads, KP_FAR_MIN_BLOCKS) wave_far_mixed_exact(const WaveDesc W) {
    far_body<SceneRiaf, kMaxFreq, true>(W);
}

__global__ void __launch_bounds__(kFarThreads, 3) wave_far_mixed_mb3(const WaveDesc W) {
    far_body<SceneRiaf, kMaxFreq, false>(W);
}

__global__ void __launch_bounds__(kFarThreads, 3) wave_far_mixed_generic(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseFar>(W);
}

// development switch between the far kernels (KP_FAR_KERNEL=fast|exact|fast3;
// default: the generic persistent body)
static int far_variant() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("KP_FAR_KERNEL");
        v = (e && !std::strcmp(e, "fast")) ? 0 : (e && !std::strcmp(e, "exact")) ? 1
            : (e && !std::strcmp(e, "fast3")) ? 3 : 2;
    }
    return v;
}

static const void* far_kernel() {
    const int v = far_variant();
    return v == 2 ? reinterpret_cast<const void*>(wave_far_mixed_generic)
           : v == 1 ? reinterpret_cast<const void*>(wave_far_mixed_exact)
           : v == 3 ? reinterpret_cast<const void*>(wave_far_mixed_mb3)
                    : reinterpret_cast<const void*>(wave_far_mixed);
}

static size_t far_smem() { return far_variant() == 2 ? 0 : kFarSmemBytes; }

__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_a_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseNearA>(W);
}

__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_b_mixed(const WaveDesc W) {
    persistent_body<PolicyMixed, kMaxFreq, kPhaseNearB>(W);
}

static const void* wave_kernel_mixed(int phase) {
    if (phase == kPhaseFar) return far_kernel();
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_mixed);
    return reinterpret_cast<const void*>(wave_near_b_mixed);
}

static size_t wave_smem_mixed(int phase) {
    if (phase != kPhaseFar) return 0;
    const size_t bytes = far_smem();
    if (bytes > 0) cudaFuncSetAttribute(far_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    return bytes;
}

cudaError_t launch_wave_mixed(int phase, const WaveDesc& W, int blocks, int threads, cudaStream_t stream) {
    if (phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    void* args[] = {const_cast<WaveDesc*>(&W)};
    const size_t smem = wave_smem_mixed(phase);
    return cudaLaunchKernel(wave_kernel_mixed(phase), dim3(blocks), dim3(threads), args, smem, stream);
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
    const size_t smem = wave_smem_mixed(phase);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_kernel_mixed(phase), threads, smem);
    return n;
}

}  // namespace kp
