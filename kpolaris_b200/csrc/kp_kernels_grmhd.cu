// kp_kernels_grmhd.cu -- the GRMHD scene (FMKS metric, grid plasma) of the
// wavefront engine with the FP64 policy, its seed kernel, and the per-cell
// derived-scalar precompute.  Compiled without FMA contraction so the
// arithmetic stays closest to the reference's CPU rounding.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

namespace kp {

template<int NF>
__global__ void __launch_bounds__(kFarThreads, 2) wave_far_grmhd(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseFar, SceneGrmhd>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_a_grmhd(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseNearA, SceneGrmhd>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, 1) wave_near_b_grmhd(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseNearB, SceneGrmhd>(W);
}

template<int NF>
static const void* wave_kernel_grmhd(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_far_grmhd<NF>);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_grmhd<NF>);
    return reinterpret_cast<const void*>(wave_near_b_grmhd<NF>);
}

cudaError_t launch_wave_grmhd(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                              cudaStream_t stream) {
    if (nf_max < 1 || nf_max > kMaxFreq || phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd<1>(phase) : wave_kernel_grmhd<kMaxFreq>(phase);
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, 0, stream);
}

int wave_occupancy_grmhd(int phase, int nf_max, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    const void* fn = nf_max == 1 ? wave_kernel_grmhd<1>(phase) : wave_kernel_grmhd<kMaxFreq>(phase);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0);
    return n;
}

__global__ void __launch_bounds__(128) seed_grmhd(const JobDesc* jobs, const SeedEntry* entries,
                                                 const long long* prefix, int nentries, RayRecord* pool,
                                                 unsigned* far_ids, unsigned* far_count) {
    seed_body<SceneGrmhd>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
}

cudaError_t launch_seed_grmhd(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                              long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                              cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    const int grid = int((total + 127) / 128);
    seed_grmhd<<<grid, 128, 0, stream>>>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
    return cudaGetLastError();
}

// One thread per cell, consecutive threads along phi (the innermost index):
// a warp reads 32 consecutive 32-byte primitive cells and writes 32
// consecutive 48-byte derived cells.
__global__ void __launch_bounds__(256) grid_derived_kernel(const GridConsts g, double* derived) {
    const long long ncell = (long long)g.n1 * g.n2 * g.n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < ncell;
         p += (long long)gridDim.x * blockDim.x) {
        const int k = int(p % g.n3);
        const int j = int((p / g.n3) % g.n2);
        const int i = int(p / ((long long)g.n2 * g.n3));
        double out[kNumDerived];
        grid_derived_cell(g, i, j, k, out);
        double* c = derived + (size_t)p * kDerStride;
        for (int v = 0; v < kNumDerived; ++v) c[v] = out[v];
        for (int v = kNumDerived; v < kDerStride; ++v) c[v] = 0.0;
    }
}

// Reference layout [8][ncell] -> cell-major [ncell][8]: thread p reads field
// v of cell p (coalesced over p for each v) and writes its cell as two
// 16-byte stores.
__global__ void __launch_bounds__(256) grid_to_cells_kernel(const float* soa, float* cells, long long ncell) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < ncell;
         p += (long long)gridDim.x * blockDim.x) {
        float v[kPrimStride];
        for (int f = 0; f < kPrimStride; ++f) v[f] = soa[(size_t)f * (size_t)ncell + (size_t)p];
        float4* c = reinterpret_cast<float4*>(cells + (size_t)p * kPrimStride);
        c[0] = make_float4(v[0], v[1], v[2], v[3]);
        c[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
}

cudaError_t launch_grid_to_cells(const float* soa, float* cells, long long ncell, int sms, cudaStream_t stream) {
    long long blocks = (ncell + 255) / 256;
    const long long cap = (long long)sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    grid_to_cells_kernel<<<int(blocks), 256, 0, stream>>>(soa, cells, ncell);
    return cudaGetLastError();
}

cudaError_t launch_grid_derived(const GridConsts& g, double* derived, int sms, cudaStream_t stream) {
    const long long ncell = (long long)g.n1 * g.n2 * g.n3;
    long long blocks = (ncell + 255) / 256;
    const long long cap = (long long)sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    grid_derived_kernel<<<int(blocks), 256, 0, stream>>>(g, derived);
    return cudaGetLastError();
}

}  // namespace kp
