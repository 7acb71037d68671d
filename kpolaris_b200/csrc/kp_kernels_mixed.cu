// kp_kernels_mixed.cu -- the mixed-precision persistent image kernel:
// FP64 ray state, stage combination and step control; the connection
// contraction runs in FP32 for warps whose rays are all outside r_fp64
// (default 4 M), FP64 inside.  Compiled with FMA contraction enabled.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

#ifndef KP_PERSISTENT_MIN_BLOCKS
// resident CTAs of 128 threads per SM the persistent kernel is compiled for
#define KP_PERSISTENT_MIN_BLOCKS 2
#endif

namespace kp {

template<int NF>
__global__ void __launch_bounds__(128, KP_PERSISTENT_MIN_BLOCKS) persistent_mixed(const LaunchDesc L) {
    persistent_body<PolicyMixed, NF>(L);
}

cudaError_t launch_persistent_mixed(const LaunchDesc& L, int nf_max, int blocks, int threads,
                                    cudaStream_t stream) {
    switch (nf_max) {
    case 1: persistent_mixed<1><<<blocks, threads, 0, stream>>>(L); break;
    case 2: persistent_mixed<2><<<blocks, threads, 0, stream>>>(L); break;
    case 3: persistent_mixed<3><<<blocks, threads, 0, stream>>>(L); break;
    case 4: persistent_mixed<4><<<blocks, threads, 0, stream>>>(L); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int persistent_occupancy_mixed(int nf_max, int threads) {
    int n = 0;
    switch (nf_max) {
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persistent_mixed<1>, threads, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persistent_mixed<2>, threads, 0); break;
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persistent_mixed<3>, threads, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, persistent_mixed<4>, threads, 0); break;
    }
    return n;
}

}  // namespace kp
