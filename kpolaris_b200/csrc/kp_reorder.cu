// kp_reorder.cu -- longest-first order for the near-B queue.  Before a near-B
// launch the rays waiting for it are regrouped by the number of pass-A steps
// they took (power-of-two buckets, most steps first): rays that crossed the
// plasma the long way round (photon-ring rays) start first and short rays
// fill the lanes at the end, so fewer lanes idle while the last rays finish.
// The order in which rays run never changes their arithmetic, so results
// are bit-identical to any other order.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_persistent.cuh"

namespace kp {

// eight buckets per octave of pass-A steps (most RIAF rays take 1000-2000)
constexpr int kLptBuckets = 256;

__device__ __forceinline__ int lpt_bucket(const RayRecord* pool, unsigned id) {
    const LaneState* ls = reinterpret_cast<const LaneState*>(pool[id].st);
    const unsigned steps = unsigned(ls->pa_steps) + 8u;  // >= 8: three bits below the leading one
    const int lg = 31 - __clz(steps);
    const int key = lg * 8 + int((steps >> (lg - 3)) & 7u);  // < 256
    return (kLptBuckets - 1) - key;  // 0 holds the longest rays
}

// hist[b]: rays per bucket, one global atomic per bucket and block.
__global__ void __launch_bounds__(256) lpt_histogram(const unsigned* ids, const unsigned* count,
                                                    const RayRecord* pool, unsigned* hist) {
    __shared__ unsigned sh[kLptBuckets];
    for (int b = threadIdx.x; b < kLptBuckets; b += blockDim.x) sh[b] = 0u;
    __syncthreads();
    const unsigned n = *count;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&sh[lpt_bucket(pool, ids[i])], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kLptBuckets; b += blockDim.x)
        if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// out: ids grouped by bucket; each block reserves its slice of every bucket
// with one atomic per bucket (cursor[b] counts placed rays of bucket b).
__global__ void __launch_bounds__(256) lpt_scatter(const unsigned* ids, const unsigned* count, const RayRecord* pool,
                                                  const unsigned* hist, unsigned* cursor, unsigned* out) {
    __shared__ unsigned start[kLptBuckets], local[kLptBuckets], base[kLptBuckets];
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int b = 0; b < kLptBuckets; ++b) {
            start[b] = acc;
            acc += hist[b];
        }
    }
    const unsigned n = *count;
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned i0 = blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        for (int c = threadIdx.x; c < kLptBuckets; c += blockDim.x) local[c] = 0u;
        __syncthreads();
        const unsigned i = i0 + threadIdx.x;
        int b = -1;
        unsigned id = 0, slot = 0;
        if (i < n) {
            id = ids[i];
            b = lpt_bucket(pool, id);
            slot = atomicAdd(&local[b], 1u);
        }
        __syncthreads();
        for (int c = threadIdx.x; c < kLptBuckets; c += blockDim.x)
            if (local[c]) base[c] = atomicAdd(&cursor[c], local[c]);
        __syncthreads();
        if (b >= 0) out[start[b] + base[b] + slot] = id;
        __syncthreads();
    }
}

cudaError_t launch_lpt_order(const unsigned* ids, const unsigned* count, const RayRecord* pool, unsigned* scratch,
                             unsigned* out, int sms, cudaStream_t stream) {
    unsigned* hist = scratch;
    unsigned* cursor = scratch + kLptBuckets;
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned) * 2 * kLptBuckets, stream);  // hist, cursor
    if (e != cudaSuccess) return e;
    const int blocks = sms * 4;
    lpt_histogram<<<blocks, 256, 0, stream>>>(ids, count, pool, hist);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    lpt_scatter<<<blocks, 256, 0, stream>>>(ids, count, pool, hist, cursor, out);
    return cudaGetLastError();
}

}  // namespace kp
