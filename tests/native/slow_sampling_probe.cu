// Test probe (test infrastructure, not part of the library): runs the slow-light
// engine's time sampling -- series_bracket (the snapshot pair and clamped
// fraction of a sample's fluid time) and time_interp (the fluid value between
// the pair) from kpolaris_b200/csrc/kp_grmhd.cuh -- on the GPU, one thread per
// sample, so tests can compare it with the reference's own functions.  Built
// by tests/test_gpu_slow_light.py with the floating-point flags of the
// slow-light kernel units (FP64: --fmad=false; mixed: --fmad=true
// --use_fast_math).
#include <cuda_runtime.h>

#include <cstring>

#include "kp_grmhd.cuh"

namespace {

__global__ void sampling_kernel(const double* times, int nsnap, double t_obs, const double* x0, const double* a,
                                const double* b, int n, int* window, double* fraction, double* value) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    kp::ImageConsts c;
    memset(&c, 0, sizeof(c));
    c.series_times = times;
    c.nseries = nsnap;
    c.t_obs = t_obs;
    double f = 0.0;
    window[i] = kp::series_bracket(c, x0[i], f);
    fraction[i] = f;
    value[i] = kp::time_interp(a[i], b[i], f);
}

}  // namespace

// Host arrays in and out; returns 0 or a cudaError_t.
extern "C" int kp_probe_slow_light_sampling(const double* times, int nsnap, double t_obs, const double* x0,
                                            const double* a, const double* b, int n, int* window, double* fraction,
                                            double* value) {
    if (nsnap < 2 || n <= 0) return int(cudaErrorInvalidValue);
    double *d_t = nullptr, *d_x = nullptr, *d_a = nullptr, *d_b = nullptr, *d_f = nullptr, *d_v = nullptr;
    int* d_w = nullptr;
    const size_t nb = sizeof(double) * size_t(n);
    cudaError_t e = cudaMalloc(&d_t, sizeof(double) * size_t(nsnap));
    if (e == cudaSuccess) e = cudaMalloc(&d_x, nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_a, nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_b, nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_f, nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_v, nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_w, sizeof(int) * size_t(n));
    if (e == cudaSuccess) e = cudaMemcpy(d_t, times, sizeof(double) * size_t(nsnap), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_x, x0, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_a, a, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_b, b, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        sampling_kernel<<<(n + 127) / 128, 128>>>(d_t, nsnap, t_obs, d_x, d_a, d_b, n, d_w, d_f, d_v);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(window, d_w, sizeof(int) * size_t(n), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(fraction, d_f, nb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(value, d_v, nb, cudaMemcpyDeviceToHost);
    cudaFree(d_t);
    cudaFree(d_x);
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(d_f);
    cudaFree(d_v);
    cudaFree(d_w);
    return int(e);
}
