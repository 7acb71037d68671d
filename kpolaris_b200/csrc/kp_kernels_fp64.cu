// kp_kernels_fp64.cu -- the plain FP64 image kernel: one thread per pixel,
// one launch per image.  This translation unit is compiled with --fmad=false
// so every double operation rounds exactly as the reference's CPU code does;
// termination reasons and fixed-step counts are bit-identical to it.
#include <cuda_runtime.h>

#include "kp_launch.h"
#include "kp_trace_fp64.cuh"

namespace kp {

template<int NF>
__global__ void __launch_bounds__(128) image_fp64_per_pixel(const ImageConsts c, const CameraFrame frame,
                                                            const ImageOutPtrs out, int npix) {
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= npix) return;
    const Ray cam = camera_ray(c, frame, pixel);
    Ray state = cam;
    PixelOut o;
    int pa_reason = kMaxSteps;
    const int valid = trace_pass_a(c, state, o.pass_a_steps, pa_reason);
    Stokes4<double> stokes[NF];
    o.steps = 0;
    o.reason = pa_reason;
    if (valid) {
        trace_pass_b_fp64<NF>(c, state, stokes, o.steps, o.reason);
    } else {
#pragma unroll
        for (int f = 0; f < NF; ++f) stokes[f] = Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    }
    double obs[NF][4];
    finish_ray<double, NF>(c, cam, state, valid, stokes, o, obs);
    store_stokes<NF>(out, pixel, npix, obs);
    store_diagnostics(out, pixel, o);
}

CameraFrame host_camera_frame(const ImageConsts& c) { return camera_frame(c); }

cudaError_t launch_image_fp64(const ImageConsts& c, const ImageOutPtrs& out, cudaStream_t stream) {
    const CameraFrame frame = camera_frame(c);
    const int npix = c.nx * c.ny;
    const int block = 128;
    const int grid = (npix + block - 1) / block;
    switch (c.nfreq) {
    case 1: image_fp64_per_pixel<1><<<grid, block, 0, stream>>>(c, frame, out, npix); break;
    case 2: image_fp64_per_pixel<2><<<grid, block, 0, stream>>>(c, frame, out, npix); break;
    case 3: image_fp64_per_pixel<3><<<grid, block, 0, stream>>>(c, frame, out, npix); break;
    case 4: image_fp64_per_pixel<4><<<grid, block, 0, stream>>>(c, frame, out, npix); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace kp
