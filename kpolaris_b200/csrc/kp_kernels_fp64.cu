// kp_kernels_fp64.cu -- FP64 image kernels.  This translation unit is
// compiled with --fmad=false so every double operation rounds exactly as the
// reference's CPU code does: termination reasons and fixed-step counts are
// bit-identical to it.
//
//  * image_fp64_per_pixel: the plain form -- one thread per pixel, one launch
//    per image, the reference's per-pixel code structure.
//  * wave_far_fp64 / wave_near_fp64: the wavefront engine with the FP64
//    policy; its arithmetic is the same, so its results equal the plain
//    kernel's bit for bit whatever the batch composition.
#include <cuda_runtime.h>

#include "kp_analysis.cuh"
#include "kp_bl.cuh"
#include "kp_launch.h"
#include "kp_persistent.cuh"
#include "kp_trace_fp64.cuh"

// resident CTAs per SM the wavefront kernels are compiled for
#ifndef KP_FAR_MIN_BLOCKS
#define KP_FAR_MIN_BLOCKS 2
#endif
#ifndef KP_NEAR_MIN_BLOCKS
#define KP_NEAR_MIN_BLOCKS 1
#endif

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

// Analysis mode: the plain per-pixel form with the analysis pass B, one
// frequency (src/image/analysis_driver.hpp:409-640).  A pixel whose pass A
// ends without a valid endpoint returns zero diagnostics, as there.
__global__ void __launch_bounds__(128) image_fp64_analysis(const ImageConsts c, const CameraFrame frame,
                                                           const AnalysisConsts k, const ImageOutPtrs out,
                                                           const AnalysisPtrs an, int npix,
                                                           const kp_response_config* resp, double* resp_data) {
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= npix) return;
    const Ray cam = camera_ray(c, frame, pixel);
    Ray state = cam;
    PixelOut o;
    int pa_reason = kMaxSteps;
    const int valid = trace_pass_a(c, state, o.pass_a_steps, pa_reason);
    Stokes4<double> stokes[1];
    stokes[0] = Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    o.steps = 0;
    o.reason = pa_reason;
    AnalysisAcc a;
    analysis_zero(a);
    if (valid) trace_pass_b_analysis(c, k, state, stokes[0], o.steps, o.reason, a, resp, resp_data, pixel, npix);
    double obs[1][4];
    finish_ray<double, 1>(c, cam, state, valid, stokes, o, obs);
    if (resp && valid) {
        // finalize_response_basis (response.hpp:186-191)
        const int channels = response_channel_count(*resp);
        for (int ch = 0; ch < channels; ++ch)
            resp_write(resp_data, pixel, npix, ch, observer_stokes(resp_read(resp_data, pixel, npix, ch), o));
    }
    store_stokes<1>(out, pixel, npix, obs);
    store_diagnostics(out, pixel, o);
    ObserverAnalysis w = {};
    if (valid) {
        for (int b = 0; b < k.radial_bins; ++b) a.radial[b] = observer_stokes(a.radial[b], o);
        w = observer_analysis(a, k, Stokes4<double>{obs[0][0], obs[0][1], obs[0][2], obs[0][3]});
    }
    an.radiating_path_length[pixel] = a.radiating_path_length;
    an.emission_weight[pixel] = a.emission_weight;
    an.emission_weighted_radius[pixel] = a.emission_weighted_radius;
    an.emission_weighted_optical_depth_to_camera[pixel] = a.emission_weighted_tau;
    an.absorption_depth[pixel] = a.absorption_depth;
    an.absorption_operator_depth[pixel] = a.absorption_operator_depth;
    an.faraday_rotation_depth[pixel] = a.faraday_rotation_depth;
    an.faraday_conversion_depth[pixel] = a.faraday_conversion_depth;
    an.faraday_operator_depth[pixel] = a.faraday_operator_depth;
    an.dominant_emission_radius[pixel] = a.dominant_radius;
    an.dominant_emission_region[pixel] = a.dominant_region;
    an.dominant_ne_cgs[pixel] = a.dominant_ne;
    an.dominant_thetae[pixel] = a.dominant_thetae;
    an.dominant_b_cgs[pixel] = a.dominant_b;
    an.dominant_beta[pixel] = a.dominant_beta;
    an.dominant_sigma[pixel] = a.dominant_sigma;
    an.emission_weighted_ne_cgs[pixel] = a.w_ne;
    an.emission_weighted_thetae[pixel] = a.w_thetae;
    an.emission_weighted_b_cgs[pixel] = a.w_b;
    an.emission_weighted_beta[pixel] = a.w_beta;
    an.emission_weighted_sigma[pixel] = a.w_sigma;
    an.photon_ring_winding_estimate[pixel] = a.winding;
    an.radiation_substeps[pixel] = a.substeps;
    for (int b = 0; b < k.radial_bins; ++b) {
        const size_t idx = size_t(b) * size_t(npix) + size_t(pixel);
        an.radial_stokes_i[idx] = a.radial[b].I;
        an.radial_stokes_q[idx] = a.radial[b].Q;
        an.radial_stokes_u[idx] = a.radial[b].U;
        an.radial_stokes_v[idx] = a.radial[b].V;
        an.radial_absorption_depth[idx] = a.radial_abs[b];
        an.radial_faraday_rotation_depth[idx] = a.radial_rot[b];
        an.radial_faraday_conversion_depth[idx] = a.radial_conv[b];
        an.radial_faraday_operator_depth[idx] = a.radial_op[b];
    }
    an.observer_weighted_radius_i[pixel] = w.radius_i;
    an.observer_weighted_radius_linear[pixel] = w.radius_linear;
    an.observer_weighted_radius_circular[pixel] = w.radius_circular;
    an.intensity_formation_radius_low[pixel] = w.q[0][0];
    an.intensity_formation_radius_median[pixel] = w.q[0][1];
    an.intensity_formation_radius_high[pixel] = w.q[0][2];
    an.linear_formation_radius_low[pixel] = w.q[1][0];
    an.linear_formation_radius_median[pixel] = w.q[1][1];
    an.linear_formation_radius_high[pixel] = w.q[1][2];
    an.circular_formation_radius_low[pixel] = w.q[2][0];
    an.circular_formation_radius_median[pixel] = w.q[2][1];
    an.circular_formation_radius_high[pixel] = w.q[2][2];
    an.los_linear_coherence[pixel] = w.linear_coherence;
    an.los_circular_coherence[pixel] = w.circular_coherence;
    an.contribution_closure_max_abs[pixel] = w.closure_max_abs;
    an.contribution_closure_relative_l1[pixel] = w.closure_relative_l1;
    an.foreground_absorption_depth[pixel] = w.fg_abs;
    an.foreground_faraday_rotation_depth[pixel] = w.fg_rot;
    an.foreground_faraday_conversion_depth[pixel] = w.fg_conv;
    an.foreground_faraday_operator_depth[pixel] = w.fg_op;
    an.foreground_faraday_operator_fraction[pixel] = w.fg_op_fraction;
}

cudaError_t launch_image_fp64_analysis(const ImageConsts& c, const AnalysisConsts& k, const ImageOutPtrs& out,
                                       const AnalysisPtrs& an, const kp_response_config* resp, double* resp_data,
                                       cudaStream_t stream) {
    if (c.nfreq != 1 || k.radial_bins < 1 || k.radial_bins > kMaxRadialBins) return cudaErrorInvalidValue;
    if ((resp == nullptr) != (resp_data == nullptr)) return cudaErrorInvalidValue;
    const CameraFrame frame = camera_frame(c);
    const int npix = c.nx * c.ny;
    const int block = 128;
    const int grid = (npix + block - 1) / block;
    image_fp64_analysis<<<grid, block, 0, stream>>>(c, frame, k, out, an, npix, resp, resp_data);
    return cudaGetLastError();
}

void host_camera_frame(const ImageConsts& c, double frame[5][4]) {
    CameraFrame f;
    if (c.scene == kSceneRiafBL) {
        bl_camera_frame(c.mass, c.spin, c.cam_radius, c.inclination, f.x, f.e0, f.e1, f.e2, f.e3);
    } else {
        f = camera_frame(c);
    }
    for (int mu = 0; mu < 4; ++mu) {
        frame[0][mu] = f.x.v[mu];
        frame[1][mu] = f.e0.v[mu];
        frame[2][mu] = f.e1.v[mu];
        frame[3][mu] = f.e2.v[mu];
        frame[4][mu] = f.e3.v[mu];
    }
}

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

// The wavefront kernels of the FP64 policy.  NF is 1 for single-frequency
// launches and 4 otherwise: the per-frequency arithmetic does not depend on
// NF (the unit is compiled without FMA contraction), so every instantiation
// traces a ray bit-identically to the plain kernel.
template<int NF>
__global__ void __launch_bounds__(kFarThreads, KP_FAR_MIN_BLOCKS) wave_far_fp64(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseFar>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_a_fp64(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseNearA>(W);
}

template<int NF>
__global__ void __launch_bounds__(kNearThreads, KP_NEAR_MIN_BLOCKS) wave_near_b_fp64(const WaveDesc W) {
    persistent_body<PolicyFP64, NF, kPhaseNearB>(W);
}

template<int NF>
static const void* wave_kernel_fp64(int phase) {
    if (phase == kPhaseFar) return reinterpret_cast<const void*>(wave_far_fp64<NF>);
    if (phase == kPhaseNearA) return reinterpret_cast<const void*>(wave_near_a_fp64<NF>);
    return reinterpret_cast<const void*>(wave_near_b_fp64<NF>);
}

cudaError_t launch_wave_fp64(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                             cudaStream_t stream) {
    if (nf_max < 1 || nf_max > kMaxFreq || phase < 0 || phase >= kPhases) return cudaErrorInvalidValue;
    const void* fn = nf_max == 1 ? wave_kernel_fp64<1>(phase) : wave_kernel_fp64<kMaxFreq>(phase);
    void* args[] = {const_cast<WaveDesc*>(&W)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, 0, stream);
}

__global__ void __launch_bounds__(128) seed_fp64(const JobDesc* jobs, const SeedEntry* entries,
                                                const long long* prefix, int nentries, RayRecord* pool,
                                                unsigned* far_ids, unsigned* far_count) {
    seed_body<SceneRiaf>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
}

cudaError_t launch_seed_fp64(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                             long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                             cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    const int grid = int((total + 127) / 128);
    seed_fp64<<<grid, 128, 0, stream>>>(jobs, entries, prefix, nentries, pool, far_ids, far_count);
    return cudaGetLastError();
}

int wave_occupancy_fp64(int phase, int nf_max, int threads) {
    if (phase < 0 || phase >= kPhases) return 0;
    const void* fn = nf_max == 1 ? wave_kernel_fp64<1>(phase) : wave_kernel_fp64<kMaxFreq>(phase);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0);
    return n;
}

}  // namespace kp
