// kp_launch.h -- internal launch interface between the C-ABI host code
// (kp_capi.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "kp_common.cuh"

namespace kp {

// Plain FP64 kernel, one thread per pixel, one image (kp_kernels_fp64.cu).
cudaError_t launch_image_fp64(const ImageConsts& c, const ImageOutPtrs& out, cudaStream_t stream);
// Analysis mode: the per-pixel FP64 image with the line-of-sight
// diagnostics (one frequency; radial_bins in 1..24).
constexpr int kMaxRadialBins = 24;  // KPOLARIS_MAX_ANALYSIS_RADIAL_BINS

struct AnalysisConsts {
    int radial_bins;
    double radial_min, radial_max, formation_fraction;
};

// Device arrays of the analysis outputs: scalars [npix]; radial arrays
// [radial_bins][npix].
struct AnalysisPtrs {
    double* radiating_path_length;
    double* emission_weight;
    double* emission_weighted_radius;
    double* emission_weighted_optical_depth_to_camera;
    double* absorption_depth;
    double* absorption_operator_depth;
    double* faraday_rotation_depth;
    double* faraday_conversion_depth;
    double* faraday_operator_depth;
    double* dominant_emission_radius;
    int32_t* dominant_emission_region;
    double* dominant_ne_cgs;
    double* dominant_thetae;
    double* dominant_b_cgs;
    double* dominant_beta;
    double* dominant_sigma;
    double* emission_weighted_ne_cgs;
    double* emission_weighted_thetae;
    double* emission_weighted_b_cgs;
    double* emission_weighted_beta;
    double* emission_weighted_sigma;
    double* photon_ring_winding_estimate;
    int32_t* radiation_substeps;
    double* radial_stokes_i;
    double* radial_stokes_q;
    double* radial_stokes_u;
    double* radial_stokes_v;
    double* radial_absorption_depth;
    double* radial_faraday_rotation_depth;
    double* radial_faraday_conversion_depth;
    double* radial_faraday_operator_depth;
    double* observer_weighted_radius_i;
    double* observer_weighted_radius_linear;
    double* observer_weighted_radius_circular;
    double* intensity_formation_radius_low;
    double* intensity_formation_radius_median;
    double* intensity_formation_radius_high;
    double* linear_formation_radius_low;
    double* linear_formation_radius_median;
    double* linear_formation_radius_high;
    double* circular_formation_radius_low;
    double* circular_formation_radius_median;
    double* circular_formation_radius_high;
    double* los_linear_coherence;
    double* los_circular_coherence;
    double* contribution_closure_max_abs;
    double* contribution_closure_relative_l1;
    double* foreground_absorption_depth;
    double* foreground_faraday_rotation_depth;
    double* foreground_faraday_conversion_depth;
    double* foreground_faraday_operator_depth;
    double* foreground_faraday_operator_fraction;
};

cudaError_t launch_image_fp64_analysis(const ImageConsts& c, const AnalysisConsts& k, const ImageOutPtrs& out,
                                       const AnalysisPtrs& an, const kp_response_config* resp, double* resp_data,
                                       cudaStream_t stream);

// Camera tetrad of an image, evaluated on the host (bit-identical to the
// reference's CPU evaluation): Cartesian Kerr-Schild, or Boyer-Lindquist for
// a kSceneRiafBL image.
void host_camera_frame(const ImageConsts& c, double frame[5][4]);

// Wavefront engine: one launch of `phase` (kPhaseFar / kPhaseNear) over the
// inputs described by `W` (a host copy whose pointers are device pointers).
// nf_max: the largest frequency count of the launch's jobs.
cudaError_t launch_wave_fp64(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                             cudaStream_t stream);
cudaError_t launch_wave_mixed(int phase, const WaveDesc& W, int blocks, int threads, cudaStream_t stream);
// Resident CTAs per SM of a phase kernel at `threads` per CTA.
int wave_occupancy_fp64(int phase, int nf_max, int threads);
int wave_occupancy_mixed(int phase, int threads);

// Seed kernels of the serving loop (same translation unit, hence the same
// camera-ray arithmetic, as the policy's phase kernels): initial records of
// the rays of newly admitted jobs, appended to the far queue.
cudaError_t launch_seed_fp64(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                             long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                             cudaStream_t stream);
cudaError_t launch_seed_mixed(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                              long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                              cudaStream_t stream);

// The GRMHD scene (FMKS metric, grid plasma), FP64 policy
// (kp_kernels_grmhd.cu), its seed kernel and the derived-scalar precompute
// (derived: [5][n1][n2][n3] device array).
cudaError_t launch_wave_grmhd(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                              cudaStream_t stream);
int wave_occupancy_grmhd(int phase, int nf_max, int threads);
// The same scene under the mixed policy (kp_kernels_grmhd_mixed.cu).
cudaError_t launch_wave_grmhd_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                                    cudaStream_t stream);
int wave_occupancy_grmhd_mixed(int phase, int nf_max, int threads);
cudaError_t launch_seed_grmhd_mixed(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix,
                                    int nentries, long long total, RayRecord* pool, unsigned* far_ids,
                                    unsigned* far_count, cudaStream_t stream);
// The RIAF in Boyer-Lindquist coordinates, FP64 policy (kp_kernels_bl.cu)
// and mixed policy (kp_kernels_bl_mixed.cu).
cudaError_t launch_wave_bl(int phase, const WaveDesc& W, int nf_max, int blocks, int threads, cudaStream_t stream);
int wave_occupancy_bl(int phase, int nf_max, int threads);
cudaError_t launch_wave_bl_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                                 cudaStream_t stream);
int wave_occupancy_bl_mixed(int phase, int nf_max, int threads);
// Longest-first order of a near-B queue (kp_reorder.cu): `count` ids from
// `ids` into `out`, grouped by pass-A steps, most first; `scratch` holds 512
// unsigned counters.
cudaError_t launch_lpt_order(const unsigned* ids, const unsigned* count, const RayRecord* pool, unsigned* scratch,
                             unsigned* out, int sms, cudaStream_t stream);
// Slow-light GRMHD (kp_kernels_grmhd_slow.cu, kp_kernels_grmhd_slow_mixed.cu).
cudaError_t launch_wave_grmhd_slow(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                                   cudaStream_t stream);
int wave_occupancy_grmhd_slow(int phase, int nf_max, int threads);
cudaError_t launch_wave_grmhd_slow_mixed(int phase, const WaveDesc& W, int nf_max, int blocks, int threads,
                                         cudaStream_t stream);
int wave_occupancy_grmhd_slow_mixed(int phase, int nf_max, int threads);
cudaError_t launch_seed_grmhd(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix, int nentries,
                              long long total, RayRecord* pool, unsigned* far_ids, unsigned* far_count,
                              cudaStream_t stream);
// Reference-layout primitives [8][ncell] into the cell-major device grid.
cudaError_t launch_grid_to_cells(const float* soa, float* cells, long long ncell, int sms, cudaStream_t stream);
cudaError_t launch_grid_derived(const GridConsts& g, double* derived, int sms, cudaStream_t stream);

// Launches of one wavefront batch run in cycles of (far, near-A, near-B)
// until no ray is left; a batch whose rays still move between phases after
// this many cycles ends with KP_ERR_TIMEOUT (a 256x256 image takes 2 cycles,
// rays grazing the radiating sphere a few more).
constexpr int kMaxWaveCycles = 24;

// Threads per CTA of each phase kernel (its __launch_bounds__): the far
// kernel runs two CTAs of 128 per SM, the near kernels one CTA of 256, so
// that every resident warp of an SM steps through the same code region.
constexpr int kFarThreads = 128;
constexpr int kNearThreads = 256;
inline int wave_threads(int phase) { return phase == kPhaseFar ? kFarThreads : kNearThreads; }

}  // namespace kp
