// kp_launch.h -- internal launch interface between the C-ABI host code
// (kp_capi.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include "kp_common.cuh"

namespace kp {

// Plain FP64 kernel, one thread per pixel, one image (kp_kernels_fp64.cu).
cudaError_t launch_image_fp64(const ImageConsts& c, const ImageOutPtrs& out, cudaStream_t stream);

// Camera tetrad of an image, evaluated on the host (bit-identical to the
// reference's CPU evaluation).
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

// Threads per CTA of each phase kernel (its __launch_bounds__): the far
// kernel runs two CTAs of 128 per SM, the near kernels one CTA of 256, so
// that every resident warp of an SM steps through the same code region.
constexpr int kFarThreads = 128;
constexpr int kNearThreads = 256;
inline int wave_threads(int phase) { return phase == kPhaseFar ? kFarThreads : kNearThreads; }

}  // namespace kp
