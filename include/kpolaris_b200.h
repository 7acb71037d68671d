/*
 * kpolaris_b200.h -- C ABI of the B200-native KPolaris per-pixel GRRT path.
 *
 * Every entry point takes plain C structs, pointers and sizes; no C++ or
 * torch types cross this boundary.  The structs mirror the reference's
 * parameter objects field for field so that the reference's C++ call sites
 * (run_riaf_image, run_riaf_multifrequency_image, run_grmhd_image,
 * run_image_batch_metric) can be forwarded here by a thin host shim
 * (kpolaris_b200/host/kpolaris_reference_shim.hpp).
 *
 * Conventions shared by every function:
 *   - return value: KP_OK (0) on success, a negative kp_status otherwise;
 *     kp_last_error() returns a human-readable message for the calling
 *     thread's most recent failure.
 *   - per-ray failures are not errors: they are reported through the
 *     per-pixel `reason` codes (kp_termination), identical to the
 *     reference's TerminationReason (src/common/types.hpp:37-48).
 *   - image arrays are laid out [nfreq][npix], pixel = j * nx + i, exactly as
 *     ImageHostData (src/image/result.hpp:9-31) and copy_real_view_2d
 *     (src/image/driver.hpp:38-49).
 */
#ifndef KPOLARIS_B200_H
#define KPOLARIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KP_ABI_VERSION 2
/* Maximum frequencies that share one geodesic in a single launch
 * (reference compile-time KPOLARIS_MAX_FREQUENCIES, src/common/types.hpp:5-7). */
#define KP_MAX_FREQUENCIES 4
/* Longest step-control frequency list of kp_image_riaf_step_control and
 * kp_image_grmhd_step_control. */
#define KP_MAX_CONTROL_FREQUENCIES 64

typedef enum kp_status {
    KP_OK = 0,
    KP_ERR_INVALID = -1,     /* invalid argument (reference: std::invalid_argument) */
    KP_ERR_OOM = -2,         /* device or host allocation failed */
    KP_ERR_CUDA = -3,        /* CUDA runtime or launch failure */
    KP_ERR_TIMEOUT = -4,     /* a bounded device/host wait ran out */
    KP_ERR_UNSUPPORTED = -5, /* feature/combination not built (reference: std::runtime_error) */
    KP_ERR_BUSY = -6,        /* admission refused: not enough device memory / slots */
    KP_ERR_NOT_FOUND = -7,   /* unknown handle or job id */
    KP_ERR_CANCELLED = -8,   /* job was cancelled before completion */
    KP_ERR_IO = -9           /* input file missing, unreadable or malformed (reference: std::runtime_error
                                from its loaders and H5::Exception from the HDF5 library) */
} kp_status;

/* Reference CoordinateSystem (src/common/types.hpp:51-57). */
typedef enum kp_coordinate_system {
    KP_COORD_CARTESIAN_KS = 0,
    KP_COORD_BOYER_LINDQUIST = 1,
    KP_COORD_SPHERICAL_KS = 2,
    KP_COORD_FMKS = 3,
    KP_COORD_MKS = 4
} kp_coordinate_system;

/* Reference CameraModel (src/camera/camera.hpp:7-10). */
typedef enum kp_camera_model {
    KP_CAMERA_PINHOLE = 0,
    KP_CAMERA_PARALLEL_PLANE = 1
} kp_camera_model;

/* Reference TerminationReason (src/common/types.hpp:37-48). */
typedef enum kp_termination {
    KP_REASON_NONE = 0,
    KP_REASON_REACHED_CAMERA = 1,
    KP_REASON_REACHED_INNER_BOUNDARY = 2,
    KP_REASON_ESCAPED_DOMAIN = 3,
    KP_REASON_MAX_STEPS = 4,
    KP_REASON_INVALID_STATE = 5,
    KP_REASON_SLOW_LIGHT_TIME_EXHAUSTED = 6,
    KP_REASON_ADAPTIVE_STEP_UNDERFLOW = 7,
    KP_REASON_METRIC_TIME_EXHAUSTED = 8,
    KP_REASON_REACHED_DIRECT_TURN = 9
} kp_termination;

/* Thermal synchrotron fit selector (src/radiation/thermal_synchrotron.hpp:8-17). */
typedef enum kp_emission_fit {
    KP_FIT_PANDYA = 1,
    KP_FIT_DEXTER = 4
} kp_emission_fit;

/* Arithmetic used by the image kernels. */
typedef enum kp_precision {
    /* FP64 everywhere, IEEE operation order of the reference (bit-exact
     * termination status and fixed-step counts). */
    KP_PRECISION_FP64 = 0,
    /* FP64 geodesic state, step control and near-hole geometry; FP32
     * coefficients and Stokes transfer with a per-job 2^E scale and
     * compensated accumulation. */
    KP_PRECISION_MIXED = 1
} kp_precision;

/* How rays are scheduled on the device. */
typedef enum kp_schedule {
    /* One thread per pixel, one launch per image: the plain form. */
    KP_SCHEDULE_PER_PIXEL = 0,
    /* Persistent kernel draining a global ray queue with per-lane refill. */
    KP_SCHEDULE_PERSISTENT = 1,
    /* The persistent engine with its launch loop captured in a CUDA graph:
     * a fixed number of (far, near-A, near-B) cycles, the counter reset and
     * the read-back of the remaining queue counts replay as one graph
     * launch (cached per device and workload shape); rays still moving
     * after it continue in ordinary launches.  Results are bit-identical to
     * KP_SCHEDULE_PERSISTENT. */
    KP_SCHEDULE_GRAPH = 2
} kp_schedule;

/* Geodesic integrator.  The reference image path uses step-doubling RK4
 * (adaptive_rk4_step, src/geodesic/rk4.hpp:109-161); the Cash-Karp embedded
 * pair (adaptive_rkf45_endpoint_step, rk4.hpp:164-250) is an added variant. */
typedef enum kp_integrator {
    KP_INTEGRATOR_STEP_DOUBLING_RK4 = 0,
    KP_INTEGRATOR_CASH_KARP = 1
} kp_integrator;

/* Mirrors CameraParams<double> (src/camera/camera.hpp:12-25). */
typedef struct kp_camera_params {
    int nx;
    int ny;
    double radius;
    double inclination; /* radians */
    double fov;
    double fov_y;
    double xspan;
    double yspan;
    double x_offset;
    double y_offset;
    int model; /* kp_camera_model */
} kp_camera_params;

/* Mirrors EmissionSelection<double> (src/radiation/emission_selection.hpp:11-19). */
typedef struct kp_emission_selection {
    double equatorial_h_over_r;
    int equatorial_samples;
    int faraday_rotation;
} kp_emission_selection;

/* Mirrors PassAParams<double> (src/geodesic/pass_a_core.hpp:10-36). */
typedef struct kp_pass_a_params {
    kp_camera_params camera;
    kp_emission_selection emission_selection;
    double mass;
    double spin;
    double inner_radius;
    double outer_radius;
    double step;
    int max_steps;
    int adaptive;
    int direct_only;
    double adaptive_tolerance;
    double min_step;
    double max_step;
    double max_radiation_step;
    double max_radiation_depth;
    double max_absorption_depth;
    double max_faraday_depth;
    double fmks_startx1;
    double fmks_hslope;
    double fmks_mks_smooth;
    double fmks_poly_alpha;
    double fmks_poly_xt;
    double fmks_poly_norm;
    int coordinate_system; /* kp_coordinate_system */
} kp_pass_a_params;

/* Mirrors the thermal fields of RIAFAnalyticRadiationModel<double>
 * (src/model/riaf.hpp:19-52).  Non-thermal fields are not carried: the
 * thermal synchrotron fits are the only emission types on this path. */
typedef struct kp_riaf_model {
    double nth0;
    double Te0;
    double disk_h;
    double pow_nth;
    double pow_T;
    double ne_unit;
    double te_unit;
    double b_unit;
    double freq_cgs;
    double mbh_solar;
    double r_min;
    double r_max;
    double horizon_buffer;
    double emission_scale;
    double absorption_scale;
    double faraday_scale;
    double max_pol_frac;
    double keplerian_factor;
    double infall_factor;
    int emission_type; /* kp_emission_fit */
    double min_frequency_scale;
    double min_sin_theta;
    double min_thetae;
    double min_radius;
} kp_riaf_model;

/* Caller-owned output buffers (host or device memory, see kp_run_options).
 * Mirrors ImageHostData (src/image/result.hpp:9-31) without the analysis
 * fields.  image_* hold nfreq*npix doubles; diagnostics hold npix values. */
typedef struct kp_image_out {
    int npix;
    int nfreq;
    double* image_i;
    double* image_q;
    double* image_u;
    double* image_v;
    double* closure_x;
    double* closure_k;
    double* final_null;
    double* frame_error;
    double* det_r;
    double* overlap_r11;
    double* overlap_r12;
    double* overlap_r21;
    double* overlap_r22;
    double* basis_identity_error;
    double* basis_rotation_angle;
    int32_t* pass_a_steps;
    int32_t* steps;
    int32_t* reason;
} kp_image_out;

/* Launch-side options that the reference expresses through build flags and
 * extra driver arguments. */
typedef struct kp_run_options {
    int precision;       /* kp_precision */
    int schedule;        /* kp_schedule */
    int integrator;      /* kp_integrator */
    int outputs_on_device; /* 1: kp_image_out pointers are device pointers */
    int device;          /* CUDA device ordinal */
    void* stream;        /* cudaStream_t, or NULL for the library's stream */
    int timing;          /* 1: print "timing <name> <seconds> s" lines like the reference */
    /* Persistent-schedule tunables.  blocks_per_sm: 0 selects the
     * occupancy-derived CTA count.  threads_per_block must be 0: the kernels
     * fix it (128 far, 256 near). */
    int blocks_per_sm;
    int threads_per_block;
} kp_run_options;

/* Fills *opt with defaults: FP64, per-pixel, step-doubling RK4, host
 * outputs, device 0, library stream. */
void kp_default_run_options(kp_run_options* opt);

/* Fills *p / *m with the reference's struct defaults
 * (pass_a_core.hpp:10-36, camera.hpp:12-25, riaf.hpp:19-52). */
void kp_default_pass_a_params(kp_pass_a_params* p);
void kp_default_riaf_model(kp_riaf_model* m);

/* Thread-local message describing the most recent failure. */
const char* kp_last_error(void);

/* ABI version, for the bindings' load-time check. */
int kp_abi_version(void);

/* sizeof of the ABI structs, for the bindings' layout check:
 * 0 kp_camera_params, 1 kp_emission_selection, 2 kp_pass_a_params,
 * 3 kp_riaf_model, 4 kp_image_out, 5 kp_run_options, 7 kp_riaf_job,
 * 8 kp_batch_stats, 9 kp_tuning, 10 kp_grmhd_model, 11 kp_grmhd_job, 12 kp_analysis_config,
 * 13 kp_analysis_out, 14 kp_iharm_options, 15 kp_response_config; 6 is the bytes of the per-image job descriptor an
 * image uploads to the device; 0 for other ids. */
size_t kp_abi_sizeof(int which);

/* Bytes of per-pixel output (15 doubles + 3 int32 = 132 B), the figure the
 * reference's batch budget uses (src/image/batch_driver.hpp:49). */
size_t kp_image_output_bytes(int npix, int nfreq);

/* Measured FMA throughput of `device` in TFLOP/s (2 flops per FMA), FP64
 * (fp64 = 1) or FP32: the pipe roofline the image kernels are reported
 * against.  No reference counterpart (a measurement helper). */
int kp_measure_fma_peak(int device, int fp64, double* tflops);

/*
 * RIAF image, one or several frequencies sharing one geodesic per pixel.
 * Replaces run_riaf_image (src/image/riaf.hpp:12-16, nfreq == 1) and
 * run_riaf_multifrequency_image (src/image/riaf.hpp:32-39, 1..4 frequencies
 * with step-control list == frequency list).  params->coordinate_system is
 * KP_COORD_BOYER_LINDQUIST (the reference's RIAF backend,
 * src/image/backends/riaf_bl.cpp) or KP_COORD_CARTESIAN_KS; other charts
 * return KP_ERR_UNSUPPORTED.  `frequencies` may be NULL when nfreq == 1, in
 * which case model->freq_cgs is used.
 * radiation_substeps is accepted for signature compatibility; the
 * reference's segment kernels ignore it (pass_b.hpp:526, :1003).
 */
int kp_image_riaf(const kp_pass_a_params* params,
                  const kp_riaf_model* model,
                  int radiation_substeps,
                  const double* frequencies,
                  int nfreq,
                  const kp_run_options* options,
                  kp_image_out* out);

/*
 * RIAF image of 1..4 frequencies whose pass-B step control (the radiation
 * substep counts and the predictive step cap) takes the largest count over a
 * separate step-control frequency list, so that every chunk of a longer
 * frequency list follows one geodesic.  Replaces
 * run_riaf_multifrequency_image with step_control_frequencies
 * (src/image/riaf.cpp:79-105 -> run_multifrequency_image_metric_with_step_control,
 * src/image/multifrequency.hpp:152-236; per-pixel loop
 * trace_pass_b_segment_model_multifrequency_control_pixel_metric,
 * src/geodesic/pass_b.hpp:1505-1895) as the image tool calls it for each
 * chunk of its frequency grid (tools/kpolaris_model_image.cpp:3432-3446).
 * A control list equal to the frequency list (same length and values, the
 * reference's test) is the plain kp_image_riaf.  1 <= ncontrol <=
 * KP_MAX_CONTROL_FREQUENCIES; every control frequency finite and positive.
 */
int kp_image_riaf_step_control(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                               const double* frequencies, int nfreq, const double* control_frequencies,
                               int ncontrol, const kp_run_options* options, kp_image_out* out);

/*
 * Analysis mode (the reference's analysis_mode=1 image path,
 * src/image/analysis_driver.hpp): the FP64 per-pixel image with
 * line-of-sight diagnostics accumulated along pass B.  Single frequency;
 * the source-partition response channels (analysis_response) are not built.
 * kp_analysis_config mirrors AnalysisConfig (:16-23).
 */
#define KP_MAX_ANALYSIS_RADIAL_BINS 24

typedef struct kp_analysis_config {
    int radial_bins;            /* 1..KP_MAX_ANALYSIS_RADIAL_BINS (16) */
    double radial_min;          /* inner edge of the logarithmic bins (2 M) */
    double radial_max;          /* outer edge (100 M) */
    double formation_fraction;  /* central fraction of the formation quantiles, in (0, 1) (0.9) */
} kp_analysis_config;

void kp_default_analysis_config(kp_analysis_config* cfg);

/* Per-pixel analysis arrays, the analysis fields of ImageHostData
 * (src/image/result.hpp:35-92): scalars hold npix values; the radial_*
 * arrays hold radial_bins * npix values, bin-major.  Host or device memory
 * as kp_run_options::outputs_on_device says; none may be NULL. */
typedef struct kp_analysis_out {
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
    double* radial_stokes_i_contribution;
    double* radial_stokes_q_contribution;
    double* radial_stokes_u_contribution;
    double* radial_stokes_v_contribution;
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
} kp_analysis_out;

/*
 * One analysis-mode RIAF image at model->freq_cgs.  Replaces the per-pixel
 * body of the reference's analysis image driver
 * (trace_pass_b_segment_model_analysis_pixel_metric,
 * src/image/analysis_driver.hpp:623-636, called per pixel by its analysis
 * image kernels).  `out` takes the image and diagnostics (nfreq = 1) as for
 * kp_image_riaf; `analysis` the arrays above.  FP64 only
 * (options->precision must be KP_PRECISION_FP64; the schedule is ignored:
 * one thread per pixel), step-doubling RK4 only, min_step > 0.
 */
int kp_image_riaf_analysis(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                           const kp_analysis_config* config, const kp_run_options* options, kp_image_out* out,
                           kp_analysis_out* analysis);

/*
 * Source-partition response channels of analysis mode (ResponseConfig,
 * src/diagnostics/response_config.hpp:10-33; the accumulation of
 * src/diagnostics/response.hpp).  `partition` tags every radiating sample
 * with a source bin.  Each bin has a channel: the Stokes vector its own
 * emission contributes at the camera.  With a response `parameter`, four
 * derivative channels per bin follow (dS/dq through the emission,
 * absorption, Faraday-rotation and Faraday-conversion coefficients of the
 * samples in the bin: mechanism m, bin k is channel bins + m * bins + k),
 * then four full-transfer reruns with the whole plasma at q = +h, -h,
 * +h/2, -h/2 (channels 5 * bins + 0..3).  q is the logarithmic scale of the
 * density (n_e, with B as sqrt(n_e)), the electron temperature, the
 * magnetic field, or of every coefficient at once.
 *
 * Bins per partition, which the entry point checks: radial: `bins` bins
 * between edges[0..bins] (edge_count = bins + 1, increasing), a sample
 * below edges[1] in bin 0 and one at or above edges[bins - 1] in the last;
 * region: 6 (funnel, disk, equatorial band by polar angle from the nearer
 * spin axis, each split into the observer's near and far side); near_far:
 * 2; plasma_region: 4 (sigma above its boundary, beta below its boundary,
 * the rest, and samples without a magnetisation, always the last bin for
 * the RIAF plasma); thetae / sigma / beta / ne_cgs / b_cgs: edge_count
 * increasing positive edges and bins = edge_count + 2 (below the first
 * edge, between edges, above the last, then unavailable).
 */
#define KP_MAX_PARTITION_EDGES 61

typedef enum kp_response_parameter {
    KP_RESPONSE_NONE = 0,
    KP_RESPONSE_DENSITY_SCALE = 1,
    KP_RESPONSE_TEMPERATURE_SCALE = 2,
    KP_RESPONSE_MAGNETIC_SCALE = 3,
    KP_RESPONSE_COEFFICIENTS = 4
} kp_response_parameter;

typedef enum kp_source_partition {
    KP_PARTITION_NONE = 0,
    KP_PARTITION_RADIAL = 1,
    KP_PARTITION_REGION = 2,
    KP_PARTITION_PLASMA_REGION = 3,
    KP_PARTITION_NEAR_FAR = 4,
    KP_PARTITION_THETAE = 5,
    KP_PARTITION_SIGMA = 6,
    KP_PARTITION_BETA = 7,
    KP_PARTITION_NE_CGS = 8,
    KP_PARTITION_B_CGS = 9
} kp_source_partition;

typedef struct kp_response_config {
    int parameter;            /* kp_response_parameter */
    int partition;            /* kp_source_partition; NONE with a parameter is refused */
    double step;              /* h, in [1e-6, 0.1] when a parameter is set (1e-3) */
    int bins;
    int edge_count;
    double edges[KP_MAX_PARTITION_EDGES];
    double funnel_angle;      /* region: radians from either spin axis (20 deg) */
    double disk_angle;        /* region: radians from either spin axis (60 deg) */
    double sigma_boundary;    /* plasma_region (1) */
    double beta_boundary;     /* plasma_region (1) */
    double observer_theta;    /* region / near_far: the observer's direction, radians */
    double observer_phi;
} kp_response_config;

/* The struct's default member initialisers (no partition, no parameter). */
void kp_default_response_config(kp_response_config* config);

/* Channels of a configuration: bins * (parameter ? 5 : 1) + (parameter ? 4 : 0),
 * 0 without a partition; negative (and kp_last_error) when the configuration
 * is invalid. */
int kp_response_channels(const kp_response_config* config);

/*
 * kp_image_riaf_analysis with source-partition response channels.
 * `response` takes 4 * channels * npix doubles, channel-major, then I, Q, U,
 * V, then pixel: response[(4 * channel + s) * npix + pixel]; each channel in
 * the observer basis, like the image.  Host or device memory as
 * options->outputs_on_device says; NULL only when channels is 0.
 */
int kp_image_riaf_analysis_response(const kp_pass_a_params* params, const kp_riaf_model* model,
                                    int radiation_substeps, const kp_analysis_config* config,
                                    const kp_response_config* response_config, const kp_run_options* options,
                                    kp_image_out* out, kp_analysis_out* analysis, double* response);

/* One image of a batch: the arguments of one kp_image_riaf call. */
typedef struct kp_riaf_job {
    kp_pass_a_params params;
    kp_riaf_model model;
    double frequencies[KP_MAX_FREQUENCIES];
    int nfreq;
    int radiation_substeps;
    kp_image_out out;
} kp_riaf_job;

/* Per-call counters of kp_batch_riaf (reference ImageBatchTiming,
 * src/image/batch_driver.hpp:34-40, plus launch facts). */
typedef struct kp_batch_stats {
    double kernel_seconds;       /* device time of the launch (CUDA events) */
    double copy_seconds;         /* device-to-host copies (host outputs only) */
    long long rays;              /* pixels traced */
    int launches;                /* kernels launched */
    int blocks;                  /* CTAs of a near-phase launch */
    int threads_per_block;
    size_t device_output_bytes;  /* library-owned output scratch used */
    /* Device time per engine phase (0 far, 1 near-A, 2 near-B), summed over
     * the phase's launches: CUDA events recorded around every launch on the
     * launching stream. */
    double phase_seconds[3];
    int phase_launches[3];
} kp_batch_stats;

/*
 * A batch of RIAF images traced by the wavefront engine: persistent far and
 * near kernels whose lanes drain ray queues spanning every image (continuous
 * refill), so images of any size, spin, inclination and frequency count
 * share the GPU.  The far kernel moves rays between the camera and the
 * radiating sphere (transport only), the near kernel traces the sphere
 * (surface crossings, radiative transfer); rays migrate between them through
 * HBM ray records.  Replaces the reference's experimental host batching
 * run_image_batch_metric (src/image/batch_driver.hpp:127-187), which launches
 * one kernel per image on a few streams.  Every job is validated before
 * anything is launched; an invalid job fails the whole call (KP_ERR_INVALID /
 * KP_ERR_UNSUPPORTED).  With KP_PRECISION_FP64 each image is bit-identical
 * to the same image traced alone by kp_image_riaf; KP_PRECISION_MIXED images
 * agree with them within the mixed-precision tolerance and are also
 * independent of the batch composition.  The call returns when the images
 * are complete (on options->stream when one is given).  `stats` may be NULL.
 */
int kp_batch_riaf(const kp_riaf_job* jobs, int njobs, const kp_run_options* options,
                  kp_batch_stats* stats);

/*
 * GRMHD snapshots (config: a grid of primitives in FMKS coordinates).
 *
 * kp_grmhd_model holds the scalars of GRMHDGridRadiationModel
 * (src/model/grmhd_grid.hpp:52-97) this path uses; the grid itself is
 * uploaded once with kp_grid_upload (primitives as FP32
 * [8][n1][n2][n3]: rho, u, U1, U2, U3, B1, B2, B3 in code units) and stays
 * resident until kp_grid_release; on the device it is stored cell-major
 * (8 floats per cell, 16-byte aligned) so each trilinear corner is two
 * vector loads.  With has_derived_scalars the derived
 * scalars (n_e, Theta_e, B, sigma, beta per cell; the loaders'
 * precompute_derived_scalars, src/grmhd/kharma_loader.cpp:261-362) are
 * computed on the device at upload.  Thermal fits only (emission_type
 * KP_FIT_PANDYA or KP_FIT_DEXTER); the reference's kappa and power-law
 * distributions are not built.
 */
typedef struct kp_grmhd_model {
    int n1, n2, n3;
    double spin, gam;
    double startx1, startx2, startx3, dx1, dx2, dx3;
    double r_in, r_out;
    double hslope, mks_smooth, poly_alpha, poly_xt, poly_norm;
    double freq_cgs, mbh_solar, M_unit;
    double trat_small, trat_large, beta_crit, sigma_cut, sigma_cut_high, ne_factor;
    int emission_type;
    double emission_scale, absorption_scale, faraday_scale, max_pol_frac;
    int has_derived_scalars;
} kp_grmhd_model;

typedef struct kp_grid kp_grid;

/* The struct's default member initialisers (grmhd_grid.hpp:52-97). */
void kp_default_grmhd_model(kp_grmhd_model* m);
int kp_grid_upload(const kp_grmhd_model* model, const float* prims, int device, kp_grid** out);
/* Host copy of the derived scalars, [5][n1][n2][n3] FP64 (KP_ERR_INVALID if
 * the grid has none). */
int kp_grid_derived(const kp_grid* grid, double* out);
int kp_grid_release(kp_grid* grid);

/*
 * iharm GRMHD dumps (HDF5 files written by the HDF5 library: header
 * datasets, /header/geom/{fmks,mmks}, /prims [n1][n2][n3][>=8]).
 * kp_iharm_options holds the fields of IHARMLoadOptions
 * (src/grmhd/iharm_loader.hpp:10-44) this path uses; the defaults are the
 * reference's.  kp_iharm_read replaces the reading half of
 * load_iharm_model_from_hdf5 (src/grmhd/iharm_loader.cpp:254-370): it fills
 * `model` from the header and the options, applies the reference's checks
 * with its messages, and with `prims` non-NULL writes the first eight
 * primitives as FP32 [8][n1][n2][n3] (capacity in floats; KP_ERR_INVALID if
 * short).  With `prims` NULL only the header is read (no device needed).
 * kp_grid_load_iharm is kp_iharm_read followed by kp_grid_upload (the
 * derived-scalar precompute of :402-520 runs on the device at upload).
 * kp_iharm_dump_time replaces read_iharm_dump_time (:240-252).  File and
 * format errors return KP_ERR_IO.
 */
typedef struct kp_iharm_options {
    double freq_cgs, M_unit, mbh_solar;
    double trat_small, trat_large, beta_crit, sigma_cut, sigma_cut_high;
    int emission_type;
    int interpolate_derived_scalars;
} kp_iharm_options;

void kp_default_iharm_options(kp_iharm_options* o);
int kp_iharm_read(const char* path, const kp_iharm_options* options, kp_grmhd_model* model, float* prims,
                  size_t capacity);
int kp_grid_load_iharm(const char* path, const kp_iharm_options* options, int device, kp_grmhd_model* model,
                       kp_grid** out);
int kp_iharm_dump_time(const char* path, double* t);

/*
 * KHARMA GRMHD dumps (Parthenon .phdf: /Info NumMeshBlocks and
 * MeshBlockSize, the run's parameter text in /Input File, Blocks/loc.lx123,
 * prims.rho / prims.u [nblocks][nx3][nx2][nx1], prims.uvec / prims.B
 * [nblocks][3][nx3][nx2][nx1]).  Replace read_kharma_staged_dump +
 * materialize_kharma_model_from_staged and read_kharma_dump_time
 * (src/grmhd/kharma_loader.cpp:556-823, 1066-1139, 726-749): the geometry
 * from the parameter text (fmks and mmks transforms), the meshblocks
 * assembled into the global grid, B negated with reverse_field; the
 * options are KHARMALoadOptions' fields of kp_iharm_options (same defaults).
 * The reference's checks and messages; file and format errors are KP_ERR_IO.
 */
int kp_kharma_read(const char* path, const kp_iharm_options* options, int reverse_field, kp_grmhd_model* model,
                   float* prims, size_t capacity);
int kp_grid_load_kharma(const char* path, const kp_iharm_options* options, int reverse_field, int device,
                        kp_grmhd_model* model, kp_grid** out);
int kp_kharma_dump_time(const char* path, double* t);

/*
 * One GRMHD image in FMKS coordinates, 1..KP_MAX_FREQUENCIES frequencies on
 * one geodesic, through the wavefront engine (options->precision FP64, or
 * MIXED: FP64 geodesic and grid sample, FP32 fits and transfer).  Replaces
 * run_grmhd_image (src/image/grmhd.hpp:12-32, src/image/grmhd.cpp:22-59) for
 * the FMKS backend; params->coordinate_system must be KP_COORD_FMKS and the
 * grid's spin must be params->spin.
 */
int kp_image_grmhd(const kp_pass_a_params* params, const kp_grid* grid, int radiation_substeps,
                   const double* frequencies, int nfreq, const kp_run_options* options, kp_image_out* out);

/* kp_image_grmhd with a separate step-control frequency list, as
 * kp_image_riaf_step_control (the GRMHD backends' multi-frequency images,
 * src/image/grmhd.cpp:131-170, with step_control_frequencies). */
int kp_image_grmhd_step_control(const kp_pass_a_params* params, const kp_grid* grid, int radiation_substeps,
                                const double* frequencies, int nfreq, const double* control_frequencies,
                                int ncontrol, const kp_run_options* options, kp_image_out* out);

/*
 * One slow-light GRMHD image: nsnap >= 2 resident snapshots of one flow
 * (uploaded grids sharing one grid shape and coordinate map, times strictly
 * increasing); a coefficient sample at coordinate time x^0 reads the fluid at
 * observation_time + x^0, linearly interpolated between the two snapshots
 * that enclose it (primitives and derived scalars after the spatial gather).
 * A radiating sample whose time lies outside [times[0], times[nsnap-1]] ends
 * its ray with KP_REASON_SLOW_LIGHT_TIME_EXHAUSTED.  Replaces
 * run_slow_light_batch_metric in its default decoupled step mode
 * (src/image/slow_light_batch_driver.hpp:107-368, window kernel
 * src/image/slow_light_driver.hpp:1084-1483, finalisation :1560-1760) with
 * every snapshot resident at once; the geodesics are the fast-light ones.
 */
int kp_image_grmhd_slow_light(const kp_pass_a_params* params, const kp_grid* const* snapshots, const double* times,
                              int nsnap, double observation_time, int radiation_substeps, const double* frequencies,
                              int nfreq, const kp_run_options* options, kp_image_out* out);

/*
 * Serving loop.  A server owns one GPU and a device-owner thread that runs
 * the wavefront engine in bounded ticks: each tick admits waiting jobs whose
 * HBM footprint fits (ray records + device outputs), seeds their rays, and
 * runs one (far, near-A, near-B) cycle in which every lane advances at most
 * `tick_budget` RK jobs before parking its ray.  Jobs that arrive while
 * others are on the GPU join the next tick, so their work shares launches
 * with the jobs in flight (continuous batching); a ray resumes from its
 * record with exactly the arithmetic it would have had, so a job's result is
 * the same alone and in any mix.  Results are copied into the job's host
 * buffers (kp_riaf_job.out) when its last ray finishes.  No counterpart in
 * the reference (closest: run_image_batch_metric, src/image/batch_driver.hpp:127-187).
 */
typedef struct kp_server kp_server;

typedef struct kp_server_config {
    int device;
    int precision;           /* kp_precision */
    int integrator;          /* kp_integrator */
    long long max_rays;      /* ray records resident at once (472 B of HBM each) */
    size_t output_bytes;     /* device output arena (kp_image_output_bytes per job) */
    int max_jobs;            /* jobs in flight at once */
    int tick_budget;         /* RK jobs per lane per launch */
} kp_server_config;

/* Job states reported by kp_server_poll. */
typedef enum kp_job_state {
    KP_JOB_PENDING = 0,      /* waiting for admission */
    KP_JOB_RUNNING = 1,      /* rays on the device */
    KP_JOB_DONE = 2,         /* outputs written to the job's buffers */
    KP_JOB_CANCELLED = 3,
    KP_JOB_FAILED = 4
} kp_job_state;

typedef struct kp_server_stats {
    long long submitted, completed, cancelled, failed;
    long long ticks;
    long long max_inflight_rays;  /* peak ray records in use */
    int max_inflight_jobs;
    double wall_seconds;          /* since the server was created */
    double busy_seconds;          /* ticks with work on the device */
    double latency_p50, latency_p99, latency_max;  /* submit -> done, seconds */
    double queue_p50;             /* submit -> admission, seconds */
} kp_server_stats;

/* Defaults: device 0, mixed precision, step-doubling RK4, 4 Mi rays
 * (2 GB of records), 1 GiB of outputs, 64 jobs, budget 128. */
void kp_default_server_config(kp_server_config* cfg);
int kp_server_create(const kp_server_config* cfg, kp_server** out);
/* Validates the job (as kp_batch_riaf does) and queues it; *ticket names it.
 * A job whose footprint exceeds the whole server fails with KP_ERR_INVALID.
 * The job's host output buffers must stay valid until it is done, cancelled
 * or failed. */
int kp_server_submit(kp_server* s, const kp_riaf_job* job, unsigned long long* ticket);

/* A GRMHD image job for the serving loop: the FMKS image of a resident grid
 * (as kp_image_grmhd).  The grid must live on the server's device; a
 * kp_grid_release while jobs still use the grid takes effect when the last
 * of them ends. */
typedef struct kp_grmhd_job {
    kp_pass_a_params params;
    const kp_grid* grid;
    double frequencies[KP_MAX_FREQUENCIES];
    int nfreq;
    int radiation_substeps;
    kp_image_out out;
} kp_grmhd_job;

int kp_server_submit_grmhd(kp_server* s, const kp_grmhd_job* job, unsigned long long* ticket);
int kp_server_poll(kp_server* s, unsigned long long ticket, int* state);
/* Waits until the job is done, cancelled or failed, or `timeout_seconds`
 * pass (KP_ERR_TIMEOUT).  Returns the job's failure status if it failed. */
int kp_server_wait(kp_server* s, unsigned long long ticket, double timeout_seconds);
/* A pending job is dropped at once; a running job finishes on the device and
 * its outputs are not written. */
int kp_server_cancel(kp_server* s, unsigned long long ticket);
int kp_server_get_stats(kp_server* s, kp_server_stats* out);
/* Stops after the tick that is running: pending jobs and jobs still in
 * flight end as cancelled (their outputs are not written), then the
 * server's device memory is released. */
int kp_server_destroy(kp_server* s);

/*
 * Output packing of one frequency (host arrays), in the convention of the
 * reference's image tool: pack_transport_frequency_image
 * (tools/kpolaris_model_image.cpp:2561-2800) with output_qu_sign
 * (tools/kpolaris_evpa.hpp:15-17).  Pixels whose ray did not reach the
 * camera are zero; Q and U change sign for the N EVPA convention
 * (evpa_north = 1), not for W; S_nu = S_inv * frequency^3; total_steps =
 * pass_a_steps + steps.  Any output array may be NULL.  The sums run over
 * returned pixels in pixel order; flux_jy = sum * frequency^3 *
 * intensity_to_flux_jy_per_pixel (flux_density_jy, :589-595), NaN when that
 * scale is not positive.
 */
typedef struct kp_packed_image {
    double* i_inv;
    double* q_inv;
    double* u_inv;
    double* v_inv;
    double* i_nu;
    double* q_nu;
    double* u_nu;
    double* v_nu;
    int32_t* total_steps;
    int returned;        /* out: pixels whose ray reached the camera */
    double sum_inv[4];   /* out: sums of I, Q, U, V (invariant, output convention) */
    double flux_jy[4];   /* out: the sums as flux densities in Jy */
} kp_packed_image;

int kp_pack_image(const kp_image_out* data, int freq_index, double frequency, int evpa_north,
                  double intensity_to_flux_jy_per_pixel, kp_packed_image* out);

/* Pixel solid angle / 1 Jy (compute_flux_scale, tools/kpolaris_model_image.cpp:
 * 551-587): image widths in M, source distance in pc; NaN unless every input
 * is positive. */
double kp_flux_scale_jy_per_pixel(double mbh_solar, double dsource_pc, double image_width_x, double image_width_y,
                                  int nx, int ny);

/*
 * Schedule autotuner for the persistent engine (no counterpart in the
 * reference, whose launch shape is Kokkos's).  Times candidate schedules --
 * CTAs per SM of each phase kernel and the number of cycles captured per
 * graph launch -- on `jobs`, a representative sample of the caller's
 * workload (e.g. its images at reduced resolution), with the precision of
 * `options`, and stores the fastest in the device's tuning table: later
 * persistent and graph launches of that precision with blocks_per_sm == 0
 * use it.  A candidate is adopted only when it beats the default eager
 * schedule (KP_SCHEDULE_PERSISTENT, occupancy-derived CTAs) by at least 2%
 * on the sample; otherwise the table keeps the defaults, blocks_per_sm and
 * graph_cycles come back 0, and the caller should keep the eager schedule.
 * The sample's outputs are written like kp_batch_riaf's.  Schedule choices
 * never change results (rays resume bit-exactly from their records).
 */
typedef struct kp_tuning {
    int blocks_per_sm[3];     /* far, near-A, near-B */
    int graph_cycles;         /* (far, near-A, near-B) cycles per graph launch; 0: keep the eager schedule */
    double seconds;           /* device time of the sample with the chosen schedule */
    double default_seconds;   /* device time of the sample with the default schedule */
    int candidates;           /* schedules timed */
} kp_tuning;

int kp_autotune_batch(const kp_riaf_job* jobs, int njobs, const kp_run_options* options, kp_tuning* out);

/* Limits of kp_batch_riaf_noalloc's static device scratch. */
#define KP_NOALLOC_MAX_RAYS 65536
#define KP_NOALLOC_MAX_JOBS 16

/*
 * kp_batch_riaf for callers that must not allocate: the same wavefront
 * engine and results (bit-identical to kp_batch_riaf with the same options),
 * but every piece of device scratch lives in one static device array of the
 * library (32 MB per device), so the call makes no cudaMalloc/cudaFree and
 * no host allocation.  For callers that run under a fixed device-memory
 * budget, and for callers that cannot afford cudaFree's device-wide
 * synchronisation while other streams are busy (a serving loop, a
 * latency-sensitive pipeline).  Limits: at most KP_NOALLOC_MAX_RAYS pixels
 * summed over the jobs (one 256x256 image) and KP_NOALLOC_MAX_JOBS jobs;
 * larger batches fail with KP_ERR_INVALID before anything runs.  Like
 * kp_batch_riaf, a batch whose rays still move between the phase kernels
 * after 24 launch cycles of (far, near-A, near-B) ends with KP_ERR_TIMEOUT
 * (a 256x256 image takes 2 to 4).  Outputs
 * must be device arrays (options->outputs_on_device = 1); options->stream
 * (NULL: the legacy default stream) carries the work, and the call returns
 * when the images are complete.  The scratch is shared: calls on the same
 * device that overlap in time (from several host threads) race and must be
 * serialised by the caller.  The first call on a device looks the scratch up
 * (cudaGetSymbolAddress) and must not happen inside a stream capture.
 * No counterpart in the reference.
 */
int kp_batch_riaf_noalloc(const kp_riaf_job* jobs, int njobs, const kp_run_options* options);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* KPOLARIS_B200_H */
