// kp_common.cuh -- shared device types and per-image launch constants for the
// B200 GRRT kernels.  Geometry types are FP64; radiation types are templated
// on the transfer precision R (double for the FP64 path, float for the mixed
// path).
#pragma once

#include <cstdint>

#include "kpolaris_b200.h"

#ifndef KP_HD
#define KP_HD __host__ __device__ __forceinline__
#endif

namespace kp {

constexpr int kMaxFreq = 4;
constexpr int kMaxControl = KP_MAX_CONTROL_FREQUENCIES;
constexpr double kTiny = 1e-300;
constexpr double kLarge = 1e300;
constexpr double kPi = 3.141592653589793238462643383279502884;
// 8 * DBL_EPSILON: adaptive_tolerance_floor (src/common/math.hpp:56-63).
constexpr double kTolFloor = 8.0 * 2.220446049250313080847263336181640625e-16;

enum Reason : int {
    kNone = 0,
    kReachedCamera = 1,
    kReachedInner = 2,
    kEscaped = 3,
    kMaxSteps = 4,
    kInvalidState = 5,
    kSlowLightTimeExhausted = 6,
    kAdaptiveUnderflow = 7,
};

template<class T> KP_HD T abs_val(T x) { return x < T(0) ? -x : x; }
template<class T> KP_HD T min_val(T a, T b) { return a < b ? a : b; }
template<class T> KP_HD T max_val(T a, T b) { return a > b ? a : b; }
template<class T> KP_HD T clamp_val(T x, T lo, T hi) { return min_val(max_val(x, lo), hi); }
template<class T> KP_HD T sq(T x) { return x * x; }

struct D4 {
    double v[4];
};

// Ray state: position x, future-directed wavevector k and the transported
// screen basis e1, e2 (src/geodesic/state.hpp:7-16), 128 bytes.
struct Ray {
    D4 x, k, e1, e2;
};

template<class R>
struct Stokes4 {
    R I, Q, U, V;
};

template<class R>
struct Coeffs {
    R jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV;
};

// FMKS coordinate parameters (PassAParams fmks_*, pass_a_core.hpp:29-34, and
// the grid mapping of GRMHDGridRadiationModel, grmhd_grid.hpp:58-66).
struct FmksParams {
    double mass, spin;
    double startx1, hslope, mks_smooth, poly_alpha, poly_xt, poly_norm;
};

// A GRMHD snapshot resident on the device (GRMHDGridRadiationModel scalars,
// grmhd_grid.hpp:52-97, with the unit conversions resolved on the host).
// Device layout of a grid: cell-major, so the eight corners of a trilinear
// stencil read whole 32-byte cells (primitives) and 48-byte cells (derived
// scalars) with 16-byte vector loads.
constexpr int kPrimStride = 8;  // floats per cell: rho, u, U1..U3, B1..B3
constexpr int kDerStride = 6;   // doubles per cell: n_e, Theta_e, B, sigma, beta, pad

struct GridConsts {
    const float* prims;      // [n1][n2][n3][kPrimStride]
    const double* derived;   // [n1][n2][n3][kDerStride] (or null)
    int n1, n2, n3, has_derived;
    double startx1, startx2, startx3, dx1, dx2, dx3;
    double r_in, r_out, gam;
    FmksParams map;          // theta(x1, x2) of the grid
    double rho_unit, b_unit, trat_small, trat_large, beta_crit, sigma_cut, sigma_cut_high, ne_factor;
};

enum Scene : int { kSceneRiafCks = 0, kSceneGrmhdFmks = 1, kSceneGrmhdFmksSlowLight = 2, kSceneRiafBL = 3 };

// Everything one image needs on the device, resolved on the host.  Host-side
// precomputation keeps libm (sin/cos of the inclination, cbrt in the ISCO
// radius) on the CPU so the device geometry uses only + - * / sqrt and stays
// bit-identical to the reference's CPU arithmetic.
struct ImageConsts {
    // spacetime (Kerr, M = mass)
    double mass, spin;
    double horizon;  // KerrSchildInMetric::horizon_radius
    // integration (PassAParams, src/geodesic/pass_a_core.hpp:10-36)
    double inner_radius, outer_radius, step;
    double min_step_abs, max_step, tolerance;
    double max_radiation_step, max_radiation_depth, max_absorption_depth, max_faraday_depth;
    int max_steps, adaptive, integrator, faraday_rotation;
    // pinhole camera (CameraParams, src/camera/camera.hpp:12-25)
    int nx, ny;
    double cam_radius, sin_inc, cos_inc;
    double inclination;  // the camera's theta in Boyer-Lindquist scenes
    double fov, fov_y, xspan, yspan, x_offset, y_offset;
    // RIAF plasma (src/model/riaf.hpp:19-52)
    double nth0, Te0, disk_h, pow_nth, pow_T, ne_unit;
    double r_min, r_max, horizon_buffer;
    double emission_scale, absorption_scale, faraday_scale, max_pol_frac;
    double keplerian_factor, infall_factor;
    double min_frequency_scale, min_sin_theta, min_thetae, min_radius;
    double thetae_unit;  // te_unit * k_B / (m_e c^2)
    double isco;         // isco_radius(spin), riaf.hpp:166-174
    // boundary of the far phase (FP32 contraction under the mixed policy):
    // outside the radiating sphere by two of the longest steps
    double fp32_radius;
    int fit;             // 1 Pandya, 4 Dexter
    // frequencies sharing one geodesic
    int nfreq;
    double freq[kMaxFreq];
    double dlambda_scale[kMaxFreq];  // length_unit / max(freq, 1)
    // mixed path: per-image power-of-two scale applied to j and S
    float emission_scale_pow2[kMaxFreq];
    double inv_emission_scale_pow2[kMaxFreq];
    // separate step-control frequency list (pass_b.hpp:1505-1895): with
    // nctl > 0 the pass-B substep counts take the largest count over these
    // frequencies instead of over freq[]; nctl == 0 is the fused form
    int nctl;
    double ctl_freq[kMaxControl];
    double ctl_dlambda_scale[kMaxControl];
    float ctl_emission_scale_pow2[kMaxControl];
    // scene: RIAF in Cartesian Kerr-Schild, or a GRMHD grid in FMKS
    int scene;
    FmksParams fmks;
    GridConsts grid;
    // slow light: the resident snapshots of one flow ([nseries] device
    // tables, times increasing) and the observation time; a sample at
    // coordinate time x^0 reads the fluid at t_obs + x^0
    const GridConsts* series;
    const double* series_times;
    int nseries;
    double t_obs;
};

// Device pointers of one image's outputs, laid out like ImageHostData.
struct ImageOutPtrs {
    double* image_i;
    double* image_q;
    double* image_u;
    double* image_v;
    double* closure_x;
    double* closure_k;
    double* final_null;
    double* frame_error;
    double* det_r;
    double* r11;
    double* r12;
    double* r21;
    double* r22;
    double* basis_identity_error;
    double* basis_rotation_angle;
    int32_t* pass_a_steps;
    int32_t* steps;
    int32_t* reason;
};

// Camera position and ipole tetrad e0..e3 at phi = 0 (identical for every
// pixel of an image; evaluated once on the host).
struct CameraFrame {
    D4 x, e0, e1, e2, e3;
};

// One image (job) of a persistent launch.
struct JobDesc {
    ImageConsts c;
    CameraFrame frame;
    ImageOutPtrs out;
    long long ray_begin;  // first global ray index of this job
    int npix;
    int precision;        // kp_precision of this job
};

// Resumable state of one ray between launches (lives in HBM, 464 bytes):
// the ray, the control state and the Stokes channels (32 bytes per frequency
// in either precision).  Rays are parked only at the top of the pass-A or
// pass-B loop, so the crossing search never spans two launches.
struct alignas(16) RayRecord {
    Ray S;
    double st[26];
    double stokes[4 * kMaxFreq];
};

// Phases of the wavefront engine (one kernel each).  Far: rays whose loop
// tops lie beyond ImageConsts::fp32_radius (camera to radiating sphere and
// back: pure transport).  Near-A: pass A inside (surface-crossing search).
// Near-B: pass B inside (radiative transfer).  Rays migrate between the
// phases through id queues.
enum Phase : int { kPhaseFar = 0, kPhaseNearA = 1, kPhaseNearB = 2, kPhases = 3 };

// A newly admitted job of the serving loop: its slot in the job table, the
// first of its contiguous ray ids and its pixel count.
struct SeedEntry {
    int slot;
    int npix;
    long long ray_base;
};

// Device-side launch description (kernel parameter).
struct WaveDesc {
    const JobDesc* jobs;           // device array, ordered by ray_begin
    int njobs;
    RayRecord* pool;               // indexed by global ray id
    // input: fresh rays [fresh_begin, fresh_end) first, then in_ids[0, *in_count)
    long long fresh_begin, fresh_end;
    const unsigned* in_ids;
    const unsigned* in_count;
    unsigned long long* in_head;   // pop counter, zero before the launch
    // queue of the next launch of each phase (this phase's own entry takes
    // the rays parked by the iteration budget)
    unsigned* out_ids[kPhases];
    unsigned* out_count[kPhases];
    int budget;                    // RK jobs per lane per launch; 0 = unlimited
    int* status;                   // device error word (0 ok)
    unsigned* job_done;            // per-job count of finished rays (may be null)
};

}  // namespace kp
