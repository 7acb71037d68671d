// kp_grmhd_setup.h -- host-side construction of the constants of a GRMHD
// image: the device view of a grid (GridConsts) with its unit conversions
// resolved, and the per-image ImageConsts for the FMKS metric.  Shared by the
// C ABI (kp_capi.cu) and the host-compiled checks of the GRMHD device code.
//
// Reference: GRMHDGridRadiationModel unit conversions length_unit_cgs /
// rho_unit_cgs / b_unit_cgs / dlambda_scale (src/model/grmhd_grid.hpp:140-161),
// the PassAParams pass controls (src/geodesic/pass_a_core.hpp:10-36).
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "kp_common.cuh"
#include "kpolaris_b200.h"

// A GRMHD snapshot resident on one device.  `users` counts the server jobs
// that read it (queued or running); a released grid is freed when the count
// drops to zero.
struct kp_grid {
    int device = 0;
    kp_grmhd_model model;
    float* prims = nullptr;     // [8][n1][n2][n3]
    double* derived = nullptr;  // [5][n1][n2][n3] or null
    std::atomic<int> users{0};
    std::atomic<bool> released{false};
    std::atomic<bool> freed{false};
};

namespace kp {

inline void grid_ref(kp_grid* g) { g->users.fetch_add(1); }

// Drops `n` users (0: none, just re-checks) and frees the grid once it is
// released and unused (kp_capi.cu).
void grid_unref(kp_grid* g, int n);

inline double grmhd_length_unit_cgs(const kp_grmhd_model& m) {
    const double gnewt = 6.67430e-8, msun = 1.98847e33, cl = 2.99792458e10;
    return gnewt * m.mbh_solar * msun / (cl * cl);
}

// Device view of a grid: prims [8][n1][n2][n3] FP32 and derived scalars
// [5][n1][n2][n3] FP64 (or null) at device addresses.
inline GridConsts grid_consts_of(const kp_grmhd_model& m, const float* prims, const double* derived) {
    GridConsts c;
    std::memset(&c, 0, sizeof(c));
    c.prims = prims;
    c.derived = derived;
    c.n1 = m.n1;
    c.n2 = m.n2;
    c.n3 = m.n3;
    c.has_derived = derived ? 1 : 0;
    c.startx1 = m.startx1;
    c.startx2 = m.startx2;
    c.startx3 = m.startx3;
    c.dx1 = m.dx1;
    c.dx2 = m.dx2;
    c.dx3 = m.dx3;
    c.r_in = m.r_in;
    c.r_out = m.r_out;
    c.gam = m.gam;
    c.map = FmksParams{1.0, m.spin, m.startx1, m.hslope, m.mks_smooth, m.poly_alpha, m.poly_xt, m.poly_norm};
    const double L = grmhd_length_unit_cgs(m);
    const double cl = 2.99792458e10;
    c.rho_unit = m.M_unit / std::max(L * L * L, 1e-300);
    c.b_unit = cl * std::sqrt(4.0 * 3.141592653589793238462643383279502884 * c.rho_unit);
    c.trat_small = m.trat_small;
    c.trat_large = m.trat_large;
    c.beta_crit = m.beta_crit;
    c.sigma_cut = m.sigma_cut;
    c.sigma_cut_high = m.sigma_cut_high;
    c.ne_factor = m.ne_factor;
    return c;
}

// Constants of one GRMHD image: the pass controls with the FMKS metric and
// the grid plasma; freqs null means the model's freq_cgs.
inline ImageConsts image_consts_fmks(const kp_pass_a_params* p, const kp_grmhd_model& m, const GridConsts& grid,
                                     const double* freqs, int nfreq, int integrator) {
    ImageConsts c;
    std::memset(&c, 0, sizeof(c));
    c.mass = p->mass;
    c.spin = p->spin;
    c.horizon = p->mass + std::sqrt(std::max(p->mass * p->mass - p->spin * p->spin, 0.0));
    c.inner_radius = p->inner_radius;
    c.outer_radius = p->outer_radius;
    c.step = p->step;
    c.min_step_abs = std::fabs(p->min_step);
    c.max_step = p->max_step;
    c.tolerance = p->adaptive_tolerance;
    c.max_radiation_step = p->max_radiation_step;
    c.max_radiation_depth = p->max_radiation_depth;
    c.max_absorption_depth = p->max_absorption_depth;
    c.max_faraday_depth = p->max_faraday_depth;
    c.max_steps = p->max_steps;
    c.adaptive = p->adaptive;
    c.integrator = integrator;
    c.faraday_rotation = p->emission_selection.faraday_rotation;
    c.nx = p->camera.nx;
    c.ny = p->camera.ny;
    c.cam_radius = p->camera.radius;
    c.sin_inc = std::sin(p->camera.inclination);
    c.cos_inc = std::cos(p->camera.inclination);
    c.fov = p->camera.fov;
    c.fov_y = p->camera.fov_y;
    c.xspan = p->camera.xspan;
    c.yspan = p->camera.yspan;
    c.x_offset = p->camera.x_offset;
    c.y_offset = p->camera.y_offset;
    c.emission_scale = m.emission_scale;
    c.absorption_scale = m.absorption_scale;
    c.faraday_scale = m.faraday_scale;
    c.max_pol_frac = m.max_pol_frac;
    c.min_sin_theta = 1e-4;  // grmhd_grid.hpp:1149
    c.fit = m.emission_type == KP_FIT_DEXTER ? 4 : 1;
    c.fp32_radius = p->outer_radius + 2.0 * std::max(std::fabs(p->max_step), std::fabs(p->step));
    c.nfreq = nfreq;
    const double length_unit = grmhd_length_unit_cgs(m);
    for (int f = 0; f < nfreq; ++f) {
        const double fr = freqs ? freqs[f] : m.freq_cgs;
        c.freq[f] = fr;
        c.dlambda_scale[f] = length_unit / std::max(fr, 1.0);  // grmhd_grid.hpp:159-161
    }
    c.scene = kSceneGrmhdFmks;
    c.fmks = FmksParams{p->mass, p->spin, p->fmks_startx1, p->fmks_hslope, p->fmks_mks_smooth,
                        p->fmks_poly_alpha, p->fmks_poly_xt, p->fmks_poly_norm};
    c.grid = grid;
    return c;
}

// FP32 emission scales 2^E of a mixed-precision GRMHD image, one per
// frequency.  The invariant emissivity j ~ n_e e^2 nu_c / (c nu^2) lies far
// below FP32 range in CGS; E puts the emission of one radiation step at a
// reference plasma point (code density 1, code field 0.05, shape factor bound
// 30) at 2^-6.  The transfer is linear in the emission, so the image is
// rescaled by 2^-E in FP64 at the end and E changes only rounding.
inline int grmhd_emission_exponent(const kp_pass_a_params* p, const kp_grmhd_model& m, const ImageConsts& c,
                                   double freq, double dls) {
    const double pi = 3.141592653589793, ee = 4.803204712570263e-10, me = 9.1093826e-28, mp = 1.67262171e-24,
                 cl = 2.99792458e10;
    const double ne = std::max(c.grid.rho_unit / (mp + me) * m.ne_factor, 1e-30);
    const double b = 0.05 * c.grid.b_unit;
    const double nu_c = ee * b / (2.0 * pi * me * cl);
    const double j_phys = ne * ee * ee * nu_c / cl * (std::sqrt(2.0) * pi / 27.0) * 30.0;
    const double step = p->max_radiation_step > 0.0 ? p->max_radiation_step : std::max(p->max_step, 1e-3);
    const double j_inv = j_phys / std::max(freq * freq, 1.0);
    const double dl = std::max(step * std::fabs(dls), 1e-300);
    double e = std::floor(std::log2(std::ldexp(1.0, -6) / std::max(j_inv * dl, 1e-300)));
    if (!(e == e)) e = 0.0;
    return int(std::min(120.0, std::max(-120.0, e)));
}

inline void grmhd_emission_scale(const kp_pass_a_params* p, const kp_grmhd_model& m, ImageConsts& c) {
    for (int f = 0; f < c.nfreq; ++f) {
        const int ei = grmhd_emission_exponent(p, m, c, c.freq[f], c.dlambda_scale[f]);
        c.emission_scale_pow2[f] = std::ldexp(1.0f, ei);
        c.inv_emission_scale_pow2[f] = std::ldexp(1.0, -ei);
    }
}

// A separate step-control list of a GRMHD image (the control frequencies,
// their dlambda scales and FP32 emission scales).
inline void grmhd_apply_control(const kp_pass_a_params* p, const kp_grmhd_model& m, ImageConsts& c,
                                const double* ctl, int nctl) {
    const double length_unit = grmhd_length_unit_cgs(m);
    c.nctl = nctl;
    for (int g = 0; g < nctl; ++g) {
        c.ctl_freq[g] = ctl[g];
        c.ctl_dlambda_scale[g] = length_unit / std::max(ctl[g], 1.0);
        c.ctl_emission_scale_pow2[g] = std::ldexp(1.0f, grmhd_emission_exponent(p, m, c, ctl[g], c.ctl_dlambda_scale[g]));
    }
}

}  // namespace kp
