// Host build of the Boyer-Lindquist RIAF scene's device code (kpolaris_b200/
// csrc/kp_bl.cuh, kp_scene.cuh, kp_radiation.cuh) as a shared library, so the
// CPU tests can compare each piece with the reference's own templates over
// KerrBoyerLindquistMetric: the transport RHS, the camera frame and pinhole
// ray, and the RIAF plasma sample + transfer coefficients at a transport
// state.  Transport states are x[4] k[4] e1[4] e2[4].
#include <cmath>
#include <cstring>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __noinline__
#include "kp_scene.cuh"
#include "kpolaris_b200.h"

namespace {

kp::Ray ray_of(const double* s) {
    kp::Ray r;
    for (int m = 0; m < 4; ++m) {
        r.x.v[m] = s[m];
        r.k.v[m] = s[4 + m];
        r.e1.v[m] = s[8 + m];
        r.e2.v[m] = s[12 + m];
    }
    return r;
}

void put(const kp::Ray& r, double* s) {
    for (int m = 0; m < 4; ++m) {
        s[m] = r.x.v[m];
        s[4 + m] = r.k.v[m];
        s[8 + m] = r.e1.v[m];
        s[12 + m] = r.e2.v[m];
    }
}

// The launch constants the BL camera and plasma read (the library's
// make_consts for these fields).
kp::ImageConsts consts_of(const kp_pass_a_params* p, const kp_riaf_model* m) {
    kp::ImageConsts c;
    std::memset(&c, 0, sizeof(c));
    c.mass = p->mass;
    c.spin = p->spin;
    c.horizon = p->mass + std::sqrt(std::fmax(p->mass * p->mass - p->spin * p->spin, 0.0));
    c.nx = p->camera.nx;
    c.ny = p->camera.ny;
    c.cam_radius = p->camera.radius;
    c.inclination = p->camera.inclination;
    c.fov = p->camera.fov;
    c.fov_y = p->camera.fov_y;
    c.xspan = p->camera.xspan;
    c.yspan = p->camera.yspan;
    c.x_offset = p->camera.x_offset;
    c.y_offset = p->camera.y_offset;
    c.scene = kp::kSceneRiafBL;
    if (m) {
        c.nth0 = m->nth0;
        c.Te0 = m->Te0;
        c.disk_h = m->disk_h;
        c.pow_nth = m->pow_nth;
        c.pow_T = m->pow_T;
        c.ne_unit = m->ne_unit;
        c.r_min = m->r_min;
        c.r_max = m->r_max;
        c.horizon_buffer = m->horizon_buffer;
        c.emission_scale = m->emission_scale;
        c.absorption_scale = m->absorption_scale;
        c.faraday_scale = m->faraday_scale;
        c.max_pol_frac = m->max_pol_frac;
        c.keplerian_factor = m->keplerian_factor;
        c.infall_factor = m->infall_factor;
        c.min_frequency_scale = 1e-6;
        c.min_sin_theta = 1e-4;
        c.min_thetae = 1e-3;
        c.min_radius = 1e-6;
        c.thetae_unit = m->te_unit * 1.380649e-16 / (9.1093837015e-28 * 2.99792458e10 * 2.99792458e10);
        c.fit = m->emission_type == KP_FIT_DEXTER ? 4 : 1;
        const double a = p->spin;
        // isco_radius (riaf.hpp:166-174), as the library resolves it
        const double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
        const double z2 = std::sqrt(3.0 * a * a + z1 * z1);
        const double sign = a < 0.0 ? -1.0 : 1.0;
        c.isco = 3.0 + z2 - sign * std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
    }
    return c;
}

}  // namespace

extern "C" {

void h_bl_rhs(double mass, double spin, const double* s16, double* d16) { put(kp::bl_rhs(mass, spin, ray_of(s16)), d16); }

void h_bl_camera_ray(const kp_pass_a_params* p, int pixel, double* out16) {
    const kp::ImageConsts c = consts_of(p, nullptr);
    kp::CameraFrame f;
    kp::bl_camera_frame(c.mass, c.spin, c.cam_radius, c.inclination, f.x, f.e0, f.e1, f.e2, f.e3);
    put(kp::bl_camera_ray(c, f, pixel), out16);
}

void h_bl_riaf_coefficients(const kp_pass_a_params* p, const kp_riaf_model* m, const double* s16, double freq,
                            double* out11) {
    const kp::ImageConsts c = consts_of(p, m);
    const kp::RiafSample smp = kp::riaf_sample_t<true>(c, ray_of(s16));
    const kp::Coeffs<double> o = kp::riaf_coefficients(c, smp, freq);
    const double v[11] = {o.jI, o.jQ, o.jU, o.jV, o.aI, o.aQ, o.aU, o.aV, o.rQ, o.rU, o.rV};
    std::memcpy(out11, v, sizeof(v));
}

}  // extern "C"
