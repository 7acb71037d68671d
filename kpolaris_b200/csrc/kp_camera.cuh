// kp_camera.cuh -- pinhole camera at BL/KS phi = 0 in Cartesian Kerr-Schild
// coordinates: ipole-style observer tetrad by Gram-Schmidt, per-pixel
// wavevector and transported screen basis.
//
// Restates src/camera/camera.hpp:97-106 (pixel offsets), :137-149 (normal
// observer), :240-273 (raise, project, normalise), :275-309 (orientation),
// :321-365 (CKS position and native trial vectors), :383-401 (centering
// covector), :415-453 (tetrad) and :485-513 (ray).  sin/cos of the
// inclination arrive precomputed from the host.
#pragma once

#include "kp_geometry.cuh"

namespace kp {

KP_HD void pixel_offsets(int pixel, const ImageConsts& c, double& sx, double& sy) {
    const int i = pixel % c.nx;
    const int j = pixel / c.nx;
    const double x_extent = c.xspan > 0.0 ? 2.0 * c.xspan : c.fov;
    const double y_extent = c.yspan > 0.0 ? 2.0 * c.yspan
                          : (c.xspan > 0.0 ? 2.0 * c.xspan * double(c.ny) / double(c.nx)
                             : (c.fov_y > 0.0 ? c.fov_y : c.fov));
    sx = ((double(i) + 0.5) / double(c.nx) - 0.5) * x_extent + c.x_offset;
    sy = ((double(j) + 0.5) / double(c.ny) - 0.5) * y_extent + c.y_offset;
}

KP_HD D4 project_out(const KSMetricPoint& w, D4 a, const D4& b) {
    const double b2 = ks_dot_at(w, b, b);
    if (abs_val(b2) > kTiny) a = d4_sub_scaled(a, b, ks_dot_at(w, a, b) / b2);
    return a;
}

KP_HD D4 normalize_basis_vector(const KSMetricPoint& w, const D4& v) {
    const double n2 = ks_dot_at(w, v, v);
    const double n = sqrt(max_val(abs_val(n2), kTiny));
    return d4_scale(v, 1.0 / n);
}

// Sum over the 24 permutations of eps_ijkl e0^i e1^j e2^k e3^l in the
// reference's loop order; the skipped terms are exact zeros.
KP_HD double tetrad_orientation(const D4& e0, const D4& e1, const D4& e2, const D4& e3) {
    double out = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            if (j == i) continue;
            for (int k = 0; k < 4; ++k) {
                if (k == i || k == j) continue;
                const int l = 6 - i - j - k;
                int a[4] = {i, j, k, l};
                int sign = 1;
                for (int m = 0; m < 4; ++m)
                    for (int n = m + 1; n < 4; ++n)
                        if (a[m] > a[n]) sign = -sign;
                out += double(sign) * e0.v[i] * e1.v[j] * e2.v[k] * e3.v[l];
            }
        }
    return out;
}

KP_HD D4 native_vector_phi0_cks(double spin, double v0, double vx1, double vx2, double vphi,
                                double radius, double si, double ci) {
    const double vr = radius * vx1;
    const double vth = kPi * vx2;
    return d4(v0, vr * si + vth * radius * ci - vphi * spin * si,
              vth * spin * ci + vphi * radius * si, vr * ci - vth * radius * si);
}

// Camera position, tetrad e0..e3 (position-only, identical for every pixel).

KP_HD CameraFrame camera_frame(const ImageConsts& c) {
    const double mass = c.mass, spin = c.spin;
    const double si = c.sin_inc, ci = c.cos_inc;
    CameraFrame f;
    f.x = d4(0.0, c.cam_radius * si, spin * si, c.cam_radius * ci);
    const KSMetricPoint w = ks_point(mass, spin, f.x);
    // normal observer: u^mu = -g^{mu 0}
    D4 e0;
    for (int mu = 0; mu < 4; ++mu) e0.v[mu] = -ks_gcon_entry(w, mu, 0);
    {
        const double n2 = ks_dot_at(w, e0, e0);
        if (n2 < 0.0) e0 = d4_scale(e0, 1.0 / sqrt(-n2));
    }
    // centering covector (1, d log r / dx^i)
    D4 cc;
    {
        const double xx = f.x.v[1], yy = f.x.v[2], zz = f.x.v[3];
        const double a2 = spin * spin;
        const double radius2 = xx * xx + yy * yy + zz * zz;
        const double s = radius2 - a2;
        const double disc = sqrt(max_val(s * s + 4.0 * a2 * zz * zz, kTiny));
        const double r2 = max_val(0.5 * (s + disc), kTiny);
        const double inv_2r2 = 0.5 / r2;
        cc = d4(1.0, xx * (1.0 + s / disc) * inv_2r2, yy * (1.0 + s / disc) * inv_2r2,
                zz * (1.0 + (s + 2.0 * a2) / disc) * inv_2r2);
    }
    D4 e3;
    for (int mu = 0; mu < 4; ++mu) {
        double sum = 0.0;
        for (int nu = 0; nu < 4; ++nu) sum += ks_gcon_entry(w, mu, nu) * cc.v[nu];
        e3.v[mu] = sum;
    }
    D4 e2 = native_vector_phi0_cks(spin, 0.0, 0.0, 1.0, 0.0, c.cam_radius, si, ci);
    D4 e1 = native_vector_phi0_cks(spin, 1.0, 1.0, 1.0, 1.0, c.cam_radius, si, ci);
    e0 = normalize_basis_vector(w, e0);
    e3 = project_out(w, e3, e0);
    e3 = project_out(w, e3, e0);
    e3 = normalize_basis_vector(w, e3);
    e2 = project_out(w, e2, e0);
    e2 = project_out(w, e2, e3);
    e2 = project_out(w, e2, e0);
    e2 = project_out(w, e2, e3);
    e2 = normalize_basis_vector(w, e2);
    e1 = project_out(w, e1, e0);
    e1 = project_out(w, e1, e2);
    e1 = project_out(w, e1, e3);
    e1 = project_out(w, e1, e0);
    e1 = project_out(w, e1, e2);
    e1 = project_out(w, e1, e3);
    e1 = normalize_basis_vector(w, e1);
    if (tetrad_orientation(e0, e1, e2, e3) < 0.0) e1 = d4_scale(e1, -1.0);
    f.e0 = e0;
    f.e1 = e1;
    f.e2 = e2;
    f.e3 = e3;
    return f;
}

// initialize_pinhole_camera_ray (camera.hpp:485-513) from a precomputed frame.
static __device__ __noinline__ Ray camera_ray(const ImageConsts& c, const CameraFrame& f, int pixel) {
    const KSMetricPoint w = ks_point(c.mass, c.spin, f.x);
    double sx = 0.0, sy = 0.0;
    pixel_offsets(pixel, c, sx, sy);
    const double spatial_norm = sqrt(1.0 + sx * sx + sy * sy);
    const double kt1 = sx / spatial_norm;
    const double kt2 = sy / spatial_norm;
    const double kt3 = 1.0 / spatial_norm;
    D4 sd;
    for (int mu = 0; mu < 4; ++mu)
        sd.v[mu] = f.e1.v[mu] * kt1 + f.e2.v[mu] * kt2 + f.e3.v[mu] * kt3;
    Ray s;
    s.x = f.x;
    for (int mu = 0; mu < 4; ++mu) s.k.v[mu] = f.e0.v[mu] * 1.0 + sd.v[mu];
    // e1: normalize_spacelike
    D4 e1 = d4_sub_scaled(f.e1, sd, kt1);
    {
        const double n2 = ks_dot_at(w, e1, e1);
        if (!(n2 <= 0.0)) e1 = d4_scale(e1, 1.0 / sqrt(n2));
    }
    D4 e2 = d4_sub_scaled(f.e2, sd, kt2);
    {
        const double denom = ks_dot_at(w, e1, e1);
        if (abs_val(denom) > kTiny) e2 = d4_sub_scaled(e2, e1, ks_dot_at(w, e2, e1) / denom);
        const double n2 = ks_dot_at(w, e2, e2);
        if (!(n2 <= 0.0)) e2 = d4_scale(e2, 1.0 / sqrt(n2));
    }
    s.e1 = e1;
    s.e2 = e2;
    return s;
}

}  // namespace kp
