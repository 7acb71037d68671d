// kp_bl.cuh -- Kerr in Boyer-Lindquist coordinates (t, r, theta, phi): the
// metric, its dot product and the transport right-hand side through the
// specialised connection contraction (KerrBoyerLindquistMetric,
// src/geometry/kerr_boyer_lindquist.hpp:9-191; build_bl_connection_work and
// bl_connection_contract, :222-304; transport_rhs, :306-322).  FP64, the
// reference's operation order inside every sum, so that with --fmad=false the
// only difference from the reference's CPU evaluation is the device's
// sin/cos of theta.
#pragma once

#include "kp_common.cuh"

namespace kp {

// The position-dependent pieces of the metric (KerrBoyerLindquistMetric::
// Work, :18-45).
struct BLWork {
    double r, a, a2, m;
    double sinth, costh, sin2, cos2;
    double sigma, delta;
    double dsigma_dr, dsigma_dth, ddelta_dr, dsin2_dth;
};

KP_HD BLWork bl_work(double mass, double spin, const D4& X) {
    BLWork w;
    w.r = max_val(X.v[1], kTiny);
    const double th = X.v[2];
    w.a = spin;
    w.a2 = spin * spin;
    w.m = mass;
    w.sinth = sin(th);
    w.costh = cos(th);
    w.sin2 = max_val(w.sinth * w.sinth, kTiny);
    w.cos2 = w.costh * w.costh;
    w.sigma = w.r * w.r + w.a2 * w.cos2;
    w.delta = w.r * w.r - 2.0 * w.m * w.r + w.a2;
    w.dsigma_dr = 2.0 * w.r;
    w.dsigma_dth = -2.0 * w.a2 * w.sinth * w.costh;
    w.ddelta_dr = 2.0 * (w.r - w.m);
    w.dsin2_dth = 2.0 * w.sinth * w.costh;
    return w;
}

// The five non-zero covariant components (gcov, :47-71).
struct BLMetricPoint {
    double g00, g03, g11, g22, g33;
};

KP_HD BLMetricPoint bl_point(double mass, double spin, const D4& X) {
    const BLWork w = bl_work(mass, spin, X);
    BLMetricPoint p;
    p.g00 = -(1.0 - 2.0 * w.m * w.r / w.sigma);
    p.g03 = -2.0 * w.m * w.a * w.r * w.sin2 / w.sigma;
    p.g11 = w.sigma / w.delta;
    p.g22 = w.sigma;
    p.g33 = w.sin2 * (w.r * w.r + w.a2 + 2.0 * w.m * w.a2 * w.r * w.sin2 / w.sigma);
    return p;
}

// g(u, v) summed as the reference's dot (:117-127): row-major over (mu, nu),
// each term (g u^mu) v^nu; the zero entries add exact zeros and are skipped.
KP_HD double bl_dot_at(const BLMetricPoint& p, const D4& u, const D4& v) {
    double out = 0.0;
    out += p.g00 * u.v[0] * v.v[0];
    out += p.g03 * u.v[0] * v.v[3];
    out += p.g11 * u.v[1] * v.v[1];
    out += p.g22 * u.v[2] * v.v[2];
    out += p.g03 * u.v[3] * v.v[0];
    out += p.g33 * u.v[3] * v.v[3];
    return out;
}

KP_HD void bl_gcov_matrix(double mass, double spin, const D4& X, double g[4][4]) {
    const BLMetricPoint p = bl_point(mass, spin, X);
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) g[mu][nu] = 0.0;
    g[0][0] = p.g00;
    g[0][3] = g[3][0] = p.g03;
    g[1][1] = p.g11;
    g[2][2] = p.g22;
    g[3][3] = p.g33;
}

// Contravariant components (gcon, :73-99).
KP_HD void bl_gcon_matrix(double mass, double spin, const D4& X, double g[4][4]) {
    const BLWork w = bl_work(mass, spin, X);
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) g[mu][nu] = 0.0;
    const double inv_sigma_delta = 1.0 / (w.sigma * w.delta);
    const double r2pa2 = w.r * w.r + w.a2;
    g[0][0] = -(r2pa2 * r2pa2 - w.a2 * w.delta * w.sin2) * inv_sigma_delta;
    g[0][3] = g[3][0] = -2.0 * w.m * w.a * w.r * inv_sigma_delta;
    g[1][1] = w.delta / w.sigma;
    g[2][2] = 1.0 / w.sigma;
    g[3][3] = (w.delta - w.a2 * w.sin2) / (w.sigma * w.delta * w.sin2);
}

// Metric derivatives d/dr (dr*) and d/dtheta (dt*) of the non-zero entries and
// the inverse metric (BLConnectionWork, :222-272).
struct BLConnWork {
    double dr00, dr03, dr11, dr22, dr33;
    double dt00, dt03, dt11, dt22, dt33;
    double g00, g03, g11, g22, g33;
};

KP_HD BLConnWork bl_conn_work(double mass, double spin, const D4& X) {
    const BLWork w = bl_work(mass, spin, X);
    BLConnWork c;
    const double sig = w.sigma;
    const double sig2 = sig * sig;
    const double del = w.delta;
    const double del2 = del * del;
    const double r = w.r;
    const double m = w.m;
    const double a = w.a;
    const double a2 = w.a2;
    const double s2 = w.sin2;
    const double ds2 = w.dsin2_dth;
    const double sig_r = w.dsigma_dr;
    const double sig_t = w.dsigma_dth;
    const double del_r = w.ddelta_dr;
    c.dr00 = 2.0 * m * (sig - r * sig_r) / sig2;
    c.dt00 = -2.0 * m * r * sig_t / sig2;
    c.dr03 = -2.0 * m * a * s2 * (sig - r * sig_r) / sig2;
    c.dt03 = -2.0 * m * a * r * (ds2 * sig - s2 * sig_t) / sig2;
    c.dr11 = (sig_r * del - sig * del_r) / del2;
    c.dt11 = sig_t / del;
    c.dr22 = sig_r;
    c.dt22 = sig_t;
    const double extra = 2.0 * m * a2 * r * s2 / sig;
    const double aterm = r * r + a2 + extra;
    const double extra_r = 2.0 * m * a2 * s2 * (sig - r * sig_r) / sig2;
    const double extra_t = 2.0 * m * a2 * r * (ds2 * sig - s2 * sig_t) / sig2;
    c.dr33 = s2 * (2.0 * r + extra_r);
    c.dt33 = ds2 * aterm + s2 * extra_t;
    const double inv_sigma_delta = 1.0 / (sig * del);
    const double r2pa2 = r * r + a2;
    c.g00 = -(r2pa2 * r2pa2 - a2 * del * s2) * inv_sigma_delta;
    c.g03 = -2.0 * m * a * r * inv_sigma_delta;
    c.g11 = del / sig;
    c.g22 = 1.0 / sig;
    c.g33 = (del - a2 * s2) / (sig * del * s2);
    return c;
}

// Row `row` of a derivative matrix dotted with v (bl_derivative_row_dot,
// :193-208) and the bilinear form (bl_derivative_bilinear, :210-220).
KP_HD double bl_row_dot(double d00, double d03, double d11, double d22, double d33, int row, const D4& v) {
    if (row == 0) return d00 * v.v[0] + d03 * v.v[3];
    if (row == 1) return d11 * v.v[1];
    if (row == 2) return d22 * v.v[2];
    return d03 * v.v[0] + d33 * v.v[3];
}

KP_HD double bl_bilinear(double d00, double d03, double d11, double d22, double d33, const D4& p, const D4& q) {
    return d00 * p.v[0] * q.v[0] + d03 * (p.v[0] * q.v[3] + p.v[3] * q.v[0]) + d11 * p.v[1] * q.v[1] +
           d22 * p.v[2] * q.v[2] + d33 * p.v[3] * q.v[3];
}

// Gamma^mu_{ab} p^a q^b (bl_connection_contract, :274-295).
KP_HD D4 bl_contract(const BLConnWork& c, const D4& p, const D4& q) {
    double t[4];
    for (int nu = 0; nu < 4; ++nu) {
        t[nu] = p.v[1] * bl_row_dot(c.dr00, c.dr03, c.dr11, c.dr22, c.dr33, nu, q) +
                p.v[2] * bl_row_dot(c.dt00, c.dt03, c.dt11, c.dt22, c.dt33, nu, q) +
                q.v[1] * bl_row_dot(c.dr00, c.dr03, c.dr11, c.dr22, c.dr33, nu, p) +
                q.v[2] * bl_row_dot(c.dt00, c.dt03, c.dt11, c.dt22, c.dt33, nu, p);
    }
    t[1] -= bl_bilinear(c.dr00, c.dr03, c.dr11, c.dr22, c.dr33, p, q);
    t[2] -= bl_bilinear(c.dt00, c.dt03, c.dt11, c.dt22, c.dt33, p, q);
    D4 out;
    out.v[0] = 0.5 * (c.g00 * t[0] + c.g03 * t[3]);
    out.v[1] = 0.5 * c.g11 * t[1];
    out.v[2] = 0.5 * c.g22 * t[2];
    out.v[3] = 0.5 * (c.g03 * t[0] + c.g33 * t[3]);
    return out;
}

// transport_rhs (:306-322): dx = k, dk = -Gamma(k, k), de_i = -Gamma(k, e_i).
KP_HD Ray bl_rhs(double mass, double spin, const Ray& s) {
    Ray d;
    d.x = s.k;
    const BLConnWork c = bl_conn_work(mass, spin, s.x);
    const D4 ck = bl_contract(c, s.k, s.k);
    const D4 ce1 = bl_contract(c, s.k, s.e1);
    const D4 ce2 = bl_contract(c, s.k, s.e2);
    for (int mu = 0; mu < 4; ++mu) {
        d.k.v[mu] = -ck.v[mu];
        d.e1.v[mu] = -ce1.v[mu];
        d.e2.v[mu] = -ce2.v[mu];
    }
    return d;
}

// ---------------------------------------------------------------- camera
// The pinhole camera of a Boyer-Lindquist image: position (0, r_cam, i, 0)
// and the ipole tetrad built in native ingoing-MKS trial vectors mapped to BL
// (camera_position_phi0, native_vector_phi0_to_metric,
// ipole_centering_covector, ipole_camera_observer_velocity and
// make_ipole_camera_tetrad, src/camera/camera.hpp:303-453).  Evaluated on the
// host, like the other scenes' frames.

// g(u, v) of the reference's BL dot at X (every call rebuilds the metric).
KP_HD double bl_dot(double mass, double spin, const D4& X, const D4& u, const D4& v) {
    return bl_dot_at(bl_point(mass, spin, X), u, v);
}

KP_HD D4 bl_raise(double mass, double spin, const D4& X, const D4& cov) {
    double g[4][4];
    bl_gcon_matrix(mass, spin, X, g);
    D4 out;
    for (int mu = 0; mu < 4; ++mu) {
        double sum = 0.0;
        for (int nu = 0; nu < 4; ++nu) sum += g[mu][nu] * cov.v[nu];
        out.v[mu] = sum;
    }
    return out;
}

KP_HD D4 bl_project_out(double mass, double spin, const D4& X, D4 a, const D4& b) {
    const double b2 = bl_dot(mass, spin, X, b, b);
    if (abs_val(b2) > kTiny) {
        const double s = bl_dot(mass, spin, X, a, b) / b2;
        for (int i = 0; i < 4; ++i) a.v[i] = a.v[i] - b.v[i] * s;
    }
    return a;
}

KP_HD D4 bl_normalize_basis(double mass, double spin, const D4& X, D4 v) {
    const double n2 = bl_dot(mass, spin, X, v, v);
    const double n = sqrt(max_val(abs_val(n2), kTiny));
    const double inv = 1.0 / n;
    for (int i = 0; i < 4; ++i) v.v[i] = v.v[i] * inv;
    return v;
}

// A native trial vector (v0, vx1, vx2, vphi) at phi = 0 in BL: x1 = log r,
// x2 = theta / pi, KS time and azimuth (dt_KS = dt_BL + 2 M r / Delta dr,
// dphi_KS = dphi_BL + a / Delta dr).
KP_HD D4 bl_native_vector(double mass, double spin, double v0, double vx1, double vx2, double vphi,
                          double radius) {
    const double r = max_val(radius, kTiny);
    const double delta = max_val(r * r - 2.0 * mass * r + spin * spin, kTiny);
    const double vr = r * vx1;
    D4 o;
    o.v[0] = v0 - 2.0 * mass * r * vr / delta;
    o.v[1] = vr;
    o.v[2] = kPi * vx2;
    o.v[3] = vphi - spin * vr / delta;
    return o;
}

// Sum over the 24 permutations of eps_ijkl e0^i e1^j e2^k e3^l (the
// reference's loop order).
KP_HD double bl_tetrad_orientation(const D4& e0, const D4& e1, const D4& e2, const D4& e3) {
    double out = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            if (j == i) continue;
            for (int k = 0; k < 4; ++k) {
                if (k == i || k == j) continue;
                const int l = 6 - i - j - k;
                const int a[4] = {i, j, k, l};
                int sign = 1;
                for (int m = 0; m < 4; ++m)
                    for (int n = m + 1; n < 4; ++n)
                        if (a[m] > a[n]) sign = -sign;
                out += double(sign) * e0.v[i] * e1.v[j] * e2.v[k] * e3.v[l];
            }
        }
    return out;
}

// Camera position and tetrad e0..e3 at (r_cam, inclination).
KP_HD void bl_camera_frame(double mass, double spin, double radius, double inclination, D4& x, D4& e0, D4& e1,
                           D4& e2, D4& e3) {
    x.v[0] = 0.0;
    x.v[1] = radius;
    x.v[2] = inclination;
    x.v[3] = 0.0;
    const double r = max_val(x.v[1], kTiny);
    const double delta = max_val(r * r - 2.0 * mass * r + spin * spin, kTiny);
    // the normal observer of the KS time slicing: -dt_KS raised
    D4 obs;
    obs.v[0] = -1.0;
    obs.v[1] = -2.0 * mass * r / delta;
    obs.v[2] = 0.0;
    obs.v[3] = 0.0;
    e0 = bl_raise(mass, spin, x, obs);
    D4 cc;
    cc.v[0] = 1.0;
    cc.v[1] = 1.0 / r + 2.0 * mass * r / delta;
    cc.v[2] = 0.0;
    cc.v[3] = 0.0;
    e3 = bl_raise(mass, spin, x, cc);
    e2 = bl_native_vector(mass, spin, 0.0, 0.0, 1.0, 0.0, radius);
    e1 = bl_native_vector(mass, spin, 1.0, 1.0, 1.0, 1.0, radius);
    e0 = bl_normalize_basis(mass, spin, x, e0);
    e3 = bl_project_out(mass, spin, x, e3, e0);
    e3 = bl_project_out(mass, spin, x, e3, e0);
    e3 = bl_normalize_basis(mass, spin, x, e3);
    e2 = bl_project_out(mass, spin, x, e2, e0);
    e2 = bl_project_out(mass, spin, x, e2, e3);
    e2 = bl_project_out(mass, spin, x, e2, e0);
    e2 = bl_project_out(mass, spin, x, e2, e3);
    e2 = bl_normalize_basis(mass, spin, x, e2);
    e1 = bl_project_out(mass, spin, x, e1, e0);
    e1 = bl_project_out(mass, spin, x, e1, e2);
    e1 = bl_project_out(mass, spin, x, e1, e3);
    e1 = bl_project_out(mass, spin, x, e1, e0);
    e1 = bl_project_out(mass, spin, x, e1, e2);
    e1 = bl_project_out(mass, spin, x, e1, e3);
    e1 = bl_normalize_basis(mass, spin, x, e1);
    if (bl_tetrad_orientation(e0, e1, e2, e3) < 0.0) {
        for (int i = 0; i < 4; ++i) e1.v[i] = e1.v[i] * -1.0;
    }
}

}  // namespace kp
