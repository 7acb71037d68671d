// kp_fmks.cuh -- Kerr spacetime in funky modified Kerr-Schild (FMKS) native
// coordinates (t, x1, x2, phi), FP64: the theta(x1, x2) map and its
// derivatives, the native metric, the transport right-hand side through the
// spherical Kerr-Schild connection, and the pinhole camera.
//
// Reference: KerrFMKSMetric and its transport_rhs
// (src/geometry/kerr_fmks.hpp:11-481), the spherical Kerr-Schild connection
// work and fixed-p contraction (src/geometry/kerr_schild_spherical.hpp:192-323),
// the ipole camera tetrad (src/camera/camera.hpp:141-270, 302-456, 485-513).
// The theta map calls exp/sin/cos on every evaluation, so this path agrees
// with the reference's CPU run to libm accuracy, not bit for bit.
#pragma once

#include "kp_camera.cuh"

namespace kp {

KP_HD double fmks_power(double x, double p) {
    const int n = int(p + 0.5);
    if (abs_val(p - double(n)) < 1e-10 && n >= 0) {
        double y = 1.0;
        const double ax = abs_val(x);
        for (int i = 0; i < n; ++i) y *= ax;
        if (x < 0.0 && (n % 2) == 1) y = -y;
        return y;
    }
    return pow(abs_val(x), p);
}

// theta(x1, x2) and its first and second derivatives
// (build_fmks_connection_work, kerr_fmks.hpp:296-348).
struct FmksTheta {
    double r, th, dth1, dth2, d2th11, d2th12, d2th22;
};

KP_HD FmksTheta fmks_theta(const FmksParams& m, double x1, double x2) {
    const double y = 2.0 * x2 - 1.0;
    const double z = y / m.poly_xt;
    const double expfac = exp(m.mks_smooth * (m.startx1 - x1));
    double za, za1, za2;
    if (abs_val(m.poly_alpha - 14.0) < 1e-12) {
        const double z2 = z * z;
        const double z4 = z2 * z2;
        const double z8 = z4 * z4;
        za2 = z8 * z4;
        za1 = za2 * z;
        za = za2 * z2;
    } else {
        za = fmks_power(z, m.poly_alpha);
        za1 = fmks_power(z, m.poly_alpha - 1.0);
        za2 = fmks_power(z, m.poly_alpha - 2.0);
    }
    double s2, c2;
    sincos(2.0 * kPi * x2, &s2, &c2);
    const double thG = kPi * x2 + ((1.0 - m.hslope) / 2.0) * s2;
    const double thJ = m.poly_norm * y * (1.0 + za / (m.poly_alpha + 1.0)) + 0.5 * kPi;
    const double dthG = kPi + (1.0 - m.hslope) * kPi * c2;
    const double dthJ = 2.0 * m.poly_norm * (1.0 + za / (m.poly_alpha + 1.0)) +
                        (2.0 * m.poly_alpha * m.poly_norm * y * za1) / ((m.poly_alpha + 1.0) * m.poly_xt);
    const double d2thG = -2.0 * (1.0 - m.hslope) * kPi * kPi * s2;
    const double d2thJ = 4.0 * m.poly_norm * m.poly_alpha / (m.poly_alpha + 1.0) *
                         (2.0 * za1 / m.poly_xt + y * (m.poly_alpha - 1.0) * za2 / (m.poly_xt * m.poly_xt));
    FmksTheta t;
    t.r = exp(x1);
    t.th = thG + expfac * (thJ - thG);
    t.dth1 = -m.mks_smooth * expfac * (thJ - thG);
    t.dth2 = dthG + expfac * (dthJ - dthG);
    t.d2th11 = -m.mks_smooth * t.dth1;
    t.d2th12 = -m.mks_smooth * expfac * (dthJ - dthG);
    t.d2th22 = d2thG + expfac * (d2thJ - d2thG);
    return t;
}

// theta alone (theta_from_x2, kerr_fmks.hpp:46-53).
KP_HD double fmks_theta_of(const FmksParams& m, double x1, double x2) {
    const double y = 2.0 * x2 - 1.0;
    const double thG = kPi * x2 + ((1.0 - m.hslope) / 2.0) * sin(2.0 * kPi * x2);
    const double thJ = m.poly_norm * y * (1.0 + fmks_power(y / m.poly_xt, m.poly_alpha) / (m.poly_alpha + 1.0)) +
                       0.5 * kPi;
    return thG + exp(m.mks_smooth * (m.startx1 - x1)) * (thJ - thG);
}

// x2 with theta(x1, x2) = theta, by 64 bisections (native_x2_from_theta, :102-112).
KP_HD double fmks_x2_of(const FmksParams& m, double x1, double theta) {
    double lo = 0.0, hi = 1.0;
    for (int it = 0; it < 64; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (fmks_theta_of(m, x1, mid) < theta) lo = mid; else hi = mid;
    }
    return 0.5 * (lo + hi);
}

KP_HD double fmks_radius(const D4& X) { return exp(X.v[1]); }

// Native metric g_{mu nu} at X (the Jacobian transform of the spherical
// Kerr-Schild metric, gcov_matrix :141-169, in closed form).
KP_HD void fmks_gcov(const FmksParams& m, const D4& X, double g[4][4]) {
    const FmksTheta t = fmks_theta(m, X.v[1], X.v[2]);
    double s, c;
    sincos(t.th, &s, &c);
    const double s2 = s * s, a = m.spin, a2 = a * a;
    const double rho2 = t.r * t.r + a2 * c * c;
    const double f = 2.0 * m.mass * t.r / rho2;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g[i][j] = 0.0;
    g[0][0] = -1.0 + f;
    g[0][1] = g[1][0] = f * t.r;
    g[0][3] = g[3][0] = -a * f * s2;
    g[1][1] = (1.0 + f) * t.r * t.r + rho2 * t.dth1 * t.dth1;
    g[1][2] = g[2][1] = rho2 * t.dth1 * t.dth2;
    g[1][3] = g[3][1] = -a * s2 * (1.0 + f) * t.r;
    g[2][2] = rho2 * t.dth2 * t.dth2;
    g[3][3] = s2 * (rho2 + a2 * s2 * (1.0 + f));
}

// Native inverse metric at X: the inverse Jacobian applied to the spherical
// Kerr-Schild inverse metric (native_metric, grmhd_grid.hpp:660-708).
KP_HD void fmks_gcon(const FmksParams& m, const D4& X, double gi[4][4]) {
    const FmksTheta t = fmks_theta(m, X.v[1], X.v[2]);
    double s, c;
    sincos(t.th, &s, &c);
    const double s2 = max_val(s * s, kTiny), a = m.spin, a2 = a * a;
    const double rho2 = t.r * t.r + a2 * c * c;
    const double delta = t.r * t.r - 2.0 * m.mass * t.r + a2;
    const double f = 2.0 * m.mass * t.r / rho2;
    double k[4][4] = {};
    k[0][0] = -(1.0 + f);
    k[0][1] = k[1][0] = f;
    k[1][1] = delta / rho2;
    k[1][3] = k[3][1] = a / rho2;
    k[2][2] = 1.0 / rho2;
    k[3][3] = 1.0 / (rho2 * s2);
    double J[4][4] = {};
    J[0][0] = 1.0;
    J[1][1] = 1.0 / t.r;
    J[2][1] = -t.dth1 / (t.r * t.dth2);
    J[2][2] = 1.0 / t.dth2;
    J[3][3] = 1.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) {
            double sum = 0.0;
            for (int p = 0; p < 4; ++p)
                for (int q = 0; q < 4; ++q) sum += J[mu][p] * J[nu][q] * k[p][q];
            gi[mu][nu] = sum;
        }
}

KP_HD double dot_gm(const double g[4][4], const D4& u, const D4& v) {
    double out = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) out += g[mu][nu] * u.v[mu] * v.v[nu];
    return out;
}

// Spherical Kerr-Schild connection work at (r, theta): g^{mu nu} and the
// r- and theta-derivatives of g_{mu nu} (build_spherical_ks_connection_work,
// kerr_schild_spherical.hpp:198-266).
struct SksConn {
    double gcon[4][4], dgr[4][4], dgth[4][4];
};

KP_HD SksConn sks_conn(double mass, double a, double r, double th) {
    SksConn c;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) c.gcon[i][j] = c.dgr[i][j] = c.dgth[i][j] = 0.0;
    double s, cc;
    sincos(th, &s, &cc);
    const double a2 = a * a, s2 = s * s, safe_s2 = max_val(s2, kTiny);
    const double rho2 = r * r + a2 * cc * cc, rho4 = rho2 * rho2;
    const double f = 2.0 * mass * r / rho2;
    const double delta = r * r - 2.0 * mass * r + a2;
    c.gcon[0][0] = -(1.0 + f);
    c.gcon[0][1] = c.gcon[1][0] = f;
    c.gcon[1][1] = delta / rho2;
    c.gcon[1][3] = c.gcon[3][1] = a / rho2;
    c.gcon[2][2] = 1.0 / rho2;
    c.gcon[3][3] = 1.0 / (rho2 * safe_s2);
    const double drho_dr = 2.0 * r, drho_dth = -2.0 * a2 * s * cc, ds2_dth = 2.0 * s * cc;
    const double df_dr = 2.0 * mass * (rho2 - r * drho_dr) / rho4;
    const double df_dth = -2.0 * mass * r * drho_dth / rho4;
    auto sr = [&](int m, int n, double v) { c.dgr[m][n] = v; c.dgr[n][m] = v; };
    auto st = [&](int m, int n, double v) { c.dgth[m][n] = v; c.dgth[n][m] = v; };
    sr(0, 0, df_dr);
    st(0, 0, df_dth);
    sr(0, 1, df_dr);
    st(0, 1, df_dth);
    sr(0, 3, -a * s2 * df_dr);
    st(0, 3, -a * (s2 * df_dth + ds2_dth * f));
    sr(1, 1, df_dr);
    st(1, 1, df_dth);
    sr(1, 3, -a * s2 * df_dr);
    st(1, 3, -a * (ds2_dth * (1.0 + f) + s2 * df_dth));
    sr(2, 2, drho_dr);
    st(2, 2, drho_dth);
    const double bracket = rho2 + a2 * s2 * (1.0 + f);
    const double dbr = drho_dr + a2 * s2 * df_dr;
    const double dbt = drho_dth + a2 * (ds2_dth * (1.0 + f) + s2 * df_dth);
    sr(3, 3, s2 * dbr);
    st(3, 3, ds2_dth * bracket + s2 * dbt);
    return c;
}

// dx = k, dk = -Gamma(k, k), de_i = -Gamma(k, e_i) in FMKS: vectors go to
// spherical Kerr-Schild components, the spherical connection is contracted
// with p = k fixed, and the second-derivative terms of theta(x1, x2) carry
// the result back (transport_rhs, kerr_fmks.hpp:455-479; fixed-p contraction,
// kerr_schild_spherical.hpp:288-323).
KP_HD Ray fmks_rhs(const FmksParams& m, const Ray& s) {
    const FmksTheta t = fmks_theta(m, s.x.v[1], s.x.v[2]);
    const SksConn c = sks_conn(m.mass, m.spin, t.r, t.th);
    auto to_sph = [&](const D4& v) {
        D4 o;
        o.v[0] = v.v[0];
        o.v[1] = t.r * v.v[1];
        o.v[2] = t.dth1 * v.v[1] + t.dth2 * v.v[2];
        o.v[3] = v.v[3];
        return o;
    };
    const D4 ks = to_sph(s.k);
    double rowk_r[4], rowk_t[4];
    for (int nu = 0; nu < 4; ++nu) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < 4; ++q) {
            a += c.dgr[nu][q] * ks.v[q];
            b += c.dgth[nu][q] * ks.v[q];
        }
        rowk_r[nu] = a;
        rowk_t[nu] = b;
    }
    auto contract = [&](const D4& qn) {
        const D4 q = to_sph(qn);
        double rr[4], rt[4];
        double d1 = 0.0, d2 = 0.0;
        for (int nu = 0; nu < 4; ++nu) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < 4; ++w) {
                a += c.dgr[nu][w] * q.v[w];
                b += c.dgth[nu][w] * q.v[w];
            }
            rr[nu] = a;
            rt[nu] = b;
            d1 += ks.v[nu] * a;
            d2 += ks.v[nu] * b;
        }
        double tt[4];
        for (int nu = 0; nu < 4; ++nu) {
            double term = ks.v[1] * rr[nu] + q.v[1] * rowk_r[nu] + ks.v[2] * rt[nu] + q.v[2] * rowk_t[nu];
            if (nu == 1) term -= d1;
            else if (nu == 2) term -= d2;
            tt[nu] = term;
        }
        double hs[4];
        for (int mu = 0; mu < 4; ++mu) {
            double comp = 0.0;
            for (int nu = 0; nu < 4; ++nu) comp += c.gcon[mu][nu] * tt[nu];
            hs[mu] = 0.5 * comp;
        }
        // back to native components (fmks_from_spherical_connection_contract, :414-431)
        hs[1] += t.r * s.k.v[1] * qn.v[1];
        hs[2] += t.d2th11 * s.k.v[1] * qn.v[1] + t.d2th12 * (s.k.v[1] * qn.v[2] + s.k.v[2] * qn.v[1]) +
                 t.d2th22 * s.k.v[2] * qn.v[2];
        D4 out;
        out.v[0] = -hs[0];
        out.v[1] = -(hs[1] / t.r);
        out.v[2] = -((hs[2] - t.dth1 * hs[1] / t.r) / t.dth2);
        out.v[3] = -hs[3];
        return out;
    };
    Ray d;
    d.x = s.k;
    d.k = contract(s.k);
    d.e1 = contract(s.e1);
    d.e2 = contract(s.e2);
    return d;
}

// The same right-hand side in factored form, for the mixed policy: the
// spherical Kerr-Schild derivatives have only seven distinct nonzero
// entries per direction (d/dr g: rows 0 and 1 coincide, A(q0 + q1) + B q3;
// d/dtheta g likewise with two different (0,3)/(1,3) entries), the inverse
// metric five, and the three divisions by rho^2, r and dtheta/dx2 become
// reciprocals.  Same algebra as fmks_rhs, regrouped: agrees to rounding.
KP_HD Ray fmks_rhs_factored(const FmksParams& m, const Ray& s) {
    const FmksTheta t = fmks_theta(m, s.x.v[1], s.x.v[2]);
    const double a = m.spin, M = m.mass, r = t.r;
    double sn, cs;
    sincos(t.th, &sn, &cs);
    const double a2 = a * a, s2 = sn * sn, safe_s2 = max_val(s2, kTiny);
    const double rho2 = r * r + a2 * cs * cs;
    const double inv_rho2 = 1.0 / rho2;
    const double inv_rho4 = inv_rho2 * inv_rho2;
    const double f = 2.0 * M * r * inv_rho2;
    const double delta = r * r - 2.0 * M * r + a2;
    // inverse metric: g00, g01 = g10, g11, g13 = g31, g22, g33
    const double G00 = -(1.0 + f), G01 = f, G11 = delta * inv_rho2, G13 = a * inv_rho2, G22 = inv_rho2;
    const double G33 = inv_rho2 / safe_s2;
    // d/dr g and d/dtheta g
    const double drho_dth = -2.0 * a2 * sn * cs, ds2_dth = 2.0 * sn * cs;
    const double df_dr = 2.0 * M * (rho2 - 2.0 * r * r) * inv_rho4;
    const double df_dth = -2.0 * M * r * drho_dth * inv_rho4;
    const double A = df_dr, B = -a * s2 * df_dr, C = 2.0 * r;
    const double Dr = s2 * (2.0 * r + a2 * s2 * df_dr);
    const double E = df_dth, F0 = -a * (s2 * df_dth + ds2_dth * f), F1 = -a * (ds2_dth * (1.0 + f) + s2 * df_dth);
    const double Gt = drho_dth;
    const double bracket = rho2 + a2 * s2 * (1.0 + f);
    const double Ht = ds2_dth * bracket + s2 * (drho_dth + a2 * (ds2_dth * (1.0 + f) + s2 * df_dth));
    const double inv_r = 1.0 / r, inv_dth2 = 1.0 / t.dth2;
    struct V {
        double v0, v1, v2, v3;
    };
    auto to_sph = [&](const D4& q) { return V{q.v[0], r * q.v[1], t.dth1 * q.v[1] + t.dth2 * q.v[2], q.v[3]}; };
    auto drow = [&](const V& q, V& rr, V& rt) {
        const double sig = q.v0 + q.v1;
        rr = V{A * sig + B * q.v3, A * sig + B * q.v3, C * q.v2, B * sig + Dr * q.v3};
        rt = V{E * sig + F0 * q.v3, E * sig + F1 * q.v3, Gt * q.v2, F0 * q.v0 + F1 * q.v1 + Ht * q.v3};
    };
    const V ks = to_sph(s.k);
    V rk, tk;
    drow(ks, rk, tk);
    auto contract = [&](const D4& qn) {
        const V q = to_sph(qn);
        V rr, rt;
        drow(q, rr, rt);
        const double d1 = ks.v0 * rr.v0 + ks.v1 * rr.v1 + ks.v2 * rr.v2 + ks.v3 * rr.v3;
        const double d2 = ks.v0 * rt.v0 + ks.v1 * rt.v1 + ks.v2 * rt.v2 + ks.v3 * rt.v3;
        const double t0 = ks.v1 * rr.v0 + q.v1 * rk.v0 + ks.v2 * rt.v0 + q.v2 * tk.v0;
        const double t1 = ks.v1 * rr.v1 + q.v1 * rk.v1 + ks.v2 * rt.v1 + q.v2 * tk.v1 - d1;
        const double t2 = ks.v1 * rr.v2 + q.v1 * rk.v2 + ks.v2 * rt.v2 + q.v2 * tk.v2 - d2;
        const double t3 = ks.v1 * rr.v3 + q.v1 * rk.v3 + ks.v2 * rt.v3 + q.v2 * tk.v3;
        const double h0 = 0.5 * (G00 * t0 + G01 * t1);
        double h1 = 0.5 * (G01 * t0 + G11 * t1 + G13 * t3);
        double h2 = 0.5 * (G22 * t2);
        const double h3 = 0.5 * (G13 * t1 + G33 * t3);
        h1 += r * s.k.v[1] * qn.v[1];
        h2 += t.d2th11 * s.k.v[1] * qn.v[1] + t.d2th12 * (s.k.v[1] * qn.v[2] + s.k.v[2] * qn.v[1]) +
              t.d2th22 * s.k.v[2] * qn.v[2];
        const double h1r = h1 * inv_r;
        D4 out;
        out.v[0] = -h0;
        out.v[1] = -h1r;
        out.v[2] = -((h2 - t.dth1 * h1r) * inv_dth2);
        out.v[3] = -h3;
        return out;
    };
    Ray d;
    d.x = s.k;
    d.k = contract(s.k);
    d.e1 = contract(s.e1);
    d.e2 = contract(s.e2);
    return d;
}

// Camera at phi = 0 and its ipole tetrad in FMKS (camera.hpp:302-456): the
// normal observer, the raised centering covector (1, 1, 0, 0), and the native
// trial vectors (0, 0, 1, 0), (1, 1, 1, 1), made orthonormal by Gram-Schmidt.
// Evaluated once per image (host side).
KP_HD void fmks_camera_frame(const FmksParams& m, double radius, double inclination, D4& x, D4& e0, D4& e1,
                             D4& e2, D4& e3) {
    const double x1 = log(max_val(radius, kTiny));
    x = D4{{0.0, x1, fmks_x2_of(m, x1, inclination), 0.0}};
    double g[4][4], gi[4][4];
    fmks_gcov(m, x, g);
    fmks_gcon(m, x, gi);
    auto dot = [&](const D4& u, const D4& v) { return dot_gm(g, u, v); };
    auto scale = [](D4 v, double s) {
        for (int i = 0; i < 4; ++i) v.v[i] *= s;
        return v;
    };
    auto proj = [&](D4 a, const D4& b) {
        const double b2 = dot(b, b);
        if (abs_val(b2) > kTiny) {
            const double k = dot(a, b) / b2;
            for (int i = 0; i < 4; ++i) a.v[i] -= b.v[i] * k;
        }
        return a;
    };
    auto norm = [&](const D4& v) { return scale(v, 1.0 / sqrt(max_val(abs_val(dot(v, v)), kTiny))); };
    // normal observer: u^mu = -g^{mu 0}, normalised
    D4 u;
    for (int i = 0; i < 4; ++i) u.v[i] = -gi[i][0];
    const double n2 = dot(u, u);
    if (n2 < 0.0) u = scale(u, 1.0 / sqrt(-n2));
    e0 = u;
    const double cov[4] = {1.0, 1.0, 0.0, 0.0};
    for (int i = 0; i < 4; ++i) {
        double sum = 0.0;
        for (int j = 0; j < 4; ++j) sum += gi[i][j] * cov[j];
        e3.v[i] = sum;
    }
    e2 = D4{{0.0, 0.0, 1.0, 0.0}};
    e1 = D4{{1.0, 1.0, 1.0, 1.0}};
    e0 = norm(e0);
    e3 = proj(e3, e0);
    e3 = proj(e3, e0);
    e3 = norm(e3);
    e2 = proj(e2, e0);
    e2 = proj(e2, e3);
    e2 = proj(e2, e0);
    e2 = proj(e2, e3);
    e2 = norm(e2);
    e1 = proj(e1, e0);
    e1 = proj(e1, e2);
    e1 = proj(e1, e3);
    e1 = proj(e1, e0);
    e1 = proj(e1, e2);
    e1 = proj(e1, e3);
    e1 = norm(e1);
    // orientation: the Levi-Civita sign of (e0, e1, e2, e3)
    const double orient = tetrad_orientation(e0, e1, e2, e3);
    if (orient < 0.0) e1 = scale(e1, -1.0);
}

}  // namespace kp
