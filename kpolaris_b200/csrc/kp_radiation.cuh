// kp_radiation.cuh -- FP64 radiation side of the path: RIAF plasma and flow,
// thermal synchrotron coefficients (Pandya and Dexter fits, Faraday rho_Q /
// rho_V), semi-analytic Strang transfer and the observer-basis transform.
//
// Restates src/model/riaf.hpp:54-549, src/radiation/thermal_synchrotron.hpp:60-627,
// src/radiation/semi_analytic.hpp:10-100, src/common/math.hpp:65-85 and
// src/frame/stokes_rotation.hpp:39-57 with their operation order.  The Bessel
// polynomial fits are the reference's own published fits (Numerical Recipes
// forms) re-expressed here.
#pragma once

#include "kp_bl.cuh"
#include "kp_geometry.cuh"

namespace kp {

// CGS constants of the reference's thermal synchrotron module.
constexpr double kEE = 4.803204712570263e-10;
constexpr double kME = 9.1093837015e-28;
constexpr double kCL = 2.99792458e10;
constexpr double kHPL = 6.62607015e-27;
constexpr double kMP = 1.67262192369e-24;

// ---- transfer ----------------------------------------------------------
__device__ __forceinline__ double stable_attenuation(double kappa, double dl) {
    const double x = kappa * dl;
    if (x > 700.0) return 0.0;
    return exp(-x);
}

__device__ __forceinline__ double stable_source_factor(double kappa, double dl) {
    const double x = kappa * dl;
    if (abs_val(x) < 1e-6) return dl * (1.0 - x / 2.0 + x * x / 6.0 - x * x * x / 24.0);
    return (1.0 - exp(-x)) / kappa;
}

// scaled Euclidean norm (src/common/vec.hpp:62-70)
__device__ __forceinline__ double norm3(double x, double y, double z) {
    const double scale = max_val(abs_val(x), max_val(abs_val(y), abs_val(z)));
    if (scale == 0.0) return 0.0;
    const double a = x / scale, b = y / scale, c = z / scale;
    return scale * sqrt(a * a + b * b + c * c);
}

__device__ __forceinline__ void faraday_rotate(Stokes4<double>& s, const Coeffs<double>& c, double dl) {
    const double px = s.Q, py = s.U, pz = s.V;
    const double rho_norm = norm3(c.rQ, c.rU, c.rV);
    if (rho_norm == 0.0 || dl == 0.0) return;
    const double theta = rho_norm * dl;
    double ox, oy, oz;
    if (abs_val(theta) < 1e-8) {
        ox = px + (c.rU * pz - c.rV * py) * dl;
        oy = py + (c.rV * px - c.rQ * pz) * dl;
        oz = pz + (c.rQ * py - c.rU * px) * dl;
    } else {
        const double inv = 1.0 / rho_norm;
        const double nx = c.rQ * inv, ny = c.rU * inv, nz = c.rV * inv;
        double st, ct;
        sincos(theta, &st, &ct);
        const double f = (nx * px + ny * py + nz * pz) * (1.0 - ct);
        ox = px * ct + nx * f + (ny * pz - nz * py) * st;
        oy = py * ct + ny * f + (nz * px - nx * pz) * st;
        oz = pz * ct + nz * f + (nx * py - ny * px) * st;
    }
    s.Q = ox;
    s.U = oy;
    s.V = oz;
}

__device__ __forceinline__ void absorb_emit(Stokes4<double>& s, const Coeffs<double>& c, double dl) {
    const double an = norm3(c.aQ, c.aU, c.aV);
    if (an < kTiny) {
        const double e = stable_attenuation(c.aI, dl);
        const double f = stable_source_factor(c.aI, dl);
        s.I = e * s.I + f * c.jI;
        s.Q = e * s.Q + f * c.jQ;
        s.U = e * s.U + f * c.jU;
        s.V = e * s.V + f * c.jV;
        return;
    }
    const double inv = 1.0 / an;
    const double nx = c.aQ * inv, ny = c.aU * inv, nz = c.aV * inv;
    const double p_par = nx * s.Q + ny * s.U + nz * s.V;
    const double ppx = s.Q - nx * p_par, ppy = s.U - ny * p_par, ppz = s.V - nz * p_par;
    const double j_par = nx * c.jQ + ny * c.jU + nz * c.jV;
    const double jpx = c.jQ - nx * j_par, jpy = c.jU - ny * j_par, jpz = c.jV - nz * j_par;
    const double s_plus = s.I + p_par;
    const double s_minus = s.I - p_par;
    const double j_plus = c.jI + j_par;
    const double j_minus = c.jI - j_par;
    const double k_plus = c.aI + an;
    const double k_minus = c.aI - an;
    const double sp = stable_attenuation(k_plus, dl) * s_plus + stable_source_factor(k_plus, dl) * j_plus;
    const double sm = stable_attenuation(k_minus, dl) * s_minus + stable_source_factor(k_minus, dl) * j_minus;
    const double e_i = stable_attenuation(c.aI, dl);
    const double f_i = stable_source_factor(c.aI, dl);
    const double ox = ppx * e_i + jpx * f_i;
    const double oy = ppy * e_i + jpy * f_i;
    const double oz = ppz * e_i + jpz * f_i;
    const double i_out = 0.5 * (sp + sm);
    const double par_out = 0.5 * (sp - sm);
    s.I = i_out;
    s.Q = nx * par_out + ox;
    s.U = ny * par_out + oy;
    s.V = nz * par_out + oz;
}

static __device__ __noinline__ void stokes_step(Stokes4<double>& s, const Coeffs<double>& c, double dl) {
    faraday_rotate(s, c, 0.5 * dl);
    absorb_emit(s, c, dl);
    faraday_rotate(s, c, 0.5 * dl);
}

// ---- thermal synchrotron ------------------------------------------------
__device__ __forceinline__ double bessel_i0(double ax) {
    if (ax < 3.75) {
        double y = ax / 3.75;
        y *= y;
        double p = 0.0045813;
        p = 0.0360768 + y * p;
        p = 0.2659732 + y * p;
        p = 1.2067492 + y * p;
        p = 3.0899424 + y * p;
        p = 3.5156229 + y * p;
        return 1.0 + y * p;
    }
    const double y = 3.75 / ax;
    double p = 0.00392377;
    p = -0.01647633 + y * p;
    p = 0.02635537 + y * p;
    p = -0.02057706 + y * p;
    p = 0.00916281 + y * p;
    p = -0.00157565 + y * p;
    p = 0.00225319 + y * p;
    p = 0.01328592 + y * p;
    p = 0.39894228 + y * p;
    return exp(ax) / sqrt(ax) * p;
}

__device__ __forceinline__ double bessel_i1(double ax) {
    if (ax < 3.75) {
        double y = ax / 3.75;
        y *= y;
        double p = 0.00032411;
        p = 0.00301532 + y * p;
        p = 0.02658733 + y * p;
        p = 0.15084934 + y * p;
        p = 0.51498869 + y * p;
        p = 0.87890594 + y * p;
        p = 0.5 + y * p;
        return ax * p;
    }
    const double y = 3.75 / ax;
    double p = -0.00420059;
    p = 0.01787654 + y * p;
    p = -0.02895312 + y * p;
    p = 0.02282967 + y * p;
    p = -0.01031555 + y * p;
    p = 0.00163801 + y * p;
    p = -0.00362018 + y * p;
    p = -0.03988024 + y * p;
    p = 0.39894228 + y * p;
    return exp(ax) / sqrt(ax) * p;
}

// K0, K1 and K2 = max(K0 + 2 K1 / x, 1e-300) (thermal_synchrotron.hpp:108-229).
__device__ __forceinline__ void bessel_k012(double x, double& k0, double& k1, double& k2) {
    if (x <= 0.0) {
        k0 = 1e300;
        k1 = 1e300;
    } else if (x <= 2.0) {
        const double y = x * x * 0.25;
        double p = 0.00000740;
        p = 0.00010750 + y * p;
        p = 0.00262698 + y * p;
        p = 0.03488590 + y * p;
        p = 0.23069756 + y * p;
        p = 0.42278420 + y * p;
        p = -0.57721566 + y * p;
        const double lg = log(x * 0.5);
        k0 = -lg * bessel_i0(x) + p;
        double q = -0.00004686;
        q = -0.00110404 + y * q;
        q = -0.01919402 + y * q;
        q = -0.18156897 + y * q;
        q = -0.67278579 + y * q;
        q = 0.15443144 + y * q;
        q = 1.0 + y * q;
        k1 = lg * bessel_i1(x) + q / x;
    } else {
        const double y = 2.0 / x;
        double p = 0.00053208;
        p = -0.00251540 + y * p;
        p = 0.00587872 + y * p;
        p = -0.01062446 + y * p;
        p = 0.02189568 + y * p;
        p = -0.07832358 + y * p;
        p = 1.25331414 + y * p;
        const double ex = exp(-x) / sqrt(x);
        k0 = ex * p;
        double q = -0.00068245;
        q = 0.00325614 + y * q;
        q = -0.00780353 + y * q;
        q = 0.01504268 + y * q;
        q = -0.03655620 + y * q;
        q = 0.23498619 + y * q;
        q = 1.25331414 + y * q;
        k1 = ex * q;
    }
    k2 = max_val(k0 + 2.0 * k1 / max_val(x, 1e-300), 1e-300);
}

__device__ __forceinline__ double bnu_inv(double nu, double thetae) {
    if (!(thetae > 0.0)) return 0.0;
    const double x = kHPL * nu / (kME * kCL * kCL * thetae);
    if (x < 2e-3) {
        const double denom = x / 24.0 * (24.0 + x * (12.0 + x * (4.0 + x)));
        return (2.0 * kHPL / max_val(denom, kTiny)) / (kCL * kCL);
    }
    const double denom = exp(x) - 1.0;
    return (2.0 * kHPL / max_val(denom, kTiny)) / (kCL * kCL);
}

// rho_Q and rho_V fits (symphony_rho_QV, thermal_synchrotron.hpp:462-506).
__device__ __forceinline__ void rho_QV(double nu, double ne, double thetae, double b, double st,
                                       double ct, double& rhoQ, double& rhoV) {
    const double omega0 = kEE * b / (kME * kCL);
    const double wp2 = 4.0 * kPi * ne * kEE * kEE / kME;
    const double two_pi_nu = 2.0 * kPi * nu;
    const double x = max_val(thetae * sqrt(max_val(0.0, sqrt(2.0) * st * (1e3 * omega0 / max_val(two_pi_nu, kTiny)))), 1e-12);
    double k0, k1, k2;
    bessel_k012(1.0 / thetae, k0, k1, k2);
    const double exp_x_47 = exp(-x / 47.2);
    const double extraterm = (0.011 * exp_x_47 - 369.69342869090815 * pow(x + 1e-16, -8.0 / 3.0)) *
                             (0.5 + 0.5 * tanh((log(x) - 4.787491742782046) / 0.1));
    const double jffunc = 2.011 * exp(-pow(x, 1.035) / 4.7) - cos(x / 2.0) * exp(-pow(x, 1.2) / 2.73) -
                          0.011 * exp_x_47 + extraterm;
    const double k1_ratio = k2 > 0.0 ? k1 / k2 : 1.0;
    const double safe = max_val(two_pi_nu, kTiny);
    double e11 = jffunc * wp2 * omega0 * omega0;
    e11 /= safe;
    e11 /= safe;
    e11 /= safe;
    e11 /= safe;
    e11 *= (k1_ratio + 6.0 * thetae) * st * st;
    rhoQ = kPi * nu / kCL * e11;
    const double shgm = 1.0 - 0.11 * log(1.0 + 0.035 * x);
    const double k0_ratio = k2 > 0.0 ? k0 / k2 : 1.0;
    const double fit_factor = k0_ratio * shgm;
    double e12 = wp2 * omega0;
    e12 /= safe;
    e12 /= safe;
    e12 /= safe;
    e12 *= fit_factor * ct;
    rhoV = 2.0 * kPi * nu / kCL * e12;
}

// symphony_rho_V with theta on the field axis (thermal_synchrotron.hpp:433-460).
__device__ __forceinline__ double rho_V_axis(double nu, double ne, double thetae, double b, double theta,
                                             double min_st) {
    const double st = max_val(sin(theta), min_st);
    const double omega0 = kEE * b / (kME * kCL);
    const double wp2 = 4.0 * kPi * ne * kEE * kEE / kME;
    const double two_pi_nu = 2.0 * kPi * nu;
    const double x = max_val(thetae * sqrt(max_val(0.0, sqrt(2.0) * st * (1e3 * omega0 / max_val(two_pi_nu, kTiny)))), 1e-12);
    double k0, k1, k2;
    bessel_k012(1.0 / thetae, k0, k1, k2);
    const double shgm = 1.0 - 0.11 * log(1.0 + 0.035 * x);
    const double k_ratio = k2 > 0.0 ? k0 / k2 : 1.0;
    const double fit_factor = k_ratio * shgm;
    const double safe = max_val(two_pi_nu, kTiny);
    double e12 = wp2 * omega0;
    e12 /= safe;
    e12 /= safe;
    e12 /= safe;
    e12 *= fit_factor * cos(theta);
    return 2.0 * kPi * nu / kCL * e12;
}

struct ThermalIn {
    double nu, ne, thetae, b, st, ct;
};

// Invariant coefficients in the magnetic basis
// (thermal_synchrotron_magnetic_basis_coefficients_fit, :512-627).
static __device__ __noinline__ Coeffs<double> thermal_coefficients(const ThermalIn& s, const ImageConsts& c) {
    Coeffs<double> o = {};
    if (!(s.nu > 0.0) || !(s.ne > 0.0) || !(s.thetae > 0.0) || !(s.b > 0.0)) return o;
    const double nu = max_val(s.nu, 1.0);
    const double st = max_val(s.st, c.min_sin_theta);
    double jI = 0.0, jQ = 0.0, jV = 0.0;
    if (c.fit == 4) {
        const double nus = 3.0 * kEE * s.b * st / (4.0 * kPi * kME * kCL) * s.thetae * s.thetae + 1.0;
        const double x = max_val(nu / max_val(nus, kTiny), kTiny);
        const double xm13 = 1.0 / cbrt(x);
        const double exp_shape = exp(-1.8899 / xm13);
        const double pref = s.ne * kEE * kEE * nu / (2.0 * sqrt(3.0) * kCL * s.thetae * s.thetae);
        const double i_val = 2.5651 * (1.0 + 1.92 * xm13 + 0.9977 * xm13 * xm13) * exp_shape;
        const double iq = 2.5651 * (1.0 + 0.93193 * xm13 + 0.499873 * xm13 * xm13) * exp_shape;
        jI = pref * i_val;
        jQ = pref * iq;
        // jV repeats the nus/x evaluation with the same sin(theta) (identical values).
        const double iv = (1.81384 / x + 3.42319 * xm13 * xm13 + 0.0292545 / sqrt(x) + 2.03773 * xm13) *
                          exp_shape;
        double cft = s.ct;
        if (abs_val(cft) < 1e-10) cft = cft >= 0.0 ? 1e-10 : -1e-10;
        const double tan_theta = st / cft;
        jV = 2.0 * s.ne * kEE * kEE * nu /
             (tan_theta * 3.0 * sqrt(3.0) * kCL * s.thetae * s.thetae * s.thetae) * iv;
    } else {
        if (!(s.thetae > 0.0) || !(s.ne > 0.0) || !(s.b > 0.0) || !(st > 0.0)) {
            jI = jQ = jV = 0.0;
        } else {
            const double nu_c = kEE * s.b / (2.0 * kPi * kME * kCL);
            const double nu_s = 2.0 / 9.0 * nu_c * st * s.thetae * s.thetae;
            const double x = max_val(nu / max_val(nu_s, kTiny), kTiny);
            const double prefactor = s.ne * kEE * kEE * nu_c / kCL;
            const double term1 = sqrt(2.0) * kPi / 27.0 * st;
            const double x13 = cbrt(x);
            const double sqx = sqrt(x);
            const double sqx13 = sqrt(x13);
            const double ex13 = exp(-x13);
            const double shape = sqx + 1.8877486253633869933 * sqx13;
            jI = prefactor * term1 * (shape * shape) * ex13;
            const double t2425 = pow(s.thetae, 24.0 / 25.0);
            const double term2 = (7.0 * t2425 + 35.0) / (10.0 * t2425 + 75.0);
            const double shapeq = sqx + term2 * 1.8877486253633869933 * sqx13;
            jQ = prefactor * term1 * (shapeq * shapeq) * ex13;
            const double sin_shift = st * 0.4356824462767121 - s.ct * 0.9001004421765051;
            const double vt1 = (37.0 - 87.0 * sin_shift) / (100.0 * (s.thetae + 1.0));
            const double vt2 = pow(1.0 + (pow(s.thetae, 3.0 / 5.0) / 25.0 + 7.0 / 10.0) * pow(x, 9.0 / 25.0), 5.0 / 3.0);
            jV = prefactor * vt1 * vt2 * ex13;
        }
    }
    const double nusq = nu * nu;
    double jI_inv = jI / max_val(nusq, kTiny);
    double jQ_inv = jQ / max_val(nusq, kTiny);
    double jV_inv = jV / max_val(nusq, kTiny);
    const double jP_scale = max_val(abs_val(jQ_inv), abs_val(jV_inv));
    const double jP = jP_scale > 0.0 ? jP_scale * sqrt(sq(jQ_inv / jP_scale) + sq(jV_inv / jP_scale)) : 0.0;
    if (jI_inv > 0.0 && jP > 0.0 && jI_inv < jP / max_val(c.max_pol_frac, 1e-30)) {
        const double scale = jI_inv / jP * c.max_pol_frac;
        jQ_inv *= scale;
        jV_inv *= scale;
    }
    double aI = 0.0, aQ = 0.0, aV = 0.0;
    const double b_inv = bnu_inv(nu, s.thetae);
    if (b_inv > 0.0) {
        aI = jI_inv / b_inv;
        aQ = jQ_inv / b_inv;
        aV = jV_inv / b_inv;
    }
    double rQ = 0.0, rV = 0.0;
    rho_QV(nu, s.ne, s.thetae, s.b, st, s.ct, rQ, rV);
    o.jI = c.emission_scale * jI_inv;
    o.jQ = c.emission_scale * jQ_inv;
    o.jV = c.emission_scale * jV_inv;
    o.aI = c.absorption_scale * aI;
    o.aQ = c.absorption_scale * aQ;
    o.aV = c.absorption_scale * aV;
    o.rQ = c.faraday_scale * (rQ * nu);
    o.rV = c.faraday_scale * (rV * nu);
    return o;
}

// ---- RIAF plasma and flow (src/model/riaf.hpp) ---------------------------
__device__ __forceinline__ void bl_metric(double r, double th, double spin, double gcov[4][4],
                                          double gcon[4][4]) {
    const double a = spin;
    const double a2 = a * a;
    double sinth, costh;
    sincos(th, &sinth, &costh);
    const double sin2 = max_val(sinth * sinth, 1e-30);
    const double sigma = r * r + a2 * costh * costh;
    const double delta = r * r - 2.0 * r + a2;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) {
            gcov[mu][nu] = 0.0;
            gcon[mu][nu] = 0.0;
        }
    gcov[0][0] = -(1.0 - 2.0 * r / sigma);
    gcov[0][3] = gcov[3][0] = -2.0 * a * r * sin2 / sigma;
    gcov[1][1] = sigma / max_val(delta, kTiny);
    gcov[2][2] = sigma;
    gcov[3][3] = (r * r + a2 + 2.0 * a2 * r * sin2 / sigma) * sin2;
    const double inv_sd = 1.0 / max_val(sigma * delta, kTiny);
    gcon[0][0] = -((r * r + a2) * (r * r + a2) - a2 * delta * sin2) * inv_sd;
    gcon[0][3] = gcon[3][0] = -2.0 * a * r * inv_sd;
    gcon[1][1] = delta / sigma;
    gcon[2][2] = 1.0 / sigma;
    gcon[3][3] = (delta - a2 * sin2) / max_val(sigma * delta * sin2, kTiny);
}

__device__ __forceinline__ double signed_nonzero(double x) {
    if (abs_val(x) > kTiny) return x;
    return x < 0.0 ? -kTiny : kTiny;
}

__device__ __forceinline__ D4 bl_to_cks(double vt, double vr, double vth, double vphi, double r,
                                        double sinth, double costh, double cphi, double sphi,
                                        double spin) {
    const double a = spin;
    const double delta = max_val(r * r - 2.0 * r + a * a, kTiny);
    const double vt_ks = vt + 2.0 * r / delta * vr;
    const double vphi_ks = vphi + a / delta * vr;
    const double dx_dr = cphi * sinth;
    const double dy_dr = sphi * sinth;
    const double dz_dr = costh;
    const double dx_dth = (r * cphi - a * sphi) * costh;
    const double dy_dth = (r * sphi + a * cphi) * costh;
    const double dz_dth = -r * sinth;
    const double dx_dphi = (-r * sphi - a * cphi) * sinth;
    const double dy_dphi = (r * cphi - a * sphi) * sinth;
    D4 o;
    o.v[0] = vt_ks;
    o.v[1] = vr * dx_dr + vth * dx_dth + vphi_ks * dx_dphi;
    o.v[2] = vr * dy_dr + vth * dy_dth + vphi_ks * dy_dphi;
    o.v[3] = vr * dz_dr + vth * dz_dth + vphi_ks * 0.0;
    return o;
}

__device__ __forceinline__ double dot_g(const double g[4][4], const D4& u, const D4& v) {
    double out = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) out += g[mu][nu] * u.v[mu] * v.v[nu];
    return out;
}

__device__ __forceinline__ D4 lower_g(const double g[4][4], const D4& v) {
    D4 o;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        double sum = 0.0;
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) sum += g[mu][nu] * v.v[nu];
        o.v[mu] = sum;
    }
    return o;
}

__device__ __forceinline__ double screen_inner(const double g[4][4], const D4& u, const D4& k,
                                               const D4& a, const D4& b) {
    const double uk = dot_g(g, u, k);
    if (abs_val(uk) <= kTiny) return dot_g(g, a, b);
    const double s = -1.0 / uk;
    D4 eK;
#pragma unroll
    for (int i = 0; i < 4; ++i) eK.v[i] = k.v[i] * s - u.v[i];
    return dot_g(g, a, b) + dot_g(g, u, a) * dot_g(g, u, b) - dot_g(g, eK, a) * dot_g(g, eK, b);
}

// Frequency-independent plasma state at a sample point.  The reference
// recomputes it for every frequency (it copies the model per channel,
// pass_b.hpp:1433-1448); computing it once gives the same values.
struct RiafSample {
    int emitting;      // 0: outside the plasma, all coefficients zero
    int on_axis;       // theta == 0 or pi: only rho_V survives
    double ne, thetae, b;
    double nu_fluid;   // -k.u
    double cos_theta, sin_theta, theta;
    double cos2chi, sin2chi;
    int has_chi;
};

// Boyer-Lindquist r, theta and the azimuth's cosine and sine of a
// Cartesian Kerr-Schild position (bl_coordinates, riaf.hpp:98-122).
struct BlCoords {
    double rc, th, sin_th, cos_th, cphi, sphi;
};

__device__ __forceinline__ BlCoords riaf_bl_coords(double spin, const D4& x) {
    BlCoords q;
    const double xx = x.v[1], yy = x.v[2], zz = x.v[3];
    const double a2 = spin * spin;
    const double radius2 = xx * xx + yy * yy + zz * zz;
    const double sqsum = radius2 - a2;
    const double discr = sqrt(sqsum * sqsum + 4.0 * a2 * zz * zz);
    q.rc = sqrt(max_val(0.5 * (sqsum + discr), kTiny));
    q.th = acos(clamp_val(zz / max_val(q.rc, kTiny), -1.0, 1.0));
    sincos(q.th, &q.sin_th, &q.cos_th);
    const double sinth_f = max_val(q.sin_th, 1e-30);
    const double denom = max_val(sinth_f * (q.rc * q.rc + a2), kTiny);
    q.cphi = (q.rc * xx + spin * yy) / denom;
    q.sphi = (q.rc * yy - spin * xx) / denom;
    const double normp = sqrt(max_val(q.cphi * q.cphi + q.sphi * q.sphi, kTiny));
    q.cphi /= normp;
    q.sphi /= normp;
    return q;
}

// n_e, Theta_e and B of the plasma at BL (r, theta): density_profile_bl
// (riaf.hpp:54-60), thetae_profile (:67-74), magnetic_field_cgs (:87-96)
// at r_bl = max(r, min_radius).  Returns 0 outside the emitting region.
__device__ __forceinline__ int riaf_plasma(const ImageConsts& c, const BlCoords& q, double& r_bl, double& ne,
                                           double& thetae, double& b) {
    r_bl = max_val(q.rc, c.min_radius);
    if (r_bl <= c.horizon + c.horizon_buffer || r_bl < c.r_min || r_bl > c.r_max) return 0;
    double ne_norm;
    {
        const double zc = r_bl * q.cos_th;
        const double rcyl = max_val(r_bl * q.sin_th, c.min_radius);
        const double h = max_val(c.disk_h, 1e-6);
        const double vertical = exp(-(zc * zc) / (2.0 * rcyl * rcyl * h * h));
        ne_norm = c.nth0 * vertical * pow(max_val(r_bl, c.min_radius), c.pow_nth);
    }
    if (!(ne_norm > 0.0)) return 0;
    ne = ne_norm * c.ne_unit;
    thetae = max_val(c.Te0 * pow(max_val(r_bl, c.min_radius), c.pow_T) * c.thetae_unit, c.min_thetae);
    {
        const double bb = sqrt(max_val(8.0 * kPi * 0.1 * ne * kMP * kCL * kCL / (6.0 * max_val(r_bl, c.min_radius)), 0.0));
        b = max_val(bb, 1e-12);
    }
    return 1;
}

// The plasma state of a sample point, in either chart of the RIAF scenes
// (kBL: the ray is in Boyer-Lindquist coordinates, where the model's BL
// quantities are the ray's own components; otherwise Cartesian Kerr-Schild,
// converted with bl_to_cks -- bl_coordinates_for_metric and the
// coordinate_system branches of riaf.hpp:124-137, 255-268, 350-364).
template<bool kBL>
static __device__ __noinline__ RiafSample riaf_sample_t(const ImageConsts& c, const Ray& s) {
    RiafSample out;
    out.emitting = 0;
    out.on_axis = 0;
    out.has_chi = 0;
    const double spin = c.spin;
    BlCoords q;
    if constexpr (kBL) {
        q.rc = s.x.v[1];
        q.th = s.x.v[2];
        q.sin_th = sin(q.th);
        q.cos_th = cos(q.th);
        q.cphi = cos(s.x.v[3]);
        q.sphi = sin(s.x.v[3]);
    } else {
        q = riaf_bl_coords(spin, s.x);
    }
    const double rc = q.rc, th = q.th, sin_th = q.sin_th, cos_th = q.cos_th, cphi = q.cphi, sphi = q.sphi;
    double r_bl;
    if (!riaf_plasma(c, q, r_bl, out.ne, out.thetae, out.b)) return out;
    out.emitting = 1;
    double g[4][4];
    if constexpr (kBL) {
        bl_gcov_matrix(c.mass, spin, s.x, g);
    } else {
        ks_gcov_matrix(c.mass, spin, s.x, g);
    }
    // fluid_four_velocity_from_bl_coords (riaf.hpp:206-273) at r = r_bl
    D4 ucon;
    {
        const double r = r_bl;
        double gcov[4][4], gcon[4][4];
        bl_metric(r, th, spin, gcov, gcon);
        double vt = 1.0, vr = 0.0, vphi = 0.0;
        if (r < c.horizon) {
            vt = 1.0 / sqrt(max_val(-gcon[0][0], kTiny));
        } else if (r < c.isco) {
            double gi[4][4], gci[4][4];
            bl_metric(c.isco, th, spin, gi, gci);
            const double risco = c.isco;
            const double omega_isco = 1.0 / (risco * sqrt(risco) + spin);
            const double qi = gi[0][0] + 2.0 * omega_isco * gi[0][3] + omega_isco * omega_isco * gi[3][3];
            const double ut_i = 1.0 / sqrt(max_val(-qi, kTiny));
            const double e = (gi[0][0] + gi[0][3] * omega_isco) * ut_i;
            const double l = (gi[3][0] + gi[3][3] * omega_isco) * ut_i;
            const double k_con = gcon[0][0] * e * e + 2.0 * gcon[0][3] * e * l + gcon[3][3] * l * l;
            const double ur_cov = -sqrt(max_val(-(1.0 + k_con) / max_val(gcon[1][1], kTiny), 0.0));
            const double vr_tmp = gcon[1][1] * ur_cov;
            const double vt_tmp = gcon[0][0] * e + gcon[0][3] * l;
            const double vphi_tmp = gcon[3][0] * e + gcon[3][3] * l;
            const double omega_k = vphi_tmp / max_val(vt_tmp, kTiny);
            const double omega_ff = gcon[0][3] / signed_nonzero(gcon[0][0]);
            const double omega = omega_k + (1.0 - c.keplerian_factor) * (omega_ff - omega_k);
            const double ur_ff = -sqrt(max_val(-(1.0 + gcon[0][0]) * gcon[1][1], 0.0));
            vr = vr_tmp + c.infall_factor * (ur_ff - vr_tmp);
            const double q = gcov[0][0] + 2.0 * omega * gcov[0][3] + omega * omega * gcov[3][3];
            vt = sqrt(max_val(-(1.0 + vr * vr * gcov[1][1]) / q, 0.0));
            vphi = omega * vt;
        } else {
            const double r_eff = max_val(r, c.min_radius);
            const double omega_k = 1.0 / (r_eff * sqrt(r_eff) + spin);
            const double omega_ff = gcon[0][3] / signed_nonzero(gcon[0][0]);
            const double omega = omega_k + (1.0 - c.keplerian_factor) * (omega_ff - omega_k);
            vr = c.infall_factor * -sqrt(max_val(-(1.0 + gcon[0][0]) * gcon[1][1], 0.0));
            const double q = gcov[0][0] + 2.0 * omega * gcov[0][3] + omega * omega * gcov[3][3];
            vt = sqrt(max_val(-(1.0 + vr * vr * gcov[1][1]) / q, 0.0));
            vphi = omega * vt;
        }
        if constexpr (kBL) {
            ucon = d4(vt, vr, 0.0, vphi);
        } else {
            ucon = bl_to_cks(vt, vr, 0.0, vphi, r, sin_th, cos_th, cphi, sphi, spin);
        }
        const double n2 = dot_g(g, ucon, ucon);
        if (n2 < 0.0) ucon = d4_scale(ucon, 1.0 / sqrt(max_val(-n2, kTiny)));
    }
    const D4 ucov = lower_g(g, ucon);
    double uk = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) uk += ucov.v[mu] * s.k.v[mu];
    out.nu_fluid = max_val(abs_val(-uk), c.min_frequency_scale);
    // magnetic_unit_four_vector_with_gcov (riaf.hpp:350-386): toroidal trial vector
    // at the raw BL radius rc of the sample.
    D4 bcon;
    {
        D4 bt = kBL ? d4(0.0, 0.0, 0.0, 1.0) : bl_to_cks(0.0, 0.0, 0.0, 1.0, rc, sin_th, cos_th, cphi, sphi, spin);
        double udotb = dot_g(g, ucon, bt);
        for (int i = 0; i < 4; ++i) bcon.v[i] = bt.v[i] + ucon.v[i] * udotb;
        double bsq = dot_g(g, bcon, bcon);
        if (!(bsq > 1e-30)) {
            bt.v[0] = 0.0; bt.v[1] = 0.0; bt.v[2] = 0.0; bt.v[3] = 1.0;
            udotb = dot_g(g, ucon, bt);
            for (int i = 0; i < 4; ++i) bcon.v[i] = bt.v[i] + ucon.v[i] * udotb;
            bsq = dot_g(g, bcon, bcon);
        }
        if (!(bsq > 1e-30)) {
            bt.v[0] = 0.0; bt.v[1] = 1.0; bt.v[2] = 0.0; bt.v[3] = 0.0;
            udotb = dot_g(g, ucon, bt);
            for (int i = 0; i < 4; ++i) bcon.v[i] = bt.v[i] + ucon.v[i] * udotb;
            bsq = dot_g(g, bcon, bcon);
        }
        if (bsq > 1e-30) bcon = d4_scale(bcon, 1.0 / sqrt(bsq));
    }
    const D4 bcov = lower_g(g, bcon);
    double kdotb = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) kdotb += s.k.v[mu] * bcov.v[mu];
    out.cos_theta = clamp_val(kdotb / max_val(out.nu_fluid, 1e-30), -1.0, 1.0);
    out.sin_theta = max_val(sqrt(max_val(0.0, 1.0 - out.cos_theta * out.cos_theta)), c.min_sin_theta);
    out.theta = acos(clamp_val(out.cos_theta, -1.0, 1.0));
    if (out.theta <= 0.0 || out.theta >= kPi) {
        out.on_axis = 1;
        return out;
    }
    const double b1 = screen_inner(g, ucon, s.k, s.e1, bcon);
    const double b2 = screen_inner(g, ucon, s.k, s.e2, bcon);
    const double bproj2 = b1 * b1 + b2 * b2;
    if (bproj2 > 1e-30) {
        out.has_chi = 1;
        out.cos2chi = (b2 * b2 - b1 * b1) / bproj2;
        out.sin2chi = -2.0 * b1 * b2 / bproj2;
    }
    return out;
}

static __device__ __forceinline__ RiafSample riaf_sample(const ImageConsts& c, const Ray& s) {
    return riaf_sample_t<false>(c, s);
}

// RIAFAnalyticRadiationModel::coefficients for one frequency (riaf.hpp:410-549).
__device__ __forceinline__ Coeffs<double> riaf_coefficients(const ImageConsts& c, const RiafSample& p,
                                                            double freq) {
    Coeffs<double> o = {};
    if (!p.emitting) return o;
    const double nu = max_val(freq * p.nu_fluid, 1.0);
    if (p.on_axis) {
        o.rV = c.faraday_scale * rho_V_axis(nu, p.ne, p.thetae, p.b, p.theta, c.min_sin_theta) * nu;
        return o;
    }
    ThermalIn ti = {nu, p.ne, p.thetae, p.b, p.sin_theta, p.cos_theta};
    const Coeffs<double> m = thermal_coefficients(ti, c);
    o.jI = m.jI;
    o.jV = m.jV;
    o.aI = m.aI;
    o.aV = m.aV;
    o.rV = m.rV;
    if (p.has_chi) {
        o.jQ = m.jQ * p.cos2chi;
        o.jU = m.jQ * p.sin2chi;
        o.aQ = m.aQ * p.cos2chi;
        o.aU = m.aQ * p.sin2chi;
        o.rQ = m.rQ * p.cos2chi;
        o.rU = m.rQ * p.sin2chi;
    }
    return o;
}

}  // namespace kp
