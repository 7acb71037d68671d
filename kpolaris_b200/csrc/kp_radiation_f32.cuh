// kp_radiation_f32.cuh -- FP32 radiation side of the mixed-precision path:
// RIAF plasma state, thermal synchrotron coefficients and the Strang transfer
// step, with the same formulas as kp_radiation.cuh (and the reference's
// src/model/riaf.hpp:54-549, src/radiation/thermal_synchrotron.hpp:60-627,
// src/radiation/semi_analytic.hpp:10-100) rearranged for FP32 range:
//
//  * invariant emissivities j ~ 1e-38..1e-48 underflow FP32, so emission and
//    the Stokes vector carry a per-image, per-frequency factor 2^E (the
//    transfer equation is linear in (j, S)); the image is unscaled in FP64;
//  * absorption a = j / B_nu is formed as j_phys * [c^2/(2h)] (e^x - 1) / nu^2
//    with nu in GHz so every intermediate stays inside FP32 range;
//  * the Bessel K ratios cancel the common e^-x / sqrt(x) factor;
//  * the Stokes update is compensated (a running TwoSum error term per
//    component).
// Absorption and Faraday coefficients times the affine step are O(1) and
// need no scaling.
#pragma once

#include "kp_geometry.cuh"

namespace kp {

namespace f32c {
constexpr float kPi = 3.14159265358979323846f;
constexpr double kEE = 4.803204712570263e-10;
constexpr double kME = 9.1093837015e-28;
constexpr double kCL = 2.99792458e10;
constexpr double kHPL = 6.62607015e-27;
constexpr double kMP = 1.67262192369e-24;
// nu_c = e B / (2 pi m_e c) per gauss
constexpr float kNuCPerB = float(kEE / (2.0 * 3.141592653589793 * kME * kCL));
// e^2 / c
constexpr float kE2OverC = float(kEE * kEE / kCL);
// sqrt(2) pi / 27
constexpr float kTerm1 = float(1.4142135623730951 * 3.141592653589793 / 27.0);
// h / (m_e c^2) * 1e9 : x = h nu / (m_e c^2 Theta_e) with nu in GHz
constexpr float kHOverMc2GHz = float(kHPL / (kME * kCL * kCL) * 1e9);
// c^2 / (2 h) / 1e18 : absorption factor with nu in GHz
constexpr float kC2Over2hGHz2 = float(kCL * kCL / (2.0 * kHPL) / 1e18);
// omega0 per gauss: e / (m_e c)
constexpr float kOmega0PerB = float(kEE / (kME * kCL));
// wp^2 per n_e: 4 pi e^2 / m_e
constexpr float kWp2PerNe = float(4.0 * 3.141592653589793 * kEE * kEE / kME);
// Dexter: 3 e / (4 pi m_e c)
constexpr float kDexNus = float(3.0 * kEE / (4.0 * 3.141592653589793 * kME * kCL));
// Dexter prefactor e^2 / (2 sqrt(3) c)
constexpr float kDexPref = float(kEE * kEE / (2.0 * 1.7320508075688772 * kCL));
// Dexter jV prefactor 2 e^2 / (3 sqrt(3) c)
constexpr float kDexPrefV = float(2.0 * kEE * kEE / (3.0 * 1.7320508075688772 * kCL));
}  // namespace f32c

struct CoeffsF {
    float jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV;
};

KP_HD float kp_rsqrtf(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / sqrtf(x);
#endif
}

KP_HD void kp_sincosf(float x, float* s, float* c) {
#ifdef __CUDA_ARCH__
    sincosf(x, s, c);
#else
    *s = sinf(x);
    *c = cosf(x);
#endif
}

// sin and cos of an angle that is usually small: below |x| = 0.5 from their
// Taylor series to the x^9 / x^8 terms (truncation < 1e-11, under FP32
// rounding), keeping full relative accuracy where a hardware sine's absolute
// error would not; above it the library (or hardware) form.
KP_HD void kp_sincos_small(float x, float* s, float* c) {
    if (fabsf(x) < 0.5f) {
        const float x2 = x * x;
        *s = x * (1.0f - x2 * (1.0f / 6.0f) * (1.0f - x2 * (1.0f / 20.0f) * (1.0f - x2 * (1.0f / 42.0f) *
                                                                                     (1.0f - x2 * (1.0f / 72.0f)))));
        *c = 1.0f - x2 * 0.5f * (1.0f - x2 * (1.0f / 12.0f) * (1.0f - x2 * (1.0f / 30.0f) * (1.0f - x2 * (1.0f / 56.0f))));
        return;
    }
    kp_sincosf(x, s, c);
}

struct StokesF {
    float I, Q, U, V;     // scaled by 2^E
    float cI, cQ, cU, cV; // compensation terms
};

// K0/K2 and K1/K2 for x = 1/Theta_e with the polynomial fits of
// thermal_synchrotron.hpp:108-158; for x > 2 the factor e^-x / sqrt(x) cancels.
KP_HD void bessel_ratios_f(float x, float& r0, float& r1) {
    float p, q;
    if (x <= 2.0f) {
        const float y = x * x * 0.25f;
        float i0, i1;
        {
            const float t = (x / 3.75f) * (x / 3.75f);
            float a = 0.0045813f;
            a = 0.0360768f + t * a;
            a = 0.2659732f + t * a;
            a = 1.2067492f + t * a;
            a = 3.0899424f + t * a;
            a = 3.5156229f + t * a;
            i0 = 1.0f + t * a;
            float b = 0.00032411f;
            b = 0.00301532f + t * b;
            b = 0.02658733f + t * b;
            b = 0.15084934f + t * b;
            b = 0.51498869f + t * b;
            b = 0.87890594f + t * b;
            b = 0.5f + t * b;
            i1 = x * b;
        }
        float a = 0.00000740f;
        a = 0.00010750f + y * a;
        a = 0.00262698f + y * a;
        a = 0.03488590f + y * a;
        a = 0.23069756f + y * a;
        a = 0.42278420f + y * a;
        a = -0.57721566f + y * a;
        const float lg = logf(x * 0.5f);
        p = -lg * i0 + a;
        float b = -0.00004686f;
        b = -0.00110404f + y * b;
        b = -0.01919402f + y * b;
        b = -0.18156897f + y * b;
        b = -0.67278579f + y * b;
        b = 0.15443144f + y * b;
        b = 1.0f + y * b;
        q = lg * i1 + b / x;
    } else {
        const float y = 2.0f / x;
        float a = 0.00053208f;
        a = -0.00251540f + y * a;
        a = 0.00587872f + y * a;
        a = -0.01062446f + y * a;
        a = 0.02189568f + y * a;
        a = -0.07832358f + y * a;
        a = 1.25331414f + y * a;
        p = a;
        float b = -0.00068245f;
        b = 0.00325614f + y * b;
        b = -0.00780353f + y * b;
        b = 0.01504268f + y * b;
        b = -0.03655620f + y * b;
        b = 0.23498619f + y * b;
        b = 1.25331414f + y * b;
        q = b;
    }
    const float k2 = p + 2.0f * q / x;
    r0 = k2 > 0.0f ? p / k2 : 1.0f;
    r1 = k2 > 0.0f ? q / k2 : 1.0f;
}

// Plasma state at a sample point (FP32), with the frequency-independent
// factors of the thermal fits (riaf_sample_thermal_f).
struct RiafSampleF {
    int emitting, on_axis, has_chi;
    float ne, thetae, b, nu_fluid, cos_theta, sin_theta, theta, cos2chi, sin2chi;
    float r0, r1;   // K0/K2, K1/K2 at 1/Theta_e (Faraday fits)
    float qterm;    // (7 T^0.96 + 35) / (10 T^0.96 + 75), Pandya jQ
    float vt1;      // (37 - 87 sin(theta - 0.45)) / (100 (T + 1)), Pandya jV
    float vt2a;     // T^0.6 / 25 + 0.7, Pandya jV
};

// x^y for x > 0 as 2^(y log2 x): one LG2 shared by several powers of x.
KP_HD float pow2_of(float y, float lg2x) {
#ifdef __CUDA_ARCH__
    return exp2f(y * lg2x);
#else
    return std::exp2(y * lg2x);
#endif
}

// Frequency-independent factors of the thermal fits at one sample
// (thermal_synchrotron.hpp:312-395, 462-506), evaluated once per sample
// instead of once per frequency.
KP_HD void riaf_sample_thermal_f(const ImageConsts& c, RiafSampleF& p) {
    const float te = p.thetae;
    bessel_ratios_f(1.0f / te, p.r0, p.r1);
    const float lt = log2f(te);
    const float t2425 = pow2_of(24.0f / 25.0f, lt);
    p.qterm = (7.0f * t2425 + 35.0f) / (10.0f * t2425 + 75.0f);
    const float st = fmaxf(p.sin_theta, float(c.min_sin_theta));
    const float sin_shift = st * 0.4356824462767121f - p.cos_theta * 0.9001004421765051f;
    p.vt1 = (37.0f - 87.0f * sin_shift) / (100.0f * (te + 1.0f));
    p.vt2a = pow2_of(0.6f, lt) / 25.0f + 0.7f;
}

KP_HD float dot_gf(const float g[4][4], const float* u, const float* v) {
    float out = 0.0f;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) out += g[mu][nu] * u[mu] * v[nu];
    return out;
}

KP_HD void bl_metric_f(float r, float sinth, float costh, float a, float gcov[4][4],
                                            float gcon[4][4]) {
    const float a2 = a * a;
    const float sin2 = fmaxf(sinth * sinth, 1e-30f);
    const float sigma = r * r + a2 * costh * costh;
    const float delta = r * r - 2.0f * r + a2;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) {
            gcov[mu][nu] = 0.0f;
            gcon[mu][nu] = 0.0f;
        }
    gcov[0][0] = -(1.0f - 2.0f * r / sigma);
    gcov[0][3] = gcov[3][0] = -2.0f * a * r * sin2 / sigma;
    gcov[1][1] = sigma / fmaxf(delta, 1e-30f);
    gcov[2][2] = sigma;
    gcov[3][3] = (r * r + a2 + 2.0f * a2 * r * sin2 / sigma) * sin2;
    const float inv_sd = 1.0f / fmaxf(sigma * delta, 1e-30f);
    gcon[0][0] = -((r * r + a2) * (r * r + a2) - a2 * delta * sin2) * inv_sd;
    gcon[0][3] = gcon[3][0] = -2.0f * a * r * inv_sd;
    gcon[1][1] = delta / sigma;
    gcon[2][2] = 1.0f / sigma;
    gcon[3][3] = (delta - a2 * sin2) / fmaxf(sigma * delta * sin2, 1e-30f);
}

KP_HD void bl_to_cks_f(float vt, float vr, float vphi, float r, float sinth, float costh,
                                            float cphi, float sphi, float a, float* o) {
    const float delta = fmaxf(r * r - 2.0f * r + a * a, 1e-30f);
    const float vt_ks = vt + 2.0f * r / delta * vr;
    const float vphi_ks = vphi + a / delta * vr;
    o[0] = vt_ks;
    o[1] = vr * cphi * sinth + vphi_ks * (-r * sphi - a * cphi) * sinth;
    o[2] = vr * sphi * sinth + vphi_ks * (r * cphi - a * sphi) * sinth;
    o[3] = vr * costh;
}

// riaf_sample (kp_radiation.cuh) in FP32.
KP_HD RiafSampleF riaf_sample_f(const ImageConsts& c, const Ray& s) {
    RiafSampleF out;
    out.emitting = 0;
    out.on_axis = 0;
    out.has_chi = 0;
    const float a = float(c.spin);
    const float xx = float(s.x.v[1]), yy = float(s.x.v[2]), zz = float(s.x.v[3]);
    const float a2 = a * a;
    const float radius2 = xx * xx + yy * yy + zz * zz;
    const float sqsum = radius2 - a2;
    const float discr = sqrtf(sqsum * sqsum + 4.0f * a2 * zz * zz);
    const float rc = sqrtf(fmaxf(0.5f * (sqsum + discr), 1e-30f));
    const float cos_th = fminf(fmaxf(zz / fmaxf(rc, 1e-30f), -1.0f), 1.0f);
    const float sin_th = sqrtf(fmaxf(0.0f, 1.0f - cos_th * cos_th));
    const float sinth_f = fmaxf(sin_th, 1e-30f);
    const float denom = fmaxf(sinth_f * (rc * rc + a2), 1e-30f);
    float cphi = (rc * xx + a * yy) / denom;
    float sphi = (rc * yy - a * xx) / denom;
    const float inv_np = kp_rsqrtf(fmaxf(cphi * cphi + sphi * sphi, 1e-30f));
    cphi *= inv_np;
    sphi *= inv_np;
    const float r_bl = fmaxf(rc, float(c.min_radius));
    if (r_bl <= float(c.horizon + c.horizon_buffer) || r_bl < float(c.r_min) || r_bl > float(c.r_max)) return out;
    float ne_norm;
    {
        const float zc = r_bl * cos_th;
        const float rcyl = fmaxf(r_bl * sin_th, float(c.min_radius));
        const float h = fmaxf(float(c.disk_h), 1e-6f);
        const float vertical = expf(-(zc * zc) / (2.0f * rcyl * rcyl * h * h));
        ne_norm = float(c.nth0) * vertical * powf(fmaxf(r_bl, float(c.min_radius)), float(c.pow_nth));
    }
    if (!(ne_norm > 0.0f)) return out;
    out.emitting = 1;
    out.ne = ne_norm * float(c.ne_unit);
    out.thetae = fmaxf(float(c.Te0) * powf(fmaxf(r_bl, float(c.min_radius)), float(c.pow_T)) * float(c.thetae_unit),
                       float(c.min_thetae));
    {
        // B = sqrt(8 pi eps n_e m_p c^2 / (6 r)), eps = 0.1 (riaf.hpp:87-96)
        const float k = float(8.0 * 3.141592653589793 * 0.1 * f32c::kMP * f32c::kCL * f32c::kCL / 6.0);
        out.b = fmaxf(sqrtf(fmaxf(k * out.ne / fmaxf(r_bl, float(c.min_radius)), 0.0f)), 1e-12f);
    }
    // Kerr-Schild metric at the sample point
    float g[4][4];
    {
        const float z = zz;
        const float r2 = rc * rc;
        const float dn = r2 * r2 + a2 * z * z;
        const float amp = 2.0f * float(c.mass) * r2 * rc / dn;
        const float r2pa2 = r2 + a2;
        const float l[4] = {1.0f, (rc * xx + a * yy) / r2pa2, (rc * yy - a * xx) / r2pa2, z / rc};
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu) {
                const float eta = mu != nu ? 0.0f : (mu == 0 ? -1.0f : 1.0f);
                g[mu][nu] = eta + amp * l[mu] * l[nu];
            }
    }
    float ucon[4];
    {
        const float r = r_bl;
        float gcov[4][4], gcon[4][4];
        bl_metric_f(r, sin_th, cos_th, a, gcov, gcon);
        float vt = 1.0f, vr = 0.0f, vphi = 0.0f;
        const float kf = float(c.keplerian_factor), inf = float(c.infall_factor);
        if (r < float(c.horizon)) {
            vt = kp_rsqrtf(fmaxf(-gcon[0][0], 1e-30f));
        } else if (r < float(c.isco)) {
            float gi[4][4], gci[4][4];
            const float risco = float(c.isco);
            bl_metric_f(risco, sin_th, cos_th, a, gi, gci);
            const float omega_isco = 1.0f / (risco * sqrtf(risco) + a);
            const float qi = gi[0][0] + 2.0f * omega_isco * gi[0][3] + omega_isco * omega_isco * gi[3][3];
            const float ut_i = kp_rsqrtf(fmaxf(-qi, 1e-30f));
            const float e = (gi[0][0] + gi[0][3] * omega_isco) * ut_i;
            const float l = (gi[3][0] + gi[3][3] * omega_isco) * ut_i;
            const float k_con = gcon[0][0] * e * e + 2.0f * gcon[0][3] * e * l + gcon[3][3] * l * l;
            const float ur_cov = -sqrtf(fmaxf(-(1.0f + k_con) / fmaxf(gcon[1][1], 1e-30f), 0.0f));
            const float vr_tmp = gcon[1][1] * ur_cov;
            const float vt_tmp = gcon[0][0] * e + gcon[0][3] * l;
            const float vphi_tmp = gcon[3][0] * e + gcon[3][3] * l;
            const float omega_k = vphi_tmp / fmaxf(vt_tmp, 1e-30f);
            const float g00 = gcon[0][0];
            const float omega_ff = gcon[0][3] / (fabsf(g00) > 1e-30f ? g00 : (g00 < 0.0f ? -1e-30f : 1e-30f));
            const float omega = omega_k + (1.0f - kf) * (omega_ff - omega_k);
            const float ur_ff = -sqrtf(fmaxf(-(1.0f + gcon[0][0]) * gcon[1][1], 0.0f));
            vr = vr_tmp + inf * (ur_ff - vr_tmp);
            const float q = gcov[0][0] + 2.0f * omega * gcov[0][3] + omega * omega * gcov[3][3];
            vt = sqrtf(fmaxf(-(1.0f + vr * vr * gcov[1][1]) / q, 0.0f));
            vphi = omega * vt;
        } else {
            const float r_eff = fmaxf(r, float(c.min_radius));
            const float omega_k = 1.0f / (r_eff * sqrtf(r_eff) + a);
            const float g00 = gcon[0][0];
            const float omega_ff = gcon[0][3] / (fabsf(g00) > 1e-30f ? g00 : (g00 < 0.0f ? -1e-30f : 1e-30f));
            const float omega = omega_k + (1.0f - kf) * (omega_ff - omega_k);
            vr = inf * -sqrtf(fmaxf(-(1.0f + gcon[0][0]) * gcon[1][1], 0.0f));
            const float q = gcov[0][0] + 2.0f * omega * gcov[0][3] + omega * omega * gcov[3][3];
            vt = sqrtf(fmaxf(-(1.0f + vr * vr * gcov[1][1]) / q, 0.0f));
            vphi = omega * vt;
        }
        bl_to_cks_f(vt, vr, vphi, r, sin_th, cos_th, cphi, sphi, a, ucon);
        const float n2 = dot_gf(g, ucon, ucon);
        if (n2 < 0.0f) {
            const float sc = kp_rsqrtf(fmaxf(-n2, 1e-30f));
            for (int i = 0; i < 4; ++i) ucon[i] *= sc;
        }
    }
    float k[4], e1[4], e2[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        k[i] = float(s.k.v[i]);
        e1[i] = float(s.e1.v[i]);
        e2[i] = float(s.e2.v[i]);
    }
    const float uk = dot_gf(g, ucon, k);
    out.nu_fluid = fmaxf(fabsf(uk), float(c.min_frequency_scale));
    // toroidal field unit vector at the raw radius
    float bcon[4];
    {
        float bt[4];
        bl_to_cks_f(0.0f, 0.0f, 1.0f, rc, sin_th, cos_th, cphi, sphi, a, bt);
        float ub = dot_gf(g, ucon, bt);
        for (int i = 0; i < 4; ++i) bcon[i] = bt[i] + ucon[i] * ub;
        float bsq = dot_gf(g, bcon, bcon);
        if (!(bsq > 1e-30f)) {
            const float z4[4] = {0.0f, 0.0f, 0.0f, 1.0f};
            ub = dot_gf(g, ucon, z4);
            for (int i = 0; i < 4; ++i) bcon[i] = z4[i] + ucon[i] * ub;
            bsq = dot_gf(g, bcon, bcon);
        }
        if (!(bsq > 1e-30f)) {
            const float x4[4] = {0.0f, 1.0f, 0.0f, 0.0f};
            ub = dot_gf(g, ucon, x4);
            for (int i = 0; i < 4; ++i) bcon[i] = x4[i] + ucon[i] * ub;
            bsq = dot_gf(g, bcon, bcon);
        }
        if (bsq > 1e-30f) {
            const float sc = kp_rsqrtf(bsq);
            for (int i = 0; i < 4; ++i) bcon[i] *= sc;
        }
    }
    const float kdotb = dot_gf(g, k, bcon);
    out.cos_theta = fminf(fmaxf(kdotb / fmaxf(out.nu_fluid, 1e-30f), -1.0f), 1.0f);
    out.sin_theta = fmaxf(sqrtf(fmaxf(0.0f, 1.0f - out.cos_theta * out.cos_theta)), float(c.min_sin_theta));
    out.theta = acosf(out.cos_theta);
    riaf_sample_thermal_f(c, out);
    if (out.theta <= 0.0f || out.theta >= f32c::kPi) {
        out.on_axis = 1;
        return out;
    }
    // screen projections of b (riaf.hpp:320-336)
    const float eK_s = -1.0f / uk;
    float eK[4];
    for (int i = 0; i < 4; ++i) eK[i] = k[i] * eK_s - ucon[i];
    const bool degenerate = fabsf(uk) <= 1e-30f;
    const float ub_ = dot_gf(g, ucon, bcon), kb_ = dot_gf(g, eK, bcon);
    const float b1 = dot_gf(g, e1, bcon) + (degenerate ? 0.0f : dot_gf(g, ucon, e1) * ub_ - dot_gf(g, eK, e1) * kb_);
    const float b2 = dot_gf(g, e2, bcon) + (degenerate ? 0.0f : dot_gf(g, ucon, e2) * ub_ - dot_gf(g, eK, e2) * kb_);
    const float bproj2 = b1 * b1 + b2 * b2;
    if (bproj2 > 1e-30f) {
        out.has_chi = 1;
        out.cos2chi = (b2 * b2 - b1 * b1) / bproj2;
        out.sin2chi = -2.0f * b1 * b2 / bproj2;
    }
    return out;
}

// Thermal coefficients at one frequency, FP32, emission scaled by 2^E
// (`escale`).  nu_ghz = max(freq * nu_fluid, 1 Hz) in GHz.
KP_HD CoeffsF riaf_coefficients_f(const ImageConsts& c, const RiafSampleF& p, float freq_ghz,
                                                        float escale) {
    CoeffsF o = {};
    if (!p.emitting) return o;
    const float nu = fmaxf(freq_ghz * p.nu_fluid, 1e-9f);  // GHz
    const float ne = p.ne, te = p.thetae, b = p.b;
    const float st = fmaxf(p.sin_theta, float(c.min_sin_theta));
    const float ct = p.cos_theta;
    // Faraday rotation / conversion (symphony_rho_QV), invariant rho * nu
    float rQ, rV;
    {
        const float omega0 = f32c::kOmega0PerB * b;
        const float wp2 = f32c::kWp2PerNe * ne;
        const float two_pi_nu = 2.0f * f32c::kPi * nu * 1e9f;
        const float sst = p.on_axis ? fmaxf(sinf(p.theta), float(c.min_sin_theta)) : st;
        const float x = fmaxf(te * sqrtf(fmaxf(0.0f, 1.41421356f * sst * (1e3f * omega0 / two_pi_nu))), 1e-12f);
        const float inv_w = 1.0f / two_pi_nu;
        // eps12 = wp2 omega0 / (2 pi nu)^3 ; rho_V = 2 pi nu / c * eps12 ; inv = rho_V * nu
        const float shgm = 1.0f - 0.11f * logf(1.0f + 0.035f * x);
        const float cosv = p.on_axis ? cosf(p.theta) : ct;
        float e12 = wp2 * omega0 * inv_w;
        e12 *= inv_w;
        e12 *= inv_w;
        e12 *= p.r0 * shgm * cosv;
        rV = float(2.0 * 3.141592653589793 / f32c::kCL) * (nu * 1e9f) * e12 * (nu * 1e9f);
        if (p.on_axis) {
            o.rV = float(c.faraday_scale) * rV;
            return o;
        }
        // every power of x from one LG2; 0.5 + 0.5 tanh(z) = 1 / (1 + e^-2z)
        const float lx = log2f(x);
        const float exp_x_47 = expf(-x / 47.2f);
        const float z = (lx * 0.6931471805599453f - 4.787491742782046f) / 0.1f;
        const float sigm = 1.0f / (1.0f + expf(-2.0f * z));
        const float extraterm = (0.011f * exp_x_47 - 369.69342869090815f * pow2_of(-8.0f / 3.0f, lx)) * sigm;
        // the cosine term is below 1e-13 of the sum beyond x = 40
        const float cterm = x < 40.0f ? cosf(x / 2.0f) * expf(-pow2_of(1.2f, lx) / 2.73f) : 0.0f;
        const float jffunc = 2.011f * expf(-pow2_of(1.035f, lx) / 4.7f) - cterm - 0.011f * exp_x_47 + extraterm;
        float e11 = jffunc * wp2 * omega0 * inv_w;
        e11 *= omega0 * inv_w;
        e11 *= inv_w;
        e11 *= inv_w;
        e11 *= (p.r1 + 6.0f * te) * st * st;
        rQ = float(3.141592653589793 / f32c::kCL) * (nu * 1e9f) * e11 * (nu * 1e9f);
    }
    // emissivities, scaled by 2^E / nu^2 (nu^2 in Hz^2)
    float jI, jQ, jV;
    const float inv_nu2 = escale / (nu * nu) * 1e-18f;  // 2^E / (nu_Hz^2)
    if (c.fit == 4) {
        const float nus = f32c::kDexNus * b * st * te * te + 1.0f / 1e9f * 1e9f;  // + 1 Hz
        const float xh = fmaxf(nu * 1e9f / fmaxf(nus, 1e-30f), 1e-30f);
        const float xm13 = 1.0f / cbrtf(xh);
        const float exps = expf(-1.8899f / xm13);
        const float pref = f32c::kDexPref * ne * (nu * 1e9f) / (te * te);
        jI = pref * (2.5651f * (1.0f + 1.92f * xm13 + 0.9977f * xm13 * xm13) * exps) * inv_nu2;
        jQ = pref * (2.5651f * (1.0f + 0.93193f * xm13 + 0.499873f * xm13 * xm13) * exps) * inv_nu2;
        const float iv = (1.81384f / xh + 3.42319f * xm13 * xm13 + 0.0292545f * kp_rsqrtf(xh) + 2.03773f * xm13) * exps;
        float cft = ct;
        if (fabsf(cft) < 1e-10f) cft = cft >= 0.0f ? 1e-10f : -1e-10f;
        const float tan_theta = st / cft;
        jV = f32c::kDexPrefV * ne * (nu * 1e9f) / (tan_theta * te * te * te) * iv * inv_nu2;
    } else {
        const float nu_c = f32c::kNuCPerB * b;
        const float nu_s = 2.0f / 9.0f * nu_c * st * te * te;
        const float x = fmaxf(nu * 1e9f / fmaxf(nu_s, 1e-30f), 1e-30f);
        const float pref = ne * f32c::kE2OverC * nu_c * f32c::kTerm1 * st;
        const float lx = log2f(x);
        const float x13 = pow2_of(1.0f / 3.0f, lx);
        const float sqx = sqrtf(x), sqx13 = sqrtf(x13);
        const float ex13 = expf(-x13);
        const float sh = sqx + 1.8877486253633869933f * sqx13;
        jI = pref * (sh * sh) * ex13 * inv_nu2;
        const float shq = sqx + p.qterm * 1.8877486253633869933f * sqx13;
        jQ = pref * (shq * shq) * ex13 * inv_nu2;
        const float vt2 = pow2_of(5.0f / 3.0f, log2f(1.0f + p.vt2a * pow2_of(0.36f, lx)));
        jV = ne * f32c::kE2OverC * nu_c * p.vt1 * vt2 * ex13 * inv_nu2;
    }
    // polarisation cap (thermal_synchrotron.hpp:575-588)
    const float jps = fmaxf(fabsf(jQ), fabsf(jV));
    const float jP = jps > 0.0f ? jps * sqrtf((jQ / jps) * (jQ / jps) + (jV / jps) * (jV / jps)) : 0.0f;
    const float mpf = float(c.max_pol_frac);
    if (jI > 0.0f && jP > 0.0f && jI < jP / fmaxf(mpf, 1e-30f)) {
        const float sc = jI / jP * mpf;
        jQ *= sc;
        jV *= sc;
    }
    // Kirchhoff: a = j / B_nu, with B_nu = 2 h nu^3 / (c^2 (e^x - 1))
    float aI = 0.0f, aQ = 0.0f, aV = 0.0f;
    if (te > 0.0f) {
        const float xb = f32c::kHOverMc2GHz * nu / te;
        const float em1 = expm1f(xb);
        // j_inv / bnu_inv = j_phys / nu^2 * c^2 (e^x - 1) / (2 h) ; j here carries 2^E / nu^2
        const float fac = f32c::kC2Over2hGHz2 * em1 / escale * 1e18f;
        aI = jI * fac;
        aQ = jQ * fac;
        aV = jV * fac;
    }
    const float es = float(c.emission_scale), as = float(c.absorption_scale), fs = float(c.faraday_scale);
    o.jI = es * jI;
    o.jV = es * jV;
    o.aI = as * aI;
    o.aV = as * aV;
    o.rV = fs * rV;
    if (p.has_chi) {
        o.jQ = es * jQ * p.cos2chi;
        o.jU = es * jQ * p.sin2chi;
        o.aQ = as * aQ * p.cos2chi;
        o.aU = as * aQ * p.sin2chi;
        o.rQ = fs * rQ * p.cos2chi;
        o.rU = fs * rQ * p.sin2chi;
    }
    return o;
}

// ---- transfer -----------------------------------------------------------
KP_HD float atten_f(float kappa, float dl) {
    const float x = kappa * dl;
    if (x > 87.0f) return 0.0f;
    return expf(-x);
}

KP_HD float source_f(float kappa, float dl) {
    const float x = kappa * dl;
    if (fabsf(x) < 1e-3f) return dl * (1.0f - x * (0.5f - x * (1.0f / 6.0f - x * (1.0f / 24.0f))));
    return -expm1f(-x) / kappa;
}

// s = a + b with the rounding error accumulated into c (TwoSum).
KP_HD float two_sum_acc(float a, float b, float& c) {
    const float s = a + b;
    const float bb = s - a;
    c += (a - (s - bb)) + (b - bb);
    return s;
}

KP_HD void faraday_rotate_f(StokesF& s, const CoeffsF& c, float dl) {
    const float rn = sqrtf(c.rQ * c.rQ + c.rU * c.rU + c.rV * c.rV);
    if (rn == 0.0f || dl == 0.0f) return;
    // fold the compensation in before rotating
    const float px = s.Q + s.cQ, py = s.U + s.cU, pz = s.V + s.cV;
    s.cQ = s.cU = s.cV = 0.0f;
    const float theta = rn * dl;
    float ox, oy, oz;
    if (fabsf(theta) < 1e-4f) {
        ox = px + (c.rU * pz - c.rV * py) * dl;
        oy = py + (c.rV * px - c.rQ * pz) * dl;
        oz = pz + (c.rQ * py - c.rU * px) * dl;
    } else {
        const float inv = 1.0f / rn;
        const float nx = c.rQ * inv, ny = c.rU * inv, nz = c.rV * inv;
        // half-angle forms: 1 - cos(theta) = 2 sin^2(theta/2) keeps its
        // relative accuracy for small rotations
        float sh, ch;
        kp_sincos_small(0.5f * theta, &sh, &ch);
        const float st = 2.0f * sh * ch;
        const float omc = 2.0f * sh * sh;
        const float ct = 1.0f - omc;
        const float f = (nx * px + ny * py + nz * pz) * omc;
        ox = px * ct + nx * f + (ny * pz - nz * py) * st;
        oy = py * ct + ny * f + (nz * px - nx * pz) * st;
        oz = pz * ct + nz * f + (nx * py - ny * px) * st;
    }
    s.Q = ox;
    s.U = oy;
    s.V = oz;
}

KP_HD void absorb_emit_f(StokesF& s, const CoeffsF& c, float dl) {
    const float an = sqrtf(c.aQ * c.aQ + c.aU * c.aU + c.aV * c.aV);
    const float I = s.I + s.cI, Q = s.Q + s.cQ, U = s.U + s.cU, V = s.V + s.cV;
    if (an < 1e-30f) {
        const float e = atten_f(c.aI, dl);
        const float f = source_f(c.aI, dl);
        float ci = 0.f, cq = 0.f, cu = 0.f, cv = 0.f;
        s.I = two_sum_acc(e * I, f * c.jI, ci);
        s.Q = two_sum_acc(e * Q, f * c.jQ, cq);
        s.U = two_sum_acc(e * U, f * c.jU, cu);
        s.V = two_sum_acc(e * V, f * c.jV, cv);
        s.cI = ci;
        s.cQ = cq;
        s.cU = cu;
        s.cV = cv;
        return;
    }
    const float inv = 1.0f / an;
    const float nx = c.aQ * inv, ny = c.aU * inv, nz = c.aV * inv;
    const float p_par = nx * Q + ny * U + nz * V;
    const float j_par = nx * c.jQ + ny * c.jU + nz * c.jV;
    const float ppx = Q - nx * p_par, ppy = U - ny * p_par, ppz = V - nz * p_par;
    const float jpx = c.jQ - nx * j_par, jpy = c.jU - ny * j_par, jpz = c.jV - nz * j_par;
    const float kp = c.aI + an, km = c.aI - an;
    float csp = 0.f, csm = 0.f;
    const float sp = two_sum_acc(atten_f(kp, dl) * (I + p_par), source_f(kp, dl) * (c.jI + j_par), csp);
    const float sm = two_sum_acc(atten_f(km, dl) * (I - p_par), source_f(km, dl) * (c.jI - j_par), csm);
    const float ei = atten_f(c.aI, dl), fi = source_f(c.aI, dl);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    const float ox = two_sum_acc(ppx * ei, jpx * fi, cx);
    const float oy = two_sum_acc(ppy * ei, jpy * fi, cy);
    const float oz = two_sum_acc(ppz * ei, jpz * fi, cz);
    const float spc = sp + csp, smc = sm + csm;
    s.I = 0.5f * (spc + smc);
    const float par = 0.5f * (spc - smc);
    float c2x = 0.f, c2y = 0.f, c2z = 0.f;
    s.Q = two_sum_acc(nx * par, ox, c2x);
    s.U = two_sum_acc(ny * par, oy, c2y);
    s.V = two_sum_acc(nz * par, oz, c2z);
    s.cI = 0.0f;
    s.cQ = cx + c2x;
    s.cU = cy + c2y;
    s.cV = cz + c2z;
}

KP_HD void stokes_step_f(StokesF& s, const CoeffsF& c, float dl) {
    faraday_rotate_f(s, c, 0.5f * dl);
    absorb_emit_f(s, c, dl);
    faraday_rotate_f(s, c, 0.5f * dl);
}

}  // namespace kp
