// Host build of the mixed path's FP32 thermal-synchrotron fits
// (kpolaris_b200/csrc/kp_radiation_f32.cuh), for tests/test_mixed_coefficients.py.
// Reads lines "fit nu ne thetae b theta sin cos" on stdin and prints the
// unscaled invariant coefficients jI jQ jV aI aQ aV rQ rV (magnetic basis).
#include <cmath>
#include <cstdio>
#include <cstring>
#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__
#include "kp_radiation_f32.cuh"

int main() {
    int fit;
    double nu, ne, te, b, th, s, c;
    while (std::scanf("%d %lf %lf %lf %lf %lf %lf %lf", &fit, &nu, &ne, &te, &b, &th, &s, &c) == 8) {
        kp::ImageConsts k;
        std::memset(&k, 0, sizeof(k));
        k.fit = fit;
        k.min_sin_theta = 1e-4;
        k.max_pol_frac = 0.99;
        k.emission_scale = k.absorption_scale = k.faraday_scale = 1.0;
        kp::RiafSampleF p;
        std::memset(&p, 0, sizeof(p));
        p.emitting = 1;
        p.ne = float(ne);
        p.thetae = float(te);
        p.b = float(b);
        p.nu_fluid = 1.0f;
        p.theta = float(th);
        p.sin_theta = float(s);
        p.cos_theta = float(c);
        p.has_chi = 1;
        p.cos2chi = 1.0f;
        p.sin2chi = 0.0f;
        kp::riaf_sample_thermal_f(k, p);
        // scale the emission into FP32 range and undo it in double
        const double j0 = ne * 2.3e-19 * 2.8e6 * b / 3e10 / (nu * nu);
        const int e = int(std::floor(std::log2(1.0 / std::max(j0, 1e-300))));
        const float escale = std::ldexp(1.0f, std::max(-120, std::min(120, e)));
        const kp::CoeffsF o = kp::riaf_coefficients_f(k, p, float(nu * 1e-9), escale);
        const double inv = 1.0 / double(escale);
        std::printf("%.9e %.9e %.9e %.9e %.9e %.9e %.9e %.9e\n", o.jI * inv, o.jQ * inv, o.jV * inv, double(o.aI),
                    double(o.aQ), double(o.aV), double(o.rQ), double(o.rV));
    }
    return 0;
}
