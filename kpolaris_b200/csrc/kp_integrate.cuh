// kp_integrate.cuh -- geodesic integrators: classical RK4, step-doubling RK4
// with the reference's step control, and the Cash-Karp 5(4) embedded pair.
//
// RK4 keeps a running accumulator acc = ((k1 + 2 k2) + 2 k3) + k4, which is
// the reference's summation order (src/geodesic/rk4.hpp:36-46) with only two
// 16-double stage buffers live instead of four.
#pragma once

#include "kp_geometry.cuh"

namespace kp {

KP_HD void ray_axpy(Ray& out, const Ray& y, double a, const Ray& x) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        out.x.v[i] = y.x.v[i] + x.x.v[i] * a;
        out.k.v[i] = y.k.v[i] + x.k.v[i] * a;
        out.e1.v[i] = y.e1.v[i] + x.e1.v[i] * a;
        out.e2.v[i] = y.e2.v[i] + x.e2.v[i] * a;
    }
}

// acc = acc + x * a
KP_HD void ray_acc(Ray& acc, const Ray& x, double a) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        acc.x.v[i] = acc.x.v[i] + x.x.v[i] * a;
        acc.k.v[i] = acc.k.v[i] + x.k.v[i] * a;
        acc.e1.v[i] = acc.e1.v[i] + x.e1.v[i] * a;
        acc.e2.v[i] = acc.e2.v[i] + x.e2.v[i] * a;
    }
}

// acc = acc + x
KP_HD void ray_add(Ray& acc, const Ray& x) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        acc.x.v[i] = acc.x.v[i] + x.x.v[i];
        acc.k.v[i] = acc.k.v[i] + x.k.v[i];
        acc.e1.v[i] = acc.e1.v[i] + x.e1.v[i];
        acc.e2.v[i] = acc.e2.v[i] + x.e2.v[i];
    }
}

// rk4_step_from_k1 (rk4.hpp:49-59).  Out of line: one copy of the three
// inlined right-hand sides serves every RK4 call site.
static __device__ __noinline__ Ray rk4_from_k1(double mass, double spin, const Ray& s, double h, const Ray& k1) {
    Ray acc = k1;
    Ray tmp;
    const double hh = 0.5 * h;
    ray_axpy(tmp, s, hh, k1);
    Ray k = ks_rhs(mass, spin, tmp);  // k2
    ray_acc(acc, k, 2.0);
    ray_axpy(tmp, s, hh, k);
    k = ks_rhs(mass, spin, tmp);  // k3
    ray_acc(acc, k, 2.0);
    ray_axpy(tmp, s, h, k);
    k = ks_rhs(mass, spin, tmp);  // k4
    ray_add(acc, k);
    Ray out;
    ray_axpy(out, s, h / 6.0, acc);
    return out;
}

// rk4_step (rk4.hpp:36-46)
__device__ __forceinline__ Ray rk4_step(double mass, double spin, const Ray& s, double h) {
    const Ray k1 = ks_rhs(mass, spin, s);
    return rk4_from_k1(mass, spin, s, h, k1);
}

// state_error_norm (rk4.hpp:75-90): max over mu of |a-b| / max(1, |a|, |b|),
// components visited in the reference's order (x, k, e1, e2 per mu).
KP_HD double state_error_norm(const Ray& a, const Ray& b) {
    double err = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const double sx = max_val(1.0, max_val(abs_val(a.x.v[mu]), abs_val(b.x.v[mu])));
        const double sk = max_val(1.0, max_val(abs_val(a.k.v[mu]), abs_val(b.k.v[mu])));
        const double s1 = max_val(1.0, max_val(abs_val(a.e1.v[mu]), abs_val(b.e1.v[mu])));
        const double s2 = max_val(1.0, max_val(abs_val(a.e2.v[mu]), abs_val(b.e2.v[mu])));
        err = max_val(err, abs_val(a.x.v[mu] - b.x.v[mu]) / sx);
        err = max_val(err, abs_val(a.k.v[mu] - b.k.v[mu]) / sk);
        err = max_val(err, abs_val(a.e1.v[mu] - b.e1.v[mu]) / s1);
        err = max_val(err, abs_val(a.e2.v[mu] - b.e2.v[mu]) / s2);
    }
    return err;
}

// The error the step control acts on.  The control needs the norm exactly
// only above tol/64: at or below it the attempt is accepted and the growth
// factor 0.9 (tol/err)^0.2 >= 2.07 clamps to 2 (rk4.hpp:130-142).  Every
// scale of the norm is >= 1, so max |a - b| bounds it from above; when that
// bound is at most tol/64 it stands in for the norm with the same accept
// decision and the same next step, and the sixteen divisions are skipped.
// A NaN difference fails the comparison and takes the exact norm.
KP_HD double control_error(const Ray& a, const Ray& b, double tol) {
    const double lim = tol * (1.0 / 64.0);
    bool small = true;
    double m = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const double d[4] = {abs_val(a.x.v[mu] - b.x.v[mu]), abs_val(a.k.v[mu] - b.k.v[mu]),
                             abs_val(a.e1.v[mu] - b.e1.v[mu]), abs_val(a.e2.v[mu] - b.e2.v[mu])};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            small = small && d[i] <= lim;
            m = max_val(m, d[i]);
        }
    }
    return small ? m : state_error_norm(a, b);
}

struct StepControl {
    double tolerance, min_step, max_step;
};

struct AdaptiveStep {
    Ray state;
    Ray mid_state;
    double used_h;
    double next_h;
    int accepted;
};

// adaptive_rk4_step (rk4.hpp:108-161): one full step against two half steps,
// at most 10 attempts.  The half-step state is the transfer sample point.
static __device__ __noinline__ void adaptive_rk4(double mass, double spin, const Ray& state,
                                             double requested_h, const StepControl& ctl,
                                             AdaptiveStep& out) {
    double h = min_val(max_val(abs_val(requested_h), ctl.min_step), ctl.max_step);
    if (requested_h < 0.0) h = -h;
    const double tol = max_val(ctl.tolerance, kTolFloor);
#pragma unroll 1
    for (int attempt = 0; attempt < 10; ++attempt) {
        const Ray k1 = ks_rhs(mass, spin, state);
        const Ray half = rk4_from_k1(mass, spin, state, h * 0.5, k1);
        const Ray two_half = rk4_step(mass, spin, half, h * 0.5);
        const Ray full = rk4_from_k1(mass, spin, state, h, k1);
        const double err = state_error_norm(full, two_half);
        if (err <= tol) {
            double factor = 2.0;
            if (err > 0.0) {
                factor = 0.9 * pow(tol / err, 0.2);
                factor = min_val(2.0, max_val(0.2, factor));
            }
            out.state = two_half;
            out.mid_state = half;
            out.used_h = h;
            out.next_h = min_val(ctl.max_step, max_val(ctl.min_step, abs_val(h) * factor));
            if (requested_h < 0.0) out.next_h = -out.next_h;
            out.accepted = 1;
            return;
        }
        if (abs_val(h) <= ctl.min_step * 1.0001) break;
        double factor = 0.9 * pow(tol / max_val(err, kTiny), 0.25);
        factor = min_val(0.8, max_val(0.1, factor));
        h *= factor;
    }
    const double next_abs = max_val(ctl.min_step, abs_val(h) * 0.5);
    out.state = state;
    out.mid_state = state;
    out.used_h = 0.0;
    out.next_h = requested_h < 0.0 ? -next_abs : next_abs;
    out.accepted = 0;
}

// s + (sum_i k_i c_i) * h, summed left to right (rk4.hpp:181-213).
template<int N>
KP_HD void ray_lincomb(Ray& out, const Ray& s, double h, const Ray* const (&k)[N],
                       const double (&c)[N]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#define KP_LC(F)                                                   \
    {                                                              \
        double a = k[0]->F.v[i] * c[0];                            \
        for (int j = 1; j < N; ++j) a = a + k[j]->F.v[i] * c[j];   \
        out.F.v[i] = s.F.v[i] + a * h;                             \
    }
        KP_LC(x) KP_LC(k) KP_LC(e1) KP_LC(e2)
#undef KP_LC
    }
}

// adaptive_rkf45_endpoint_step (rk4.hpp:163-250): Cash-Karp 5(4), 6 RHS per
// attempt, the same acceptance rule with a 0.2 shrink exponent; the sample
// point is the accepted endpoint.  Not used by the reference's image tool;
// offered as an integrator variant.
static __device__ __noinline__ void adaptive_cash_karp(double mass, double spin, const Ray& state,
                                                   double requested_h, const StepControl& ctl,
                                                   AdaptiveStep& out) {
    double h = min_val(max_val(abs_val(requested_h), ctl.min_step), ctl.max_step);
    if (requested_h < 0.0) h = -h;
    const double tol = max_val(ctl.tolerance, kTolFloor);
#pragma unroll 1
    for (int attempt = 0; attempt < 10; ++attempt) {
        const Ray k1 = ks_rhs(mass, spin, state);
        Ray t;
        ray_axpy(t, state, h * 1.0 / 5.0, k1);
        const Ray k2 = ks_rhs(mass, spin, t);
        {
            const Ray* const kk[2] = {&k1, &k2};
            const double cc[2] = {3.0 / 40.0, 9.0 / 40.0};
            ray_lincomb<2>(t, state, h, kk, cc);
        }
        const Ray k3 = ks_rhs(mass, spin, t);
        {
            const Ray* const kk[3] = {&k1, &k2, &k3};
            const double cc[3] = {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0};
            ray_lincomb<3>(t, state, h, kk, cc);
        }
        const Ray k4 = ks_rhs(mass, spin, t);
        {
            const Ray* const kk[4] = {&k1, &k2, &k3, &k4};
            const double cc[4] = {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0};
            ray_lincomb<4>(t, state, h, kk, cc);
        }
        const Ray k5 = ks_rhs(mass, spin, t);
        {
            const Ray* const kk[5] = {&k1, &k2, &k3, &k4, &k5};
            const double cc[5] = {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0,
                                  44275.0 / 110592.0, 253.0 / 4096.0};
            ray_lincomb<5>(t, state, h, kk, cc);
        }
        const Ray k6 = ks_rhs(mass, spin, t);
        Ray fifth, fourth;
        {
            const Ray* const kk[4] = {&k1, &k3, &k4, &k6};
            const double cc[4] = {37.0 / 378.0, 250.0 / 621.0, 125.0 / 594.0, 512.0 / 1771.0};
            ray_lincomb<4>(fifth, state, h, kk, cc);
        }
        {
            const Ray* const kk[5] = {&k1, &k3, &k4, &k5, &k6};
            const double cc[5] = {2825.0 / 27648.0, 18575.0 / 48384.0, 13525.0 / 55296.0,
                                  277.0 / 14336.0, 1.0 / 4.0};
            ray_lincomb<5>(fourth, state, h, kk, cc);
        }
        const double err = state_error_norm(fifth, fourth);
        if (err <= tol) {
            double factor = 2.0;
            if (err > 0.0) {
                factor = 0.9 * pow(tol / err, 0.2);
                factor = min_val(2.0, max_val(0.2, factor));
            }
            out.state = fifth;
            out.mid_state = fifth;
            out.used_h = h;
            out.next_h = min_val(ctl.max_step, max_val(ctl.min_step, abs_val(h) * factor));
            if (requested_h < 0.0) out.next_h = -out.next_h;
            out.accepted = 1;
            return;
        }
        if (abs_val(h) <= ctl.min_step * 1.0001) break;
        double factor = 0.9 * pow(tol / max_val(err, kTiny), 0.2);
        factor = min_val(0.8, max_val(0.1, factor));
        h *= factor;
    }
    const double next_abs = max_val(ctl.min_step, abs_val(h) * 0.5);
    out.state = state;
    out.mid_state = state;
    out.used_h = 0.0;
    out.next_h = requested_h < 0.0 ? -next_abs : next_abs;
    out.accepted = 0;
}

__device__ __forceinline__ void adaptive_step(int integrator, double mass, double spin,
                                              const Ray& state, double requested_h,
                                              const StepControl& ctl, AdaptiveStep& out) {
    if (integrator == 1) {
        adaptive_cash_karp(mass, spin, state, requested_h, ctl, out);
    } else {
        adaptive_rk4(mass, spin, state, requested_h, ctl, out);
    }
}

}  // namespace kp
