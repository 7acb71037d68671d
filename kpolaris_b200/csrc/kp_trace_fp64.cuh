// kp_trace_fp64.cuh -- one ray, FP64: backward pass A from the camera to the
// radiating-sphere endpoint, then forward pass B with NF Stokes channels
// sharing the geodesic, then the observer-basis transform.
//
// Restates the fused per-pixel kernels trace_pass_b_segment_model_pixel_metric
// (src/geodesic/pass_b.hpp:769-1114) and its multi-frequency twin
// (pass_b.hpp:1131-1501) for the Kerr metric in Cartesian KS: the metric has
// no time domain, no excision hook and no effective-min-step hook, so those
// calls reduce to identities (src/geodesic/metric_domain.hpp:78-225).  The
// surface-crossing refinement restates locate_metric_surface_crossing
// (src/geodesic/pass_a_core.hpp:94-197).
#pragma once

#include "kp_camera.cuh"
#include "kp_integrate.cuh"
#include "kp_radiation.cuh"

namespace kp {

__device__ __forceinline__ int finite_ray(const Ray& s) {
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const double v[4] = {s.x.v[mu], s.k.v[mu], s.e1.v[mu], s.e2.v[mu]};
#pragma unroll
        for (int f = 0; f < 4; ++f)
            if (!(v[f] == v[f]) || abs_val(v[f]) >= kLarge) return 0;
    }
    return 1;
}

// metric_surface_path_state (pass_a_core.hpp:76-87)
__device__ __forceinline__ Ray surface_path_state(double mass, double spin, const Ray& first,
                                                  double h, int composed) {
    if (composed) {
        const Ray half = rk4_step(mass, spin, first, h * 0.5);
        return rk4_step(mass, spin, half, h * 0.5);
    }
    return rk4_step(mass, spin, first, h);
}

// locate_metric_surface_crossing (pass_a_core.hpp:94-197) for the spherical
// surfaces r = surface_parameter; returns the last point on the original side.
static __device__ __noinline__ void locate_crossing(double mass, double spin, const Ray& first,
                                             const Ray& second, double full_h,
                                             double surface_parameter, int composed,
                                             Ray& out_state, double& out_h) {
    out_state = first;
    out_h = 0.0;
    double lo = 0.0, hi = 1.0;
    double flo = ks_radius(spin, first.x) - surface_parameter;
    if (flo == 0.0) return;
    if (!finite_ray(second)) return;
    const Ray hs = surface_path_state(mass, spin, first, full_h, composed);
    if (!finite_ray(hs)) return;
    double fhi = ks_radius(spin, hs.x) - surface_parameter;
    if (!(fhi == fhi) || abs_val(fhi) >= kLarge) return;
    if (fhi == 0.0) {
        out_state = hs;
        out_h = full_h;
        return;
    }
    if ((flo > 0.0) == (fhi > 0.0)) return;
    int use_secant = 1;
#pragma unroll 1
    for (int iter = 0; iter < 12; ++iter) {
        const double width = hi - lo;
        double trial = (lo + hi) * 0.5;
        const double denom = flo - fhi;
        if (use_secant && abs_val(denom) > kTiny) {
            const double secant = lo + width * flo / denom;
            const double guard = width * 0.1;
            if (secant > lo + guard && secant < hi - guard) trial = secant;
        }
        const Ray ts = surface_path_state(mass, spin, first, full_h * trial, composed);
        if (!finite_ray(ts)) {
            hi = trial;
            use_secant = 0;
            continue;
        }
        const double ft = ks_radius(spin, ts.x) - surface_parameter;
        if (!(ft == ft) || abs_val(ft) >= kLarge) {
            hi = trial;
            use_secant = 0;
            continue;
        }
        if (ft == 0.0) {
            out_state = ts;
            out_h = full_h * trial;
            return;
        }
        if ((flo > 0.0) == (ft > 0.0)) {
            lo = trial;
            flo = ft;
            out_state = ts;
            out_h = full_h * trial;
        } else {
            hi = trial;
            fhi = ft;
        }
    }
}

__device__ __forceinline__ double max_frame_error(double mass, double spin, const Ray& s) {
    const KSMetricPoint w = ks_point(mass, spin, s.x);
    double o = abs_val(ks_dot_at(w, s.k, s.k));
    o = max_val(o, abs_val(ks_dot_at(w, s.e1, s.k)));
    o = max_val(o, abs_val(ks_dot_at(w, s.e2, s.k)));
    o = max_val(o, abs_val(ks_dot_at(w, s.e1, s.e1) - 1.0));
    o = max_val(o, abs_val(ks_dot_at(w, s.e2, s.e2) - 1.0));
    o = max_val(o, abs_val(ks_dot_at(w, s.e1, s.e2)));
    return o;
}

__device__ __forceinline__ double spatial_distance(const D4& a, const D4& b) {
    return sqrt(sq(a.v[1] - b.v[1]) + sq(a.v[2] - b.v[2]) + sq(a.v[3] - b.v[3]));
}

__device__ __forceinline__ double vmaxabsdiff(const D4& a, const D4& b) {
    double o = abs_val(a.v[0] - b.v[0]);
    for (int i = 1; i < 4; ++i) o = max_val(o, abs_val(a.v[i] - b.v[i]));
    return o;
}

// radiation_substep_count (pass_b.hpp:147-179) with requested_substeps = 1.
// nsub is a power of two, so q / nsub > lim is exactly q > lim * nsub (both
// sides are exact scalings): the doubling loops compare against lim * nsub
// instead of dividing, with the reference's outcomes.
template<class C>
__device__ __forceinline__ int radiation_substep_count(const C& co, double h, double dls,
                                                       double max_rad_step, double max_rad_depth,
                                                       double max_abs_depth, double max_far_depth) {
    int nsub = 1;
    const double abs_h = abs_val(h);
    if (max_rad_step > 0.0)
        while (abs_h > max_rad_step * double(nsub) && nsub < 4096) nsub *= 2;
    const double dl = abs_h * abs_val(dls);
    const double alim = max_abs_depth >= 0.0 ? max_abs_depth : max_rad_depth;
    if (alim > 0.0) {
        const double aQ = co.aQ, aU = co.aU, aV = co.aV;
        const double depth = (abs_val(double(co.aI)) + sqrt(aQ * aQ + aU * aU + aV * aV)) * dl;
        while (depth > alim * double(nsub) && nsub < 4096) nsub *= 2;
    }
    const double flim = max_far_depth >= 0.0 ? max_far_depth : max_rad_depth;
    if (flim > 0.0) {
        const double rQ = co.rQ, rU = co.rU, rV = co.rV;
        const double depth = sqrt(rQ * rQ + rU * rU + rV * rV) * dl;
        while (depth > flim * double(nsub) && nsub < 4096) nsub *= 2;
    }
    return nsub;
}

struct PixelOut {
    double r11, r12, r21, r22;
    double closure_x, closure_k, final_null, frame_error;
    int pass_a_steps, steps, reason;
};

// Pass A (pass_b.hpp:786-938).  Returns 1 when the endpoint is valid for
// pass B (entered the radiating sphere and ended on its inner or outer surface).
__device__ __forceinline__ int trace_pass_a(const ImageConsts& c, Ray& state, int& pa_steps,
                                            int& pa_reason) {
    const double mass = c.mass, spin = c.spin;
    pa_reason = kMaxSteps;
    pa_steps = 0;
    StepControl ctl;
    ctl.tolerance = c.tolerance;
    ctl.min_step = c.min_step_abs;
    ctl.max_step = c.max_step;
    double h_current = -abs_val(c.step);
    int entered = 0;
    int inside = 0;
#pragma unroll 1
    for (int n = 0; n < c.max_steps; ++n) {
        const double r_bl = ks_radius(spin, state.x);
        if (!entered) {
            if (r_bl <= c.outer_radius) {
                entered = 1;
                inside = 0;
            }
        } else {
            if (r_bl - c.inner_radius <= 0.0) {
                pa_reason = kReachedInner;
                break;
            }
            if (inside > 0 && r_bl >= c.outer_radius) {
                pa_reason = kEscaped;
                break;
            }
        }
        const double old_r = r_bl;
        const double old_inner = r_bl - c.inner_radius;
        double used_h = h_current;
        Ray next;
        if (c.adaptive) {
            StepControl tc = ctl;
            if (abs_val(used_h) < tc.min_step) tc.min_step = abs_val(used_h);
            AdaptiveStep st;
            adaptive_step(c.integrator, mass, spin, state, used_h, tc, st);
            if (!st.accepted) {
                h_current = st.next_h;
                if (abs_val(h_current) <= c.min_step_abs * 1.0001) {
                    pa_reason = kAdaptiveUnderflow;
                    break;
                }
                continue;
            }
            next = st.state;
            used_h = st.used_h;
            h_current = st.next_h;
        } else {
            next = rk4_step(mass, spin, state, used_h);
        }
        const double next_r = ks_radius(spin, next.x);
        const double next_inner = next_r - c.inner_radius;
        if (!entered && next_r <= c.outer_radius) {
            entered = 1;
            inside = 0;
        } else if (!entered && next_r >= old_r) {
            state = next;
            pa_steps += 1;
            pa_reason = kEscaped;
            break;
        }
        int crossing = kNone;
        if (entered && old_inner > 0.0 && next_inner <= 0.0) {
            crossing = kReachedInner;
        } else if (entered && inside > 0 && old_r < c.outer_radius && next_r >= c.outer_radius) {
            crossing = kEscaped;
        }
        if (crossing != kNone) {
            const double sp = crossing == kReachedInner ? c.inner_radius : c.outer_radius;
            Ray ev;
            double ev_h;
            locate_crossing(mass, spin, state, next, used_h, sp, c.adaptive, ev, ev_h);
            state = ev;
            pa_steps += 1;
            pa_reason = crossing;
            break;
        }
        state = next;
        pa_steps += 1;
        if (entered) inside += 1;
    }
    return entered && (pa_reason == kReachedInner || pa_reason == kEscaped);
}

// Pass B (pass_b.hpp:940-1114 / :1312-1501) with NF channels, FP64 transfer.
template<int NF>
__device__ __forceinline__ void trace_pass_b_fp64(const ImageConsts& c, Ray& state,
                                                  Stokes4<double> (&stokes)[NF], int& steps,
                                                  int& reason) {
    const double mass = c.mass, spin = c.spin;
    StepControl ctl;
    ctl.tolerance = c.tolerance;
    ctl.min_step = c.min_step_abs;
    ctl.max_step = c.max_step;
#pragma unroll
    for (int f = 0; f < NF; ++f) stokes[f] = Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    int reached = 0;
    steps = 0;
    double h_current = c.step;
    double cap = c.max_radiation_step > 0.0 ? c.max_radiation_step : c.max_step;
    const double eff_min = c.min_step_abs;
#pragma unroll 1
    while (!reached && steps < c.max_steps) {
        double h = h_current;
        const Ray old = state;
        const double start_r = ks_radius(spin, old.x);
        if (start_r <= c.outer_radius && cap > 0.0) h = min_val(h, cap);
        Ray next, sample;
        if (c.adaptive) {
            AdaptiveStep st;
            adaptive_step(c.integrator, mass, spin, old, h, ctl, st);
            if (!st.accepted) {
                h_current = abs_val(st.next_h);
                if (h_current <= eff_min * 1.0001) {
                    reason = kAdaptiveUnderflow;
                    break;
                }
                continue;
            }
            h = abs_val(st.used_h);
            h_current = abs_val(st.next_h);
            next = st.state;
            sample = st.mid_state;
        } else {
            next = rk4_step(mass, spin, old, h);
            sample = next;
        }
        const double old_r = start_r;
        const double s0 = old_r - c.cam_radius;
        const double s1 = ks_radius(spin, next.x) - c.cam_radius;
        const int crosses = (s0 == 0.0 || s1 == 0.0) ? 1 : ((s0 < 0.0 && s1 > 0.0) || (s0 > 0.0 && s1 < 0.0));
        if (crosses) {
            const double denom = s0 - s1;
            const double frac = abs_val(denom) <= kTiny ? 1.0 : min_val(1.0, max_val(0.0, s0 / denom));
            const double h_cross = h * frac;
            if (abs_val(h_cross) <= 1e-14) {
                h = 0.0;
                next = old;
                sample = old;
            } else if (frac < 0.999999999999) {
                h = h_cross;
                if (c.adaptive) {
                    StepControl cc = ctl;
                    cc.min_step = min_val(eff_min, abs_val(h));
                    cc.max_step = max_val(cc.min_step, abs_val(h));
                    AdaptiveStep cs;
                    adaptive_step(c.integrator, mass, spin, old, h, cc, cs);
                    if (!cs.accepted) {
                        h_current = abs_val(cs.next_h);
                        continue;
                    }
                    h = abs_val(cs.used_h);
                    next = cs.state;
                    sample = cs.mid_state;
                } else {
                    next = rk4_step(mass, spin, old, h);
                    sample = next;
                }
            }
        }
        const double sample_r = ks_radius(spin, sample.x);
        const double next_r = ks_radius(spin, next.x);
        const double local_max_rs =
            (c.max_radiation_step > 0.0 &&
             (old_r <= c.outer_radius || sample_r <= c.outer_radius || next_r <= c.outer_radius))
                ? c.max_radiation_step : 0.0;
        Coeffs<double> co[NF];
        const int inside = sample_r - c.inner_radius > 0.0 && sample_r < c.outer_radius;
        RiafSample ps;
        ps.emitting = 0;
        if (inside) ps = riaf_sample(c, sample);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            co[f] = riaf_coefficients(c, ps, c.freq[f]);
            if (!c.faraday_rotation) co[f].rV = 0.0;
        }
        // Substep counts at h (required) and at h_current (predictive) in
        // one pass: neither test changes h or h_current.  Over the image's
        // frequencies, or over a separate step-control list
        // (pass_b.hpp:1787-1833).
        int required = 1, pred = 1;
        if (c.nctl == 0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const int cand = radiation_substep_count(co[f], h, c.dlambda_scale[f], local_max_rs,
                                                         c.max_radiation_depth, c.max_absorption_depth,
                                                         c.max_faraday_depth);
                required = cand > required ? cand : required;
                const int pc = radiation_substep_count(co[f], h_current, c.dlambda_scale[f], local_max_rs,
                                                       c.max_radiation_depth, c.max_absorption_depth,
                                                       c.max_faraday_depth);
                pred = pc > pred ? pc : pred;
            }
        } else {
#pragma unroll 1
            for (int g = 0; g < c.nctl; ++g) {
                Coeffs<double> cg = riaf_coefficients(c, ps, c.ctl_freq[g]);
                if (!c.faraday_rotation) cg.rV = 0.0;
                const int cand = radiation_substep_count(cg, h, c.ctl_dlambda_scale[g], local_max_rs,
                                                         c.max_radiation_depth, c.max_absorption_depth,
                                                         c.max_faraday_depth);
                required = cand > required ? cand : required;
                const int pc = radiation_substep_count(cg, h_current, c.ctl_dlambda_scale[g], local_max_rs,
                                                       c.max_radiation_depth, c.max_absorption_depth,
                                                       c.max_faraday_depth);
                pred = pc > pred ? pc : pred;
            }
        }
        if (required > 1 && h > eff_min * 1.0001) {
            h_current = max_val(eff_min, h / double(required));
            cap = h_current;
            continue;
        }
        if (local_max_rs > 0.0 || c.max_radiation_depth > 0.0 || c.max_absorption_depth > 0.0 ||
            c.max_faraday_depth > 0.0) {
            cap = pred > 1 ? max_val(eff_min, h_current / double(pred)) : c.max_step;
        } else {
            cap = c.max_step;
        }
        if (h > 0.0) {
#pragma unroll
            for (int f = 0; f < NF; ++f) stokes_step(stokes[f], co[f], abs_val(h) * c.dlambda_scale[f]);
        }
        state = next;
        steps += 1;
        if (crosses) reached = 1;
    }
    if (reached) {
        reason = kReachedCamera;
    } else if (reason != kAdaptiveUnderflow) {
        reason = kMaxSteps;
    }
}

// Screen overlap, observer transform and closure diagnostics
// (pass_b.hpp:87-98, :1096-1113; stokes_rotation.hpp:39-57).
template<class R, int NF>
__device__ __forceinline__ void finish_ray(const ImageConsts& c, const Ray& cam, const Ray& state,
                                           int passed_b, Stokes4<R> (&stokes)[NF], PixelOut& o,
                                           double (&obs)[NF][4]) {
    const KSMetricPoint w = ks_point(c.mass, c.spin, state.x);
    if (passed_b) {
        o.r11 = ks_dot_at(w, cam.e1, state.e1);
        o.r12 = ks_dot_at(w, cam.e1, state.e2);
        o.r21 = ks_dot_at(w, cam.e2, state.e1);
        o.r22 = ks_dot_at(w, cam.e2, state.e2);
    } else {
        o.r11 = 1.0;
        o.r12 = 0.0;
        o.r21 = 0.0;
        o.r22 = 1.0;
    }
    const double r11 = o.r11, r12 = o.r12, r21 = o.r21, r22 = o.r22;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (passed_b) {
            const double I = stokes[f].I, Q = stokes[f].Q, U = stokes[f].U, V = stokes[f].V;
            obs[f][0] = I;
            obs[f][1] = 0.5 * Q * (r11 * r11 - r12 * r12 - r21 * r21 + r22 * r22) + U * (r11 * r12 - r21 * r22);
            obs[f][2] = Q * (r11 * r21 - r12 * r22) + U * (r11 * r22 + r12 * r21);
            obs[f][3] = (r11 * r22 - r12 * r21) * V;
        } else {
            obs[f][0] = obs[f][1] = obs[f][2] = obs[f][3] = 0.0;
        }
    }
    o.closure_x = spatial_distance(state.x, cam.x);
    o.closure_k = vmaxabsdiff(state.k, cam.k);
    o.final_null = ks_dot_at(w, state.k, state.k);
    o.frame_error = max_frame_error(c.mass, c.spin, state);
}

__device__ __forceinline__ void store_diagnostics(const ImageOutPtrs& out, int pixel, const PixelOut& o) {
    out.closure_x[pixel] = o.closure_x;
    out.closure_k[pixel] = o.closure_k;
    out.final_null[pixel] = o.final_null;
    out.frame_error[pixel] = o.frame_error;
    out.det_r[pixel] = o.r11 * o.r22 - o.r12 * o.r21;
    out.r11[pixel] = o.r11;
    out.r12[pixel] = o.r12;
    out.r21[pixel] = o.r21;
    out.r22[pixel] = o.r22;
    out.basis_identity_error[pixel] = max_val(max_val(abs_val(o.r11 - 1.0), abs_val(o.r22 - 1.0)),
                                              max_val(abs_val(o.r12), abs_val(o.r21)));
    out.basis_rotation_angle[pixel] = atan2(o.r21 - o.r12, o.r11 + o.r22);
    out.pass_a_steps[pixel] = o.pass_a_steps;
    out.steps[pixel] = o.steps;
    out.reason[pixel] = o.reason;
}

template<int NF>
__device__ __forceinline__ void store_stokes(const ImageOutPtrs& out, int pixel, int npix,
                                             const double (&obs)[NF][4]) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const size_t idx = size_t(f) * size_t(npix) + size_t(pixel);
        out.image_i[idx] = obs[f][0];
        out.image_q[idx] = obs[f][1];
        out.image_u[idx] = obs[f][2];
        out.image_v[idx] = obs[f][3];
    }
}

}  // namespace kp
