// kp_persistent.cuh -- the persistent image kernel: lanes claim rays from a
// global queue that spans every job of the launch, advance them one RK job
// per loop iteration through the pass-A / crossing / pass-B control machine,
// and write the finished pixel.  See kp_engine.cuh for the design.
#pragma once

#include "kp_engine.cuh"

namespace kp {

enum : int { kEndA = 7 };

struct LaneState {
    int job, pixel, mode, in_b;
    // adaptive attempt sequence (rk4.hpp:108-161)
    int attempt, rk_kind;
    double h_try, req_h, ctl_min, ctl_max;
    // pass A (pass_b.hpp:786-938)
    int n, entered, inside, pa_steps, reason;
    double h_current, old_r;
    // surface-crossing search (pass_a_core.hpp:94-197)
    int cross_reason, iter, use_secant;
    double lo, hi, flo, fhi, full_h, surf, trial;
    // pass B (pass_b.hpp:940-1114)
    int steps, reached;
    double cap, hB, start_r;
};

__device__ __forceinline__ void begin_adaptive(LaneState& L, double requested, double min_step,
                                               double max_step) {
    L.req_h = requested;
    L.ctl_min = min_step;
    L.ctl_max = max_step;
    double h = min_val(max_val(abs_val(requested), min_step), max_step);
    if (requested < 0.0) h = -h;
    L.h_try = h;
    L.attempt = 0;
}

// Step growth after an accepted attempt (rk4.hpp:130-142).
__device__ __forceinline__ double accepted_next_h(double h, double err, double tol, double min_step,
                                                  double max_step, double requested) {
    double factor = 2.0;
    if (err > 0.0) {
        factor = 0.9 * pow(tol / err, 0.2);
        factor = min_val(2.0, max_val(0.2, factor));
    }
    double next_h = min_val(max_step, max_val(min_step, abs_val(h) * factor));
    if (requested < 0.0) next_h = -next_h;
    return next_h;
}

// A rejected attempt: shrink and retry, or give up (rk4.hpp:143-160).
// Returns 1 when the sequence is exhausted; L.h_current then holds the
// signed next_h of the failed sequence.
__device__ __forceinline__ int rejected_attempt(LaneState& L, double err, double tol) {
    L.attempt += 1;
    int exhausted = L.attempt >= 10;
    if (abs_val(L.h_try) <= L.ctl_min * 1.0001) {
        exhausted = 1;
    } else {
        double factor = 0.9 * pow(tol / max_val(err, kTiny), L.rk_kind == kRkCK ? 0.2 : 0.25);
        factor = min_val(0.8, max_val(0.1, factor));
        L.h_try *= factor;
    }
    if (exhausted) {
        const double next_abs = max_val(L.ctl_min, abs_val(L.h_try) * 0.5);
        L.h_current = L.req_h < 0.0 ? -next_abs : next_abs;
    }
    return exhausted;
}

__device__ __forceinline__ void issue_step(LaneState& L, const ImageConsts& c, double h, double min_step,
                                           double max_step) {
    if (c.adaptive) {
        begin_adaptive(L, h, min_step, max_step);
        L.rk_kind = c.integrator == 1 ? kRkCK : kRkSD;
    } else {
        L.h_try = h;
        L.rk_kind = kRkRK4;
    }
}

template<int NF>
__device__ __forceinline__ void store_stokes_n(const ImageOutPtrs& out, int pixel, int npix, int nf,
                                               const double (&obs)[NF][4]) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        if (f < nf) {
            const size_t idx = size_t(f) * size_t(npix) + size_t(pixel);
            out.image_i[idx] = obs[f][0];
            out.image_q[idx] = obs[f][1];
            out.image_u[idx] = obs[f][2];
            out.image_v[idx] = obs[f][3];
        }
    }
}

template<class P, int NF>
__device__ __forceinline__ void persistent_body(const LaunchDesc& L) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    LaneState st;
    st.mode = kIdle;
    st.job = -1;
    st.rk_kind = -1;
    Ray S;
    Ray best;
    using RT = RadTraits<P>;
    typename RT::Stokes stokes[NF];
    int finished = 0;
    long long my_ray = -1;
    if (!L.refill) {
        my_ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (my_ray >= L.total_rays) finished = 1;
    }
    const JobDesc* J = nullptr;
    long long guard = 0;

#pragma unroll 1
    while (true) {
        // ------------------------------------------------------------ refill
        const bool want = !finished && st.mode == kIdle;
        if (L.refill) {
            const unsigned need = __ballot_sync(FULL, want);
            if (need) {
                unsigned long long base = 0;
                const int leader = __ffs(need) - 1;
                if (lane == leader) base = atomicAdd(L.next_ray, (unsigned long long)__popc(need));
                base = __shfl_sync(FULL, base, leader);
                if (want) {
                    my_ray = (long long)(base + __popc(need & ((1u << lane) - 1u)));
                    if (my_ray >= L.total_rays) finished = 1;
                }
            }
        }
        if (!finished && st.mode == kIdle) {
            int lo = 0, hi = L.njobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (L.jobs[mid].ray_begin <= my_ray) lo = mid; else hi = mid - 1;
            }
            st.job = lo;
            J = &L.jobs[lo];
            st.pixel = int(my_ray - J->ray_begin);
            S = camera_ray(J->c, J->frame, st.pixel);
            st.reason = kMaxSteps;
            st.pa_steps = 0;
            st.n = 0;
            st.entered = 0;
            st.inside = 0;
            st.in_b = 0;
            st.steps = 0;
            st.h_current = -abs_val(J->c.step);
            st.mode = kAStep;
            st.rk_kind = -1;
            guard = 0;
        }
        const bool active = !finished && st.mode != kIdle;
        if (!__any_sync(FULL, active)) break;

        // ---------------------------------------------- control before the job
        if (active && st.mode == kAStep && st.rk_kind < 0) {
            // pass-A loop top (pass_b.hpp:793-838)
            const ImageConsts& c = J->c;
            if (st.n >= c.max_steps) {
                st.mode = kEndA;
            } else {
                const double r_bl = ks_radius(c.spin, S.x);
                if (!st.entered) {
                    if (r_bl <= c.outer_radius) {
                        st.entered = 1;
                        st.inside = 0;
                    }
                } else if (r_bl - c.inner_radius <= 0.0) {
                    st.reason = kReachedInner;
                    st.mode = kEndA;
                } else if (st.inside > 0 && r_bl >= c.outer_radius) {
                    st.reason = kEscaped;
                    st.mode = kEndA;
                }
                if (st.mode == kAStep) {
                    st.old_r = r_bl;
                    double mn = c.min_step_abs;
                    if (abs_val(st.h_current) < mn) mn = abs_val(st.h_current);
                    issue_step(st, c, st.h_current, mn, c.max_step);
                }
            }
        }
        if (active && st.mode == kEndA) {
            // end of pass A (pass_b.hpp:940-955)
            const ImageConsts& c = J->c;
            if (st.entered && (st.reason == kReachedInner || st.reason == kEscaped)) {
                st.in_b = 1;
                st.mode = kBStep;
                st.rk_kind = -1;
                st.steps = 0;
                st.reached = 0;
                st.h_current = c.step;
                st.cap = c.max_radiation_step > 0.0 ? c.max_radiation_step : c.max_step;
#pragma unroll
                for (int f = 0; f < NF; ++f) RT::zero(stokes[f]);
            } else {
                st.mode = kDone;
            }
        }
        if (active && st.mode == kBStep && st.rk_kind < 0) {
            // pass-B loop top (pass_b.hpp:966-981)
            const ImageConsts& c = J->c;
            if (st.reached || st.steps >= c.max_steps) {
                st.mode = kDone;
            } else {
                double h = st.h_current;
                st.start_r = ks_radius(c.spin, S.x);
                if (st.start_r <= c.outer_radius && st.cap > 0.0) h = min_val(h, st.cap);
                st.hB = h;
                issue_step(st, c, h, c.min_step_abs, c.max_step);
            }
        }

        // ------------------------------------------------------------ RK job
        const bool run = active && (st.mode == kAStep || st.mode == kACrossHi || st.mode == kACrossTrial ||
                                    st.mode == kBStep || st.mode == kBCamCross);
        // Mixed policy: FP32 contraction only for jobs that start outside the
        // radiating sphere (by two maximal steps).  Inside it, FP32 noise in
        // the RHS reaches the step-doubling error estimate at the tolerance
        // level and reshapes the accepted-step sequence the Faraday-thick
        // transfer is sensitive to.  The choice depends only on the lane's own
        // ray, so a ray's result does not depend on its warp-mates.
        bool fp32 = false;
        if constexpr (P::kMixed) {
            fp32 = run && ks_radius(J->c.spin, S.x) > J->c.fp32_radius;
        }
        Ray next, mid;
        double err = 0.0;
        if (run) {
            const double mass = J->c.mass, spin = J->c.spin;
            if (st.mode == kACrossHi || st.mode == kACrossTrial) {
                const double hh = st.mode == kACrossHi ? st.full_h : st.full_h * st.trial;
                rk_job<P>(J->c.adaptive ? kRkRK4x2 : kRkRK4, mass, spin, S, hh, fp32, next, mid, err);
            } else {
                rk_job<P>(st.rk_kind, mass, spin, S, st.h_try, fp32, next, mid, err);
            }
            if (++guard > (1LL << 28)) {
                st.reason = kInvalidState;
                st.mode = kDone;
                st.in_b = 0;
                atomicExch(L.status, 2);
            }
        }

        // ----------------------------------------------- control after the job
        if (run && st.mode == kAStep) {
            const ImageConsts& c = J->c;
            bool accepted = true;
            double used_h = st.h_try;
            if (st.rk_kind != kRkRK4) {
                const double tol = max_val(c.tolerance, kTolFloor);
                if (err <= tol) {
                    st.h_current = accepted_next_h(st.h_try, err, tol, st.ctl_min, st.ctl_max, st.req_h);
                } else {
                    accepted = false;
                    if (rejected_attempt(st, err, tol)) {
                        st.rk_kind = -1;
                        if (abs_val(st.h_current) <= c.min_step_abs * 1.0001) {
                            st.reason = kAdaptiveUnderflow;
                            st.mode = kEndA;
                        } else {
                            st.n += 1;  // `continue` of the pass-A for loop
                        }
                    }
                }
            }
            if (accepted) {
                // pass_b.hpp:864-937
                st.rk_kind = -1;
                const double next_r = ks_radius(c.spin, next.x);
                const double old_r = st.old_r;
                if (!st.entered && next_r <= c.outer_radius) {
                    st.entered = 1;
                    st.inside = 0;
                } else if (!st.entered && next_r >= old_r) {
                    S = next;
                    st.pa_steps += 1;
                    st.reason = kEscaped;
                    st.mode = kEndA;
                }
                if (st.mode == kAStep) {
                    int crossing = kNone;
                    if (st.entered && old_r - c.inner_radius > 0.0 && next_r - c.inner_radius <= 0.0) {
                        crossing = kReachedInner;
                    } else if (st.entered && st.inside > 0 && old_r < c.outer_radius && next_r >= c.outer_radius) {
                        crossing = kEscaped;
                    }
                    if (crossing != kNone) {
                        st.cross_reason = crossing;
                        st.surf = crossing == kReachedInner ? c.inner_radius : c.outer_radius;
                        st.full_h = used_h;
                        best = S;
                        st.lo = 0.0;
                        st.hi = 1.0;
                        st.flo = ks_radius(c.spin, S.x) - st.surf;
                        if (st.flo == 0.0 || !finite_ray(next)) {
                            st.pa_steps += 1;  // the event keeps the first state
                            st.reason = crossing;
                            st.mode = kEndA;
                        } else {
                            st.mode = kACrossHi;
                        }
                    } else {
                        S = next;
                        st.pa_steps += 1;
                        if (st.entered) st.inside += 1;
                        st.n += 1;
                    }
                }
            }
        } else if (run && (st.mode == kACrossHi || st.mode == kACrossTrial)) {
            const ImageConsts& c = J->c;
            bool finish = false;
            if (st.mode == kACrossHi) {
                if (!finite_ray(next)) {
                    finish = true;
                } else {
                    const double fhi = ks_radius(c.spin, next.x) - st.surf;
                    if (!(fhi == fhi) || abs_val(fhi) >= kLarge) {
                        finish = true;
                    } else if (fhi == 0.0) {
                        best = next;
                        finish = true;
                    } else if ((st.flo > 0.0) == (fhi > 0.0)) {
                        finish = true;
                    } else {
                        st.fhi = fhi;
                        st.iter = 0;
                        st.use_secant = 1;
                    }
                }
            } else {
                const double ft = finite_ray(next) ? ks_radius(c.spin, next.x) - st.surf : 0.0;
                if (!finite_ray(next) || !(ft == ft) || abs_val(ft) >= kLarge) {
                    st.hi = st.trial;
                    st.use_secant = 0;
                } else if (ft == 0.0) {
                    best = next;
                    finish = true;
                } else if ((st.flo > 0.0) == (ft > 0.0)) {
                    st.lo = st.trial;
                    st.flo = ft;
                    best = next;
                } else {
                    st.hi = st.trial;
                    st.fhi = ft;
                }
                st.iter += 1;
            }
            if (!finish && st.iter >= 12) finish = true;
            if (finish) {
                S = best;
                st.pa_steps += 1;
                st.reason = st.cross_reason;
                st.mode = kEndA;
            } else {
                const double width = st.hi - st.lo;
                double trial = (st.lo + st.hi) * 0.5;
                const double denom = st.flo - st.fhi;
                if (st.use_secant && abs_val(denom) > kTiny) {
                    const double secant = st.lo + width * st.flo / denom;
                    const double g = width * 0.1;
                    if (secant > st.lo + g && secant < st.hi - g) trial = secant;
                }
                st.trial = trial;
                st.mode = kACrossTrial;
            }
        } else if (run && (st.mode == kBStep || st.mode == kBCamCross)) {
            const ImageConsts& c = J->c;
            const bool cam = st.mode == kBCamCross;
            bool proceed = true;
            double h = st.hB;
            if (st.rk_kind != kRkRK4) {
                const double tol = max_val(c.tolerance, kTolFloor);
                if (err <= tol) {
                    h = abs_val(st.h_try);
                    if (!cam) st.h_current = abs_val(accepted_next_h(st.h_try, err, tol, st.ctl_min, st.ctl_max, st.req_h));
                } else {
                    proceed = false;
                    if (rejected_attempt(st, err, tol)) {
                        st.h_current = abs_val(st.h_current);
                        st.rk_kind = -1;
                        st.mode = kBStep;
                        if (!cam && st.h_current <= c.min_step_abs * 1.0001) {
                            st.reason = kAdaptiveUnderflow;
                            st.mode = kDone;
                        }
                    }
                }
            }
            if (proceed) {
                Ray sample = st.rk_kind == kRkSD ? mid : next;
                int crosses = 1;
                if (!cam) {
                    // camera surface (pass_b.hpp:999-1028)
                    const double s0 = st.start_r - c.cam_radius;
                    const double s1 = ks_radius(c.spin, next.x) - c.cam_radius;
                    crosses = (s0 == 0.0 || s1 == 0.0) ? 1 : ((s0 < 0.0 && s1 > 0.0) || (s0 > 0.0 && s1 < 0.0));
                    if (crosses) {
                        const double denom = s0 - s1;
                        const double frac = abs_val(denom) <= kTiny ? 1.0 : min_val(1.0, max_val(0.0, s0 / denom));
                        const double h_cross = h * frac;
                        if (abs_val(h_cross) <= 1e-14) {
                            h = 0.0;
                            next = S;
                            sample = S;
                        } else if (frac < 0.999999999999) {
                            h = h_cross;
                            const double mn = min_val(c.min_step_abs, abs_val(h));
                            issue_step(st, c, h, mn, max_val(mn, abs_val(h)));
                            st.mode = kBCamCross;
                            st.hB = h;
                            proceed = false;
                        }
                    }
                }
                if (proceed) {
                    // radiation at the sample point (pass_b.hpp:1414-1496)
                    const double sample_r = ks_radius(c.spin, sample.x);
                    const double next_r = ks_radius(c.spin, next.x);
                    const double local_max_rs =
                        (c.max_radiation_step > 0.0 &&
                         (st.start_r <= c.outer_radius || sample_r <= c.outer_radius || next_r <= c.outer_radius))
                            ? c.max_radiation_step : 0.0;
                    typename RT::Co co[NF];
                    typename RT::Sample ps = RT::none();
                    if (sample_r - c.inner_radius > 0.0 && sample_r < c.outer_radius) ps = RT::sample(c, sample);
                    int required = 1;
                    const int nf = c.nfreq;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        co[f] = typename RT::Co{};
                        if (f < nf) {
                            co[f] = RT::coeffs(c, ps, f);
                            if (!c.faraday_rotation) co[f].rV = 0.0;
                            const int cand = radiation_substep_count(co[f], h, c.dlambda_scale[f], local_max_rs,
                                                                     c.max_radiation_depth, c.max_absorption_depth,
                                                                     c.max_faraday_depth);
                            required = cand > required ? cand : required;
                        }
                    }
                    if (required > 1 && h > c.min_step_abs * 1.0001) {
                        st.h_current = max_val(c.min_step_abs, h / double(required));
                        st.cap = st.h_current;
                    } else {
                        if (local_max_rs > 0.0 || c.max_radiation_depth > 0.0 || c.max_absorption_depth > 0.0 ||
                            c.max_faraday_depth > 0.0) {
                            int pred = 1;
#pragma unroll
                            for (int f = 0; f < NF; ++f) {
                                if (f < nf) {
                                    const int cand = radiation_substep_count(
                                        co[f], st.h_current, c.dlambda_scale[f], local_max_rs,
                                        c.max_radiation_depth, c.max_absorption_depth, c.max_faraday_depth);
                                    pred = cand > pred ? cand : pred;
                                }
                            }
                            st.cap = pred > 1 ? max_val(c.min_step_abs, st.h_current / double(pred)) : c.max_step;
                        } else {
                            st.cap = c.max_step;
                        }
                        if (h > 0.0) {
#pragma unroll
                            for (int f = 0; f < NF; ++f)
                                if (f < nf) RT::step(stokes[f], co[f], h, c, f);
                        }
                        S = next;
                        st.steps += 1;
                        if (crosses) st.reached = 1;
                    }
                    st.mode = kBStep;
                    st.rk_kind = -1;
                }
            }
        }

        // ------------------------------------------------------------ finish
        if (active && st.mode == kDone) {
            const ImageConsts& c = J->c;
            PixelOut o;
            o.pass_a_steps = st.pa_steps;
            o.steps = st.in_b ? st.steps : 0;
            int reason = st.reason;
            if (st.in_b) {
                if (st.reached) {
                    reason = kReachedCamera;
                } else if (reason != kAdaptiveUnderflow) {
                    reason = kMaxSteps;
                }
            }
            o.reason = reason;
            const Ray cam = camera_ray(c, J->frame, st.pixel);
            double obs[NF][4];
            Stokes4<double> sd[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f)
                sd[f] = st.in_b ? RT::result(stokes[f], c, f) : Stokes4<double>{0.0, 0.0, 0.0, 0.0};
            finish_ray<double, NF>(c, cam, S, st.in_b, sd, o, obs);
            store_stokes_n<NF>(J->out, st.pixel, J->npix, c.nfreq, obs);
            store_diagnostics(J->out, st.pixel, o);
            st.mode = kIdle;
            if (!L.refill) finished = 1;
        }
    }
}

}  // namespace kp
