// kp_far.cuh -- the far-phase kernel of the mixed policy.
//
// Beyond ImageConsts::fp32_radius a ray is pure transport: no surface lies
// within a step and no plasma is sampled, and every RK job runs the FP32
// stage chains of the Cartesian Kerr-Schild connection.  This kernel is built
// for that: one loop iteration is ONE right-hand-side evaluation of one RK
// stage, so the lanes of a warp evaluate the connection together however far
// into their jobs they are, and only the FP32 working set of a stage lives in
// registers:
//   * the job's FP64 chain bases -- the ray state S and the second chain's
//     base / the two-half-step endpoint T -- sit in shared memory, one SoA
//     column per lane, read once per stage for the FP64 k of the stage input
//     (exact form) and at chain ends;
//   * the control state of the pass-A / pass-B machine (FarCtl: the LaneState
//     fields the far phase touches) sits in shared memory too, touched once per
//     job;
//   * claim, park and finish of a ray, and the loop-top and after-job control,
//     are out of line: they run once per ray or per job, and inlined they would
//     crowd the stage loop's registers.
// The control machine is persistent_body's far phase (kp_persistent.cuh),
// statement for statement, so rays park, resume and finish exactly as there.
//
// Two forms of the stage arithmetic:
//   kExact   far_chain_f's arithmetic bit for bit (FP64 k of each stage input
//            and FP64 position accumulator): images equal the generic
//            kernel's;
//   !kExact  the position increment of a chain is rewritten without FP64 work
//            per stage.  Stage s = 0..3 evaluates dk_s at an input whose k is
//            k_B, k_B + (h/2) dk_0, k_B + (h/2) dk_1, k_B + h dk_2; with the
//            RK4 weights (1, 2, 2, 1) these sum to 6 k_B + h (dk_0 + dk_1 +
//            dk_2), so x_end = x_B + h k_B + (h^2 / 6) (dk_0 + dk_1 + dk_2):
//            the large term in FP64 once per chain, the small one accumulated
//            in FP32 (|h^2 dk| <~ 4e-4 M beyond the sphere, rounded to ~1e-11
//            M, far under the step-doubling tolerance).
#pragma once

#include "kp_persistent.cuh"

namespace kp {

constexpr int kFarLeanThreads = 128;

// Control state of a far-phase lane (the LaneState fields the far phase reads
// or writes) plus the position of the pending job's sample point.
// Small fields are packed (144 bytes per lane), so that four 128-lane CTAs
// fit an SM's shared memory.
struct FarCtl {
    double h_try, req_h, ctl_min, ctl_max;
    double h_current, old_r;
    double cap, hB, start_r;
    double x3_ref;
    double mid_x[3];  // SD: spatial position of the half-step endpoint (the sample point)
    int job, pixel, n, pa_steps, steps, inside;
    int mode : 8, rk_kind : 8, attempt : 8, reason : 8;
    int in_b : 2, entered : 2, reached : 2, chart : 2, fresh : 2, exhausted : 2, lean : 2;
    unsigned my_id;  // the lane's ray
    int lane_jobs;   // RK jobs the lane has run in this launch
};

// Per-CTA shared storage: FP64 rays as [component][lane] columns (lanes read
// consecutive doubles: no bank conflicts), control state per lane.
struct FarSmem {
    double S[16][kFarLeanThreads];  // ray state: the base of a job's first (and SD full) chain
    double T[16][kFarLeanThreads];  // SD: first half-step endpoint, then the two-half endpoint; RK4: endpoint
    float k1[12][kFarLeanThreads];  // SD: RHS of S, reused by the full chain
    FarCtl ctl[kFarLeanThreads];
};
constexpr size_t kFarSmemBytes = sizeof(FarSmem);
static_assert(kFarSmemBytes <= 56 * 1024, "four far CTAs must fit an SM's shared memory");

__device__ __forceinline__ void far_get(const double (&A)[16][kFarLeanThreads], int t, Ray& R) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        R.x.v[i] = A[i][t];
        R.k.v[i] = A[4 + i][t];
        R.e1.v[i] = A[8 + i][t];
        R.e2.v[i] = A[12 + i][t];
    }
}

__device__ __forceinline__ void far_put(double (&A)[16][kFarLeanThreads], int t, const Ray& R) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        A[i][t] = R.x.v[i];
        A[4 + i][t] = R.k.v[i];
        A[8 + i][t] = R.e1.v[i];
        A[12 + i][t] = R.e2.v[i];
    }
}

__device__ __forceinline__ void far_get_x(const double (&A)[16][kFarLeanThreads], int t, D4& x) {
#pragma unroll
    for (int i = 0; i < 4; ++i) x.v[i] = A[i][t];
}

// LaneState <-> FarCtl at claim and park.
__device__ __forceinline__ void far_from_lane(FarCtl& f, const LaneState& L) {
    f.h_try = L.h_try;
    f.req_h = L.req_h;
    f.ctl_min = L.ctl_min;
    f.ctl_max = L.ctl_max;
    f.h_current = L.h_current;
    f.old_r = L.old_r;
    f.cap = L.cap;
    f.hB = L.hB;
    f.start_r = L.start_r;
    f.x3_ref = L.x3_ref;
    f.job = L.job;
    f.pixel = L.pixel;
    f.mode = L.mode;
    f.in_b = L.in_b;
    f.attempt = L.attempt;
    f.rk_kind = L.rk_kind;
    f.n = L.n;
    f.entered = L.entered;
    f.inside = L.inside;
    f.pa_steps = L.pa_steps;
    f.reason = L.reason;
    f.steps = L.steps;
    f.reached = L.reached;
    f.chart = L.chart;
}

__device__ __forceinline__ void far_to_lane(LaneState& L, const FarCtl& f) {
    L.h_try = f.h_try;
    L.req_h = f.req_h;
    L.ctl_min = f.ctl_min;
    L.ctl_max = f.ctl_max;
    L.h_current = f.h_current;
    L.old_r = f.old_r;
    L.cap = f.cap;
    L.hB = f.hB;
    L.start_r = f.start_r;
    L.x3_ref = f.x3_ref;
    L.job = f.job;
    L.pixel = f.pixel;
    L.mode = f.mode;
    L.in_b = f.in_b;
    L.attempt = f.attempt;
    L.rk_kind = f.rk_kind;
    L.n = f.n;
    L.entered = f.entered;
    L.inside = f.inside;
    L.pa_steps = f.pa_steps;
    L.reason = f.reason;
    L.steps = f.steps;
    L.reached = f.reached;
    L.chart = f.chart;
}

// A fresh camera ray at the top of pass A (start_ray), in the far phase's
// chart.
template<class SC>
static __device__ __noinline__ void far_fresh(FarSmem& sm, int t, const JobDesc* J, int job, int pixel) {
    LaneState L;
    Ray S;
    start_ray<SC>(L, S, J, job, pixel);
    if constexpr (SC::kFarChart) {
        if (SC::chart_active(J->c)) {
            L.x3_ref = S.x.v[3];
            S = SC::to_phase(J->c, S);
            L.chart = 1;
        }
    }
    FarCtl& f = sm.ctl[t];
    far_from_lane(f, L);
    f.fresh = 1;
    far_put(sm.S, t, S);
}

// A parked ray resumed from its record; returns its job.
template<class SC>
static __device__ __noinline__ const JobDesc* far_resume(FarSmem& sm, int t, const RayRecord& rec,
                                                        const JobDesc* jobs) {
    LaneState L;
    memcpy(&L, rec.st, sizeof(LaneState));
    const JobDesc* J = &jobs[L.job];
    Ray S = rec.S;
    if constexpr (SC::kFarChart) {
        // a record parked for this phase already holds its chart
        if (!L.chart && SC::chart_active(J->c)) {
            L.x3_ref = S.x.v[3];
            S = SC::to_phase(J->c, S);
            L.chart = 1;
        }
    }
    FarCtl& f = sm.ctl[t];
    far_from_lane(f, L);
    f.fresh = 0;
    far_put(sm.S, t, S);
    return J;
}

// Parks the ray for phase `dest` (its own: a tick budget): the record gets the
// state and the control state; fields the far phase never touches keep the
// record's values (zero for a fresh ray, as start_ray leaves them).
template<class SC>
static __device__ __noinline__ void far_park(FarSmem& sm, int t, RayRecord& rec, const JobDesc* J, int dest) {
    FarCtl& f = sm.ctl[t];
    LaneState L;
    if (f.fresh) {
        memset(&L, 0, sizeof(L));
    } else {
        memcpy(&L, rec.st, sizeof(LaneState));
    }
    Ray S;
    far_get(sm.S, t, S);
    if constexpr (SC::kFarChart) {
        // leaving the phase: back to the records' chart; parked for this phase
        // (a tick budget): kept as is, so the ray resumes bit for bit
        if (f.chart && dest != kPhaseFar) {
            S = SC::to_record(J->c, S, f.x3_ref);
            f.chart = 0;
        }
    }
    far_to_lane(L, f);
    rec.S = S;
    memcpy(rec.st, &L, sizeof(LaneState));
}

// End of the ray: observer-basis Stokes from the record's channels, closure
// diagnostics, outputs (persistent_body's finish).
template<class SC, int NF>
static __device__ __noinline__ void far_finish(FarSmem& sm, int t, const WaveDesc& W, unsigned my_id,
                                               const JobDesc* J) {
    using RT = RadTraits<PolicyMixed, SC>;
    const FarCtl& f = sm.ctl[t];
    const ImageConsts& c = J->c;
    PixelOut o;
    o.pass_a_steps = f.pa_steps;
    o.steps = f.in_b ? f.steps : 0;
    int reason = f.reason;
    if (f.in_b) {
        if (f.reached) {
            reason = kReachedCamera;
        } else if (reason != kAdaptiveUnderflow && reason != kSlowLightTimeExhausted) {
            reason = kMaxSteps;
        }
    }
    o.reason = reason;
    const Ray cam = SC::camera(c, J->frame, f.pixel);
    typename RT::Stokes stokes[NF];
    if (f.in_b) memcpy(&stokes[0], W.pool[my_id].stokes, sizeof(stokes));
    double obs[NF][4];
    Stokes4<double> sd[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) sd[q] = f.in_b ? RT::result(stokes[q], c, q) : Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    Ray S;
    far_get(sm.S, t, S);
    if constexpr (SC::kFarChart) {
        const Ray S_rec = f.chart ? SC::to_record(c, S, f.x3_ref) : S;
        finish_ray_scene<typename RecordScene<SC>::type, NF>(c, cam, S_rec, f.in_b, sd, o, obs);
    } else {
        finish_ray_scene<SC, NF>(c, cam, S, f.in_b, sd, o, obs);
    }
    store_stokes_n<NF>(J->out, f.pixel, J->npix, c.nfreq, obs);
    store_diagnostics(J->out, f.pixel, o);
    if constexpr (SC::kSlowLight) {
        if (!f.in_b) J->out.basis_identity_error[f.pixel] = 0.0;
    }
    if (W.job_done) atomicAdd(&W.job_done[f.job], 1u);
}

// Control at a loop top (persistent_body's control before the job, far
// phase): returns the phase the ray is handed to, or -1 (a job was issued,
// or the ray is done).
template<class SC, int NF>
static __device__ __noinline__ int far_before_job(FarSmem& sm, int t, const WaveDesc& W, unsigned my_id,
                                                  const JobDesc* J, bool over_budget) {
    FarCtl& st = sm.ctl[t];
    const ImageConsts& c = J->c;
    int dest = -1;
    if (st.mode == kAStep && st.rk_kind < 0) {
        D4 x;
        far_get_x(sm.S, t, x);
        const double r_bl = SC::radius(c, x);
        const int want_phase = phase_of(c, 0, r_bl);
        if (want_phase != kPhaseFar) {
            dest = want_phase;
        } else if (over_budget) {
            dest = kPhaseFar;
        } else if (st.n >= c.max_steps) {
            // pass-A loop top (pass_b.hpp:793-838)
            st.mode = kEndA;
        } else {
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
    if (dest < 0 && st.mode == kEndA) {
        // end of pass A (pass_b.hpp:940-955)
        if (st.entered && (st.reason == kReachedInner || st.reason == kEscaped)) {
            using RT = RadTraits<PolicyMixed, SC>;
            st.in_b = 1;
            st.mode = kBStep;
            st.rk_kind = -1;
            st.steps = 0;
            st.reached = 0;
            st.h_current = c.step;
            st.cap = c.max_radiation_step > 0.0 ? c.max_radiation_step : c.max_step;
            typename RT::Stokes stokes[NF];
#pragma unroll
            for (int q = 0; q < NF; ++q) RT::zero(stokes[q]);
            memcpy(W.pool[my_id].stokes, &stokes[0], sizeof(stokes));
        } else {
            st.mode = kDone;
        }
    }
    if (dest < 0 && st.mode == kBStep && st.rk_kind < 0) {
        if (st.reached || st.steps >= c.max_steps) {
            st.mode = kDone;
        } else {
            D4 x;
            far_get_x(sm.S, t, x);
            const double r_bl = SC::radius(c, x);
            const int want_phase = phase_of(c, 1, r_bl);
            if (want_phase != kPhaseFar) {
                dest = want_phase;
            } else if (over_budget) {
                dest = kPhaseFar;
            } else {
                // pass-B loop top (pass_b.hpp:966-981)
                double h = st.h_current;
                st.start_r = r_bl;
                if (st.start_r <= c.outer_radius && st.cap > 0.0) h = min_val(h, st.cap);
                st.hB = h;
                issue_step(st, c, h, c.min_step_abs, c.max_step);
            }
        }
    }
    return dest;
}

// Control after a job (persistent_body's control after the job, far phase):
// the job's endpoint is in T, an SD job's sample point in mid_x, its error
// estimate in err.
template<class SC>
static __device__ __noinline__ void far_after_job(FarSmem& sm, int t, const WaveDesc& W, const JobDesc* J,
                                                  double err) {
    FarCtl& st = sm.ctl[t];
    const ImageConsts& c = J->c;
    if (st.mode == kAStep) {
        bool accepted = true;
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
            D4 xn;
            far_get_x(sm.T, t, xn);
            const double next_r = SC::radius(c, xn);
            const double old_r = st.old_r;
            if (!st.entered && next_r <= c.outer_radius) {
                st.entered = 1;
                st.inside = 0;
            } else if (!st.entered && next_r >= old_r) {
#pragma unroll
                for (int i = 0; i < 16; ++i) sm.S[i][t] = sm.T[i][t];
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
                    atomicExch(W.status, 3);  // surfaces lie inside the near phase
                    st.reason = kInvalidState;
                    st.mode = kDone;
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) sm.S[i][t] = sm.T[i][t];
                    st.pa_steps += 1;
                    if (st.entered) st.inside += 1;
                    st.n += 1;
                }
            }
        }
    } else if (st.mode == kBStep || st.mode == kBCamCross) {
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
                        st.reason = SC::kSlowLight ? kMaxSteps : kAdaptiveUnderflow;
                        st.mode = kDone;
                    }
                }
            }
        }
        if (proceed) {
            // the sample point: SD's first half step, otherwise the endpoint
            D4 xm;
            if (st.rk_kind == kRkSD) {
                xm.v[0] = 0.0;
                xm.v[1] = st.mid_x[0];
                xm.v[2] = st.mid_x[1];
                xm.v[3] = st.mid_x[2];
            } else {
                far_get_x(sm.T, t, xm);
            }
            double sample_r = SC::radius(c, xm);
            bool next_is_S = false;
            int crosses = 1;
            if (!cam) {
                // camera surface (pass_b.hpp:999-1028)
                D4 xn;
                far_get_x(sm.T, t, xn);
                const double s0 = st.start_r - c.cam_radius;
                const double s1 = SC::radius(c, xn) - c.cam_radius;
                crosses = (s0 == 0.0 || s1 == 0.0) ? 1 : ((s0 < 0.0 && s1 > 0.0) || (s0 > 0.0 && s1 < 0.0));
                if (crosses) {
                    const double denom = s0 - s1;
                    const double frac = abs_val(denom) <= kTiny ? 1.0 : min_val(1.0, max_val(0.0, s0 / denom));
                    const double h_cross = h * frac;
                    if (abs_val(h_cross) <= 1e-14) {
                        h = 0.0;
                        next_is_S = true;
                        D4 xs;
                        far_get_x(sm.S, t, xs);
                        sample_r = SC::radius(c, xs);
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
                D4 xn;
                if (next_is_S) far_get_x(sm.S, t, xn); else far_get_x(sm.T, t, xn);
                const double next_r = SC::radius(c, xn);
                const double local_max_rs =
                    (c.max_radiation_step > 0.0 &&
                     (st.start_r <= c.outer_radius || sample_r <= c.outer_radius || next_r <= c.outer_radius))
                        ? c.max_radiation_step : 0.0;
                // the sample lies outside the radiating sphere: every
                // coefficient is zero, the transfer step leaves the Stokes
                // vector unchanged, the step cap resolves to max_step
                // (pass_b.hpp:1482-1486)
                if (local_max_rs > 0.0 || (sample_r - c.inner_radius > 0.0 && sample_r < c.outer_radius)) {
                    atomicExch(W.status, 3);
                }
                st.cap = c.max_step;
                if (!next_is_S) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) sm.S[i][t] = sm.T[i][t];
                }
                st.steps += 1;
                if (crosses) st.reached = 1;
                st.mode = kBStep;
                st.rk_kind = -1;
            }
        }
    }
}

// A job the stage loop does not run (Cash-Karp, or a chart scene's ray in
// its record chart): the whole job through rk_job, endpoint to T.
template<class SC>
static __device__ __noinline__ double far_slow_job(FarSmem& sm, int t, const JobDesc* J) {
    const FarCtl& st = sm.ctl[t];
    Ray S, next, mid;
    far_get(sm.S, t, S);
    double err = 0.0;
    rk_job<PolicyMixed, true, SC>(st.rk_kind, J->c, S, st.h_try, next, mid, err);
    far_put(sm.T, t, next);
    sm.ctl[t].mid_x[0] = mid.x.v[1];
    sm.ctl[t].mid_x[1] = mid.x.v[2];
    sm.ctl[t].mid_x[2] = mid.x.v[3];
    return err;
}

// state_error_norm(E, T) (the scaled norm of control_error) for the SD full
// step's endpoint E, left by the stage loop in the ray's record (whose state
// slot the far phase writes only when it parks the ray): the rare branch of
// the error estimate, run by the control pass so that the stage loop holds no
// call and no division.
__device__ __forceinline__ double far_norm(const FarSmem& sm, int t, const Ray& E) {
    const D4* e4[4] = {&E.x, &E.k, &E.e1, &E.e2};
    double m = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const double e = e4[w]->v[mu], n = sm.T[4 * w + mu][t];
            const double sc = max_val(1.0, max_val(abs_val(e), abs_val(n)));
            m = max_val(m, abs_val(e - n) / sc);
        }
    }
    return m;
}

// Stage-loop registers of a lane's job: the FP32 stage input, its chain
// base's FP32 copy, the accumulators.
struct FarChain {
    float bx[3], bq[3][4];  // FP32 copy of the chain base
    float Xx[3], Xq[3][4];  // stage input
    float Aq[3][4];         // accumulator of dk, de1, de2
    D4 Xk, Ax;              // exact form: FP64 k of the stage input, position accumulator
    float Sk[4];            // fast form: dk of stages 1..3
};

// The stage loop of the lanes whose job (rk_kind, h_try of their FarCtl)
// runs as FP32 chains (`lean`): stages until every such job of the warp is
// complete; returns the lane's error estimate (0 for RK4 jobs; -1 when the
// scaled norm is needed: the full step's endpoint is then in the ray's
// record, `rec`).  Run by all
// lanes of the warp together, in the kernel's own register context: every
// call of the control machine happens between stage loops, where none of the
// stage state is live.
template<class SC, bool kExact>
__device__ __forceinline__ double far_stages(int t, const JobDesc* J, bool lean, RayRecord* rec) {
    // the block's shared storage, named here so that its accesses compile to
    // shared-memory instructions
    extern __shared__ __align__(16) unsigned char kp_far_smem[];
    FarSmem& sm = *reinterpret_cast<FarSmem*>(kp_far_smem);
    const unsigned FULL = 0xffffffffu;
    // the job in flight
    int kind = 0, ch = 0, stg = 0;  // kRkSD or kRkRK4; chain 0..2; stage 0..3
    double h = 0.0, hc = 0.0;       // job step, chain step
    double h6_full = 0.0, h6_half = 0.0;  // h / 6 and (h / 2) / 6, formed at job start
    float M = 0.f, a = 0.f;
    FarChain C;

    // Loads the FP32 copy of chain `ch`'s base and sets up its first stage
    // input; the SD full chain takes its first stage from k1.
    auto begin_chain = [&]() {
        double (&B)[16][kFarLeanThreads] = (ch == 1) ? sm.T : sm.S;
        hc = (kind == kRkRK4 || ch == 2) ? h : 0.5 * h;
#pragma unroll
        for (int i = 0; i < 3; ++i) C.bx[i] = float(B[1 + i][t]);
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.bq[w][i] = float(B[4 * (w + 1) + i][t]);
#pragma unroll
        for (int i = 0; i < 3; ++i) C.Xx[i] = C.bx[i];
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Xq[w][i] = C.bq[w][i];
        if constexpr (kExact) {
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Xk.v[i] = B[4 + i][t];
        }
        stg = 0;
    };

    // acc = ((k1 + 2 k2) + 2 k3) + k4 of the chain; the fast form's position
    // sum takes dk of the stages 0..2 (the inputs of stages 1..3).
    auto accumulate = [&](const float (&kq)[3][4]) {
        if (stg == 0) {
            if constexpr (kExact) {
                C.Ax = C.Xk;
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) C.Sk[i] = kq[0][i];
            }
#pragma unroll
            for (int w = 0; w < 3; ++w)
#pragma unroll
                for (int i = 0; i < 4; ++i) C.Aq[w][i] = kq[w][i];
        } else {
            const float wf = stg == 3 ? 1.0f : 2.0f;
            if constexpr (kExact) {
                const double wd = stg == 3 ? 1.0 : 2.0;
#pragma unroll
                for (int i = 0; i < 4; ++i) C.Ax.v[i] = C.Ax.v[i] + C.Xk.v[i] * wd;
            } else if (stg < 3) {
#pragma unroll
                for (int i = 0; i < 4; ++i) C.Sk[i] = C.Sk[i] + kq[0][i];
            }
#pragma unroll
            for (int w = 0; w < 3; ++w)
#pragma unroll
                for (int i = 0; i < 4; ++i) C.Aq[w][i] = C.Aq[w][i] + kq[w][i] * wf;
        }
    };

    // Forms the next stage input B + cc * kq (stage stg < 3 done).
    auto next_input = [&](const float (&kq)[3][4]) {
        const double cc = stg < 2 ? 0.5 * hc : hc;
        const float cf = float(cc);
#pragma unroll
        for (int i = 0; i < 3; ++i) C.Xx[i] = C.bx[i] + C.Xq[0][i + 1] * cf;
        if constexpr (kExact) {
            const double (&B)[16][kFarLeanThreads] = (ch == 1) ? sm.T : sm.S;
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Xk.v[i] = B[4 + i][t] + double(kq[0][i]) * cc;
        }
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Xq[w][i] = C.bq[w][i] + kq[w][i] * cf;
        ++stg;
    };

    // Accumulates the stage derivative kq and forms the next stage input; at
    // the chain's last stage, writes the chain endpoint.  Returns true when
    // the job is complete (err set).
    auto stage_done = [&](const float (&kq)[3][4], double& err) -> bool {
        if (ch == 0 && stg == 0 && kind == kRkSD) {
#pragma unroll
            for (int w = 0; w < 3; ++w)
#pragma unroll
                for (int i = 0; i < 4; ++i) sm.k1[4 * w + i][t] = kq[w][i];
        }
        accumulate(kq);
        if (stg < 3) {
            next_input(kq);
            return false;
        }
        // chain endpoint B + (hc / 6) acc, one component at a time (w: x, k,
        // e1, e2; mu: 0..3), straight to shared memory
        const double h6 = (kind == kRkRK4 || ch == 2) ? h6_full : h6_half;
        double (&B)[16][kFarLeanThreads] = (ch == 1) ? sm.T : sm.S;
        auto endpoint = [&](int w, int mu) -> double {
            const double base = B[4 * w + mu][t];
            if (w == 0) {
                if constexpr (kExact) {
                    return base + C.Ax.v[mu] * h6;
                } else {
                    // x_B + hc k_B + (hc^2 / 6) (dk_0 + dk_1 + dk_2)
                    return base + (B[4 + mu][t] * hc + double(C.Sk[mu]) * (hc * h6));
                }
            }
            return base + double(C.Aq[w - 1][mu]) * h6;
        };
        if (kind == kRkSD && ch == 2) {
            // control_error(full, two-half) in its own order: max |a - b| when
            // every difference is at most tol/64, else the scaled norm
            // (state_error_norm)
            const double tol = max_val(J->c.tolerance, kTolFloor);
            const double lim = tol * (1.0 / 64.0);
            bool small = true;
            double m = 0.0;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
#pragma unroll
                for (int w = 0; w < 4; ++w) {
                    const double d = abs_val(endpoint(w, mu) - sm.T[4 * w + mu][t]);
                    small = small && d <= lim;
                    m = max_val(m, d);
                }
            }
            if (!small) {
                // the scaled norm: the control pass forms it from E (below)
                double* E = &rec->S.x.v[0];
#pragma unroll
                for (int w = 0; w < 4; ++w)
#pragma unroll
                    for (int mu = 0; mu < 4; ++mu) E[4 * w + mu] = endpoint(w, mu);
                m = -1.0;
            }
            err = m;
            return true;
        }
#pragma unroll
        for (int w = 0; w < 4; ++w)
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) sm.T[4 * w + mu][t] = endpoint(w, mu);
        if (kind == kRkSD && ch == 0) {
            // the half-step endpoint is the SD job's sample point
            sm.ctl[t].mid_x[0] = sm.T[1][t];
            sm.ctl[t].mid_x[1] = sm.T[2][t];
            sm.ctl[t].mid_x[2] = sm.T[3][t];
        }
        if (kind == kRkRK4) {
            err = 0.0;
            return true;
        }
        ++ch;
        begin_chain();
        if (ch == 2) {
            // the full chain's first stage is k1 of S, already evaluated
            float kq1[3][4];
#pragma unroll
            for (int w = 0; w < 3; ++w)
#pragma unroll
                for (int i = 0; i < 4; ++i) kq1[w][i] = sm.k1[4 * w + i][t];
            accumulate(kq1);
            next_input(kq1);
        }
        return false;
    };

    // Starts the job the control machine issued (rk_kind, h_try).
    auto begin_job = [&]() -> bool {
        const FarCtl& st = sm.ctl[t];
        kind = st.rk_kind;
        if (!((kind == kRkSD || kind == kRkRK4) && SC::chart_active(J->c))) return false;
        h = st.h_try;
        h6_full = h / 6.0;
        h6_half = (0.5 * h) / 6.0;
        M = float(J->c.mass);
        a = float(J->c.spin);
        ch = 0;
        begin_chain();
        return true;
    };

    double job_err = 0.0;
    bool in_job = lean && begin_job();
#pragma unroll 1
    while (__any_sync(FULL, in_job)) {
        if (in_job) {
            float kq[3][4];
            ks_transport_factored<float>(M, a, C.Xx[0], C.Xx[1], C.Xx[2], C.Xq, kq);
            if (stage_done(kq, job_err)) in_job = false;
        }
    }
    return job_err;
}

// The control machine of one pass over the warp (all lanes together):
// after-job control of the lane's completed stage-loop job (`done`, error
// `err`), claim, loop-top control, park, finish, job start.  Jobs of another
// form run whole here.  Leaves FarCtl::lean set on lanes whose next job runs
// in the stage loop; returns false when the warp has no work left.
template<class SC, int NF>
static __device__ __noinline__ bool far_control(const WaveDesc& W, int t, bool done, double err) {
    extern __shared__ __align__(16) unsigned char kp_far_smem[];
    FarSmem& sm = *reinterpret_cast<FarSmem*>(kp_far_smem);
    const unsigned FULL = 0xffffffffu;
    const int lane = t & 31;
    FarCtl& st = sm.ctl[t];
    unsigned my_id = st.my_id;
    int lane_jobs = st.lane_jobs;
    const JobDesc* J = st.job >= 0 ? &W.jobs[st.job] : nullptr;
    const long long nfresh = W.fresh_end - W.fresh_begin;
    const long long total_in = nfresh + (long long)(W.in_ids ? *W.in_count : 0u);
    st.lean = 0;

    // ---------------------------------------------------- control after a job
    auto after = [&](double e) {
        if (++lane_jobs > (1 << 30)) {
            st.reason = kInvalidState;
            st.mode = kDone;
            st.in_b = 0;
            atomicExch(W.status, 2);
        } else {
            far_after_job<SC>(sm, t, W, J, e);
        }
        if (st.mode == kDone) {
            far_finish<SC, NF>(sm, t, W, my_id, J);
            st.mode = kIdle;
        }
    };
    if (done) {
        // the SD error estimate's scaled norm, deferred by the stage loop
        if (err < 0.0) err = far_norm(sm, t, W.pool[my_id].S);
        after(err);
    }

    // ------------------------------------------------------------------ claim
    const bool want = !st.exhausted && st.mode == kIdle;
    bool forward = false;
    const unsigned need = __ballot_sync(FULL, want);
    if (need) {
        unsigned long long base = 0;
        const int leader = __ffs(need) - 1;
        if (lane == leader) base = atomicAdd(W.in_head, (unsigned long long)__popc(need));
        base = __shfl_sync(FULL, base, leader);
        if (want) {
            const long long k = (long long)(base + __popc(need & ((1u << lane) - 1u)));
            if (k >= total_in) {
                st.exhausted = 1;
            } else if (k < nfresh) {
                // a fresh camera ray: locate its job and start pass A
                const long long id = W.fresh_begin + k;
                int lo = 0, hi = W.njobs - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (W.jobs[mid].ray_begin <= id) lo = mid; else hi = mid - 1;
                }
                my_id = unsigned(id);
                J = &W.jobs[lo];
                far_fresh<SC>(sm, t, J, lo, int(id - J->ray_begin));
            } else if (W.budget > 0 && lane_jobs >= W.budget) {
                // past the budget: hand the id on untouched (below)
                my_id = W.in_ids[k - nfresh];
                forward = true;
            } else {
                // a parked ray: resume from its record
                my_id = W.in_ids[k - nfresh];
                J = far_resume<SC>(sm, t, W.pool[my_id], W.jobs);
            }
        }
    }
    queue_push(W.out_ids[kPhaseFar], W.out_count[kPhaseFar], forward, my_id);
    st.my_id = my_id;
    // a lane that forwarded an id has more input to claim
    if (!__any_sync(FULL, st.mode != kIdle || forward)) {
        st.lane_jobs = lane_jobs;
        return false;
    }

    // -------------------------------------------------- control at a loop top
    int dest = -1;
    if (st.mode != kIdle && st.mode != kDone) {
        dest = far_before_job<SC, NF>(sm, t, W, my_id, J, W.budget > 0 && lane_jobs >= W.budget);
    }
    const bool park = dest >= 0;
    if (park) far_park<SC>(sm, t, W.pool[my_id], J, dest);
    // a lane past its budget keeps claiming and parks each claimed ray at
    // once, so every input ends the launch finished or in a queue
#pragma unroll
    for (int d = 0; d < kPhases; ++d) queue_push(W.out_ids[d], W.out_count[d], dest == d, my_id);
    if (park) st.mode = kIdle;
    if (st.mode == kDone) {
        far_finish<SC, NF>(sm, t, W, my_id, J);
        st.mode = kIdle;
    }

    // -------------------------------------------------------------- job start
    if (st.mode == kAStep || st.mode == kBStep || st.mode == kBCamCross) {
        const int kind = st.rk_kind;
        if ((kind == kRkSD || kind == kRkRK4) && SC::chart_active(J->c)) {
            st.lean = 1;
        } else {
            // a job of another form: whole, out of line; its next attempt
            // (if any) starts in the next pass
            after(far_slow_job<SC>(sm, t, J));
        }
    }
    st.lane_jobs = lane_jobs;
    return true;
}

template<class SC, int NF, bool kExact>
__device__ __forceinline__ void far_body(const WaveDesc& W) {
    extern __shared__ __align__(16) unsigned char kp_far_smem[];
    FarSmem& sm = *reinterpret_cast<FarSmem*>(kp_far_smem);
    if (blockDim.x != kFarLeanThreads) {
        // the shared columns are sized for kFarLeanThreads lanes
        if (threadIdx.x == 0) atomicExch(W.status, 4);
        return;
    }
    const int t = threadIdx.x;
    FarCtl& st = sm.ctl[t];
    st.mode = kIdle;
    st.job = -1;
    st.rk_kind = -1;
    st.exhausted = 0;
    st.lean = 0;
    st.my_id = 0;
    st.lane_jobs = 0;
    bool done = false;
    double err = 0.0;
    // control of every lane, then the stage loop until the warp's jobs are
    // complete
#pragma unroll 1
    while (far_control<SC, NF>(W, t, done, err)) {
        done = st.lean;
        err = far_stages<SC, kExact>(t, st.job >= 0 ? &W.jobs[st.job] : nullptr, done, W.pool + st.my_id);
    }
}

}  // namespace kp
