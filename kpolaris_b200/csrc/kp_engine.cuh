// kp_engine.cuh -- persistent ray engine: every lane of a warp holds one ray
// and advances it through a resumable state machine whose loop iteration is
// one RK job (a step-doubling attempt, an RK4 step, a composed pair of RK4
// half steps or a Cash-Karp attempt) started from the lane's current state.
// Jobs run as a stage loop around ONE right-hand-side site, so lanes of a warp
// evaluate the RHS together whatever their phase (pass A, surface refinement,
// pass B, camera crossing).  Finished lanes refill from a global ray queue
// shared by every image of the launch (warp-aggregated atomics), which removes
// both the tail of uneven rays and the launch-per-image cost.
//
// The control machine restates, as explicit states, the loops of
// trace_pass_b_segment_model_pixel_metric / _multifrequency_pixel_metric
// (src/geodesic/pass_b.hpp:769-1114, :1131-1501), adaptive_rk4_step
// (src/geodesic/rk4.hpp:108-161) and locate_metric_surface_crossing
// (src/geodesic/pass_a_core.hpp:94-197).  With the FP64 policy every
// arithmetic operation is the reference's, in its order: results are
// bit-identical to the per-pixel FP64 kernel.
#pragma once

#include "kp_camera.cuh"
#include "kp_integrate.cuh"
#include "kp_radiation.cuh"
#include "kp_trace_fp64.cuh"
#include "kp_geometry_f32.cuh"
#include "kp_radiation_f32.cuh"
#include "kp_scene.cuh"

namespace kp {

// Kinds of RK job.
enum RkKind : int { kRkSD = 0, kRkRK4 = 1, kRkRK4x2 = 2, kRkCK = 3 };

// Control modes: what the pending RK job's result is for.
enum Mode : int {
    kIdle = 0,
    kAStep = 1,        // pass-A step attempt (adaptive sequence or fixed RK4)
    kACrossHi = 2,     // crossing search: full-step endpoint with the trial evaluator
    kACrossTrial = 3,  // crossing search: trial at fraction `trial`
    kBStep = 4,        // pass-B step attempt
    kBCamCross = 5,    // pass-B partial step to the camera surface
    kDone = 6,
};

// ---------------------------------------------------------------- RHS policy
// FP64 policy: the reference's arithmetic.
struct PolicyFP64 {
    static constexpr bool kMixed = false;
};
// Mixed policy: FP32 connection contraction in the far-phase kernel (rays
// beyond ImageConsts::fp32_radius), FP64 inside; FP64 state, stage
// combination and step control everywhere; FP32 radiative transfer.
struct PolicyMixed {
    static constexpr bool kMixed = true;
};

// Radiation side of a policy and scene: FP64 (the reference's arithmetic) or
// FP32 with the per-frequency 2^E emission scale (kp_radiation_f32.cuh).
template<class P, class S = SceneRiaf>
struct RadTraits;

template<>
struct RadTraits<PolicyFP64, SceneRiaf> {
    using Stokes = Stokes4<double>;
    using Co = Coeffs<double>;
    using Sample = RiafSample;
    __device__ static void zero(Stokes& s) { s = Stokes4<double>{0.0, 0.0, 0.0, 0.0}; }
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return riaf_sample(c, r); }
    __device__ static Sample none() {
        Sample s;
        s.emitting = 0;
        return s;
    }
    __device__ static Co coeffs(const ImageConsts& c, const Sample& p, int f) {
        return riaf_coefficients(c, p, c.freq[f]);
    }
    __device__ static Co coeffs_ctl(const ImageConsts& c, const Sample& p, int g) {
        return riaf_coefficients(c, p, c.ctl_freq[g]);
    }
    __device__ static void step(Stokes& s, const Co& co, double h, const ImageConsts& c, int f) {
        stokes_step(s, co, abs_val(h) * c.dlambda_scale[f]);
    }
    __device__ static Stokes4<double> result(const Stokes& s, const ImageConsts&, int) { return s; }
};

template<>
struct RadTraits<PolicyMixed, SceneRiaf> {
    using Stokes = StokesF;
    using Co = CoeffsF;
    using Sample = RiafSampleF;
    __device__ static void zero(Stokes& s) { s = StokesF{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}; }
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return riaf_sample_f(c, r); }
    __device__ static Sample none() {
        Sample s;
        s.emitting = 0;
        return s;
    }
    __device__ static Co coeffs(const ImageConsts& c, const Sample& p, int f) {
        return riaf_coefficients_f(c, p, float(c.freq[f] * 1e-9), c.emission_scale_pow2[f]);
    }
    __device__ static Co coeffs_ctl(const ImageConsts& c, const Sample& p, int g) {
        return riaf_coefficients_f(c, p, float(c.ctl_freq[g] * 1e-9), c.ctl_emission_scale_pow2[g]);
    }
    __device__ static void step(Stokes& s, const Co& co, double h, const ImageConsts& c, int f) {
        stokes_step_f(s, co, float(abs_val(h) * c.dlambda_scale[f]));
    }
    __device__ static Stokes4<double> result(const Stokes& s, const ImageConsts& c, int f) {
        const double inv = c.inv_emission_scale_pow2[f];
        return Stokes4<double>{(double(s.I) + double(s.cI)) * inv, (double(s.Q) + double(s.cQ)) * inv,
                               (double(s.U) + double(s.cU)) * inv, (double(s.V) + double(s.cV)) * inv};
    }
};

// GRMHD grid plasma, FP64 throughout.
template<>
struct RadTraits<PolicyFP64, SceneGrmhd> {
    using Stokes = Stokes4<double>;
    using Co = Coeffs<double>;
    using Sample = GrmhdSample;
    __device__ static void zero(Stokes& s) { s = Stokes4<double>{0.0, 0.0, 0.0, 0.0}; }
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return grmhd_sample(c, r); }
    __device__ static Sample none() {
        Sample s;
        s.emitting = 0;
        return s;
    }
    __device__ static Co coeffs(const ImageConsts& c, const Sample& p, int f) {
        return grmhd_coefficients(c, p, c.freq[f]);
    }
    __device__ static Co coeffs_ctl(const ImageConsts& c, const Sample& p, int g) {
        return grmhd_coefficients(c, p, c.ctl_freq[g]);
    }
    __device__ static void step(Stokes& s, const Co& co, double h, const ImageConsts& c, int f) {
        stokes_step(s, co, abs_val(h) * c.dlambda_scale[f]);
    }
    __device__ static Stokes4<double> result(const Stokes& s, const ImageConsts&, int) { return s; }
};

// GRMHD grid plasma under the mixed policy: the grid gather, the fluid and
// field four-vectors and the screen angle stay FP64 (grmhd_sample, the
// reference's fluid_state); the thermal fit per frequency and the Stokes
// update run in FP32 with the 2^E emission scale and compensated sums, the
// same code as the mixed RIAF scene.
__device__ __forceinline__ RiafSampleF grmhd_sample_to_f(const ImageConsts& c, const GrmhdSample& p) {
    RiafSampleF o;
    o.emitting = p.emitting;
    o.on_axis = 0;
    o.has_chi = p.has_chi;
    if (!p.emitting) return o;
    o.ne = float(p.ne);
    o.thetae = float(p.thetae);
    o.b = float(p.b);
    o.nu_fluid = float(p.nu_scale);
    o.cos_theta = float(p.ct);
    o.sin_theta = float(p.st);
    o.theta = 0.0f;
    o.cos2chi = float(p.cos2chi);
    o.sin2chi = float(p.sin2chi);
    riaf_sample_thermal_f(c, o);
    return o;
}

__device__ __forceinline__ RiafSampleF grmhd_sample_f(const ImageConsts& c, const Ray& r) {
    return grmhd_sample_to_f(c, grmhd_sample(c, r));
}

template<>
struct RadTraits<PolicyMixed, SceneGrmhd> : RadTraits<PolicyMixed, SceneRiaf> {
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return grmhd_sample_f(c, r); }
};

// Slow light: the grid plasma interpolated in time between the resident
// snapshots around each sample's fluid time (grmhd_sample_series).
template<>
struct RadTraits<PolicyFP64, SceneGrmhdSlow> : RadTraits<PolicyFP64, SceneGrmhd> {
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return grmhd_sample_series(c, r); }
};

__device__ __forceinline__ RiafSampleF grmhd_series_sample_f(const ImageConsts& c, const Ray& r) {
    return grmhd_sample_to_f(c, grmhd_sample_series(c, r));
}

template<>
struct RadTraits<PolicyMixed, SceneGrmhdSlow> : RadTraits<PolicyMixed, SceneRiaf> {
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return grmhd_series_sample_f(c, r); }
};

// The RIAF in Boyer-Lindquist coordinates: the same plasma model, sampled
// in the ray's own BL components (riaf_sample_t<true>); under the mixed
// policy the FP64 sample feeds the FP32 fits and transfer.
template<>
struct RadTraits<PolicyFP64, SceneRiafBL> : RadTraits<PolicyFP64, SceneRiaf> {
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) { return riaf_sample_t<true>(c, r); }
};

__device__ __forceinline__ RiafSampleF riaf_sample_to_f(const ImageConsts& c, const RiafSample& p) {
    RiafSampleF o;
    o.emitting = p.emitting;
    o.on_axis = p.on_axis;
    o.has_chi = p.has_chi;
    if (!p.emitting) return o;
    o.ne = float(p.ne);
    o.thetae = float(p.thetae);
    o.b = float(p.b);
    o.nu_fluid = float(p.nu_fluid);
    o.cos_theta = float(p.cos_theta);
    o.sin_theta = float(p.sin_theta);
    o.theta = float(p.theta);
    o.cos2chi = float(p.cos2chi);
    o.sin2chi = float(p.sin2chi);
    riaf_sample_thermal_f(c, o);
    return o;
}

template<>
struct RadTraits<PolicyMixed, SceneRiafBL> : RadTraits<PolicyMixed, SceneRiaf> {
    __device__ static Sample sample(const ImageConsts& c, const Ray& r) {
        return riaf_sample_to_f(c, riaf_sample_t<true>(c, r));
    }
};

// A far-phase chart scene radiates nothing; its Stokes types are its
// record scene's.
template<class P, class B>
struct RadTraits<P, SceneFarCks<B>> : RadTraits<P, B> {};

// The scene's transport RHS under a policy; FP32 is a compile-time choice of
// the calling kernel, so each kernel holds one contraction body.  The FP64
// policy keeps the reference's operation order; the mixed policy uses the
// factored form (kp_geometry_f32.cuh).
template<class P, bool FP32, class S>
__device__ __forceinline__ Ray policy_rhs(const ImageConsts& c, const Ray& X) {
    return S::template rhs<P::kMixed, FP32>(c, X);
}

// ---------------------------------------------------------------- RK jobs
// Runs one RK job from S with signed step h.  Outputs: next (endpoint), mid
// (sample point: the first half step for SD, the endpoint otherwise) and err
// (SD / CK only).  The stage arithmetic is the reference's (see file header).
// Cash-Karp attempt with the reference's stage coefficients (rk4.hpp:171-228).
template<class P, bool FP32, class SC>
__device__ __noinline__ void ck_job(const ImageConsts& c, const Ray& S, double h, Ray& next,
                                    Ray& mid, double& err) {
    {
        const Ray k1 = policy_rhs<P, FP32, SC>(c, S);
        Ray t;
        ray_axpy(t, S, h * 1.0 / 5.0, k1);
        const Ray k2 = policy_rhs<P, FP32, SC>(c, t);
        {
            const Ray* const kk[2] = {&k1, &k2};
            const double cc[2] = {3.0 / 40.0, 9.0 / 40.0};
            ray_lincomb<2>(t, S, h, kk, cc);
        }
        const Ray k3 = policy_rhs<P, FP32, SC>(c, t);
        {
            const Ray* const kk[3] = {&k1, &k2, &k3};
            const double cc[3] = {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0};
            ray_lincomb<3>(t, S, h, kk, cc);
        }
        const Ray k4 = policy_rhs<P, FP32, SC>(c, t);
        {
            const Ray* const kk[4] = {&k1, &k2, &k3, &k4};
            const double cc[4] = {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0};
            ray_lincomb<4>(t, S, h, kk, cc);
        }
        const Ray k5 = policy_rhs<P, FP32, SC>(c, t);
        {
            const Ray* const kk[5] = {&k1, &k2, &k3, &k4, &k5};
            const double cc[5] = {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0,
                                  253.0 / 4096.0};
            ray_lincomb<5>(t, S, h, kk, cc);
        }
        const Ray k6 = policy_rhs<P, FP32, SC>(c, t);
        {
            const Ray* const kk[4] = {&k1, &k3, &k4, &k6};
            const double cc[4] = {37.0 / 378.0, 250.0 / 621.0, 125.0 / 594.0, 512.0 / 1771.0};
            ray_lincomb<4>(next, S, h, kk, cc);
        }
        Ray fourth;
        {
            const Ray* const kk[5] = {&k1, &k3, &k4, &k5, &k6};
            const double cc[5] = {2825.0 / 27648.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0,
                                  1.0 / 4.0};
            ray_lincomb<5>(fourth, S, h, kk, cc);
        }
        err = control_error(next, fourth, max_val(c.tolerance, kTolFloor));
        mid = next;
    }
}

// Far-field RK chains of the mixed policy (Kerr-Schild scene).  Beyond the
// radiating sphere the transports change the ray by ~M/r^2 per unit step, so
// their FP32 rounding is far below the step-doubling tolerance; the state,
// the position derivative (= k) and every chain endpoint stay FP64.  What
// only feeds the FP32 contraction or sums FP32 derivatives is carried in
// FP32: the stage inputs x, k, e1, e2 (formed from the chain base's FP32
// copy) and the accumulator of dk, de1, de2.  Per stage that leaves four
// FP32->FP64 conversions and eight FP64 FMAs (k of the next stage input, the
// position accumulator) around the contraction, where converting FP64 stage
// states took 28 conversions and 48 FP64 operations.  Stage order,
// coefficients and the k1 reuse of step doubling are the reference's
// (rk4.hpp:37-59, 108-161).
struct ChainF {
    float x[3];      // x^1..x^3 of the stage input
    float q[3][4];   // k, e1, e2 of the stage input
};

__device__ __forceinline__ void chain_base_f(const Ray& B, ChainF& b) {
#pragma unroll
    for (int i = 0; i < 3; ++i) b.x[i] = float(B.x.v[i + 1]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        b.q[0][i] = float(B.k.v[i]);
        b.q[1][i] = float(B.e1.v[i]);
        b.q[2][i] = float(B.e2.v[i]);
    }
}

// State of one RK4 chain between its stages: the next stage input (FP32,
// with its k in FP64 as the position derivative) and the accumulators.
struct ChainAcc {
    ChainF X;      // stage input
    D4 Xk;         // k of the stage input, FP64: the position derivative
    D4 Ax;         // position accumulator, FP64
    float Aq[3][4];
};

// Folds stage st's derivative kq into the chain of step hc from B (base b):
// acc = ((k1 + 2 k2) + 2 k3) + k4, then the next stage input
// B + cc * (this stage's derivative).
__device__ __forceinline__ void chain_stage_f(ChainAcc& C, const ChainF& b, const Ray& B, double hc, int st,
                                              const float (&kq)[3][4]) {
    if (st == 0) {
        C.Ax = C.Xk;
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Aq[w][i] = kq[w][i];
    } else {
        const double wd = st == 3 ? 1.0 : 2.0;
        const float wf = st == 3 ? 1.0f : 2.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) C.Ax.v[i] = C.Ax.v[i] + C.Xk.v[i] * wd;
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.Aq[w][i] = C.Aq[w][i] + kq[w][i] * wf;
    }
    if (st < 3) {
        const double cc = st < 2 ? 0.5 * hc : hc;
        const float cf = float(cc);
#pragma unroll
        for (int i = 0; i < 3; ++i) C.X.x[i] = b.x[i] + C.X.q[0][i + 1] * cf;
#pragma unroll
        for (int i = 0; i < 4; ++i) C.Xk.v[i] = B.k.v[i] + double(kq[0][i]) * cc;
#pragma unroll
        for (int w = 0; w < 3; ++w)
#pragma unroll
            for (int i = 0; i < 4; ++i) C.X.q[w][i] = b.q[w][i] + kq[w][i] * cf;
    }
}

__device__ __forceinline__ void chain_end_f(const ChainAcc& C, const Ray& B, double hc, Ray& end) {
    const double h6 = hc / 6.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        end.x.v[i] = B.x.v[i] + C.Ax.v[i] * h6;
        end.k.v[i] = B.k.v[i] + double(C.Aq[0][i]) * h6;
        end.e1.v[i] = B.e1.v[i] + double(C.Aq[1][i]) * h6;
        end.e2.v[i] = B.e2.v[i] + double(C.Aq[2][i]) * h6;
    }
}

// One RK4 chain of step hc from B.
__device__ __forceinline__ void far_chain_f(const ImageConsts& c, const Ray& B, double hc, Ray& end) {
    const float M = float(c.mass), a = float(c.spin);
    ChainF b;
    chain_base_f(B, b);
    ChainAcc C;
    C.X = b;
    C.Xk = B.k;
#pragma unroll 1
    for (int st = 0; st < 4; ++st) {
        float kq[3][4];
        ks_transport_factored<float>(M, a, C.X.x[0], C.X.x[1], C.X.x[2], C.X.q, kq);
        chain_stage_f(C, b, B, hc, st, kq);
    }
    chain_end_f(C, B, hc, end);
}

// Step-doubling attempt from far_chain_f pieces.  The full-step chain starts
// from S like the first half chain and reuses its first derivative, so the
// two run interleaved, stage by stage: their contractions are independent,
// which gives the scheduler two dependency chains per lane.  Then the
// second half chain from the half-step state.  Each chain's arithmetic is
// the sequential chain's (same operations in the same order).
__device__ __forceinline__ void far_sd_f(const ImageConsts& c, const Ray& S, double h, Ray& next, Ray& mid,
                                         double& err) {
    const float M = float(c.mass), a = float(c.spin);
    ChainF b;
    chain_base_f(S, b);
    const double hh = 0.5 * h;
    ChainAcc H, F;
    H.X = b;
    H.Xk = S.k;
    F.X = b;
    F.Xk = S.k;
    Ray full;
    {
        float kq[3][4];
        ks_transport_factored<float>(M, a, b.x[0], b.x[1], b.x[2], b.q, kq);
        chain_stage_f(H, b, S, hh, 0, kq);
        chain_stage_f(F, b, S, h, 0, kq);
    }
#pragma unroll 1
    for (int st = 1; st < 4; ++st) {
        float kh[3][4], kf[3][4];
        ks_transport_factored<float>(M, a, H.X.x[0], H.X.x[1], H.X.x[2], H.X.q, kh);
        ks_transport_factored<float>(M, a, F.X.x[0], F.X.x[1], F.X.x[2], F.X.q, kf);
        chain_stage_f(H, b, S, hh, st, kh);
        chain_stage_f(F, b, S, h, st, kf);
    }
    chain_end_f(H, S, hh, mid);
    chain_end_f(F, S, h, full);
    far_chain_f(c, mid, hh, next);
    err = control_error(full, next, max_val(c.tolerance, kTolFloor));
}

// Step-doubling attempt, RK4 step or composed RK4 pair from the FP32
// chains; outputs as rk_job's.
__device__ __forceinline__ void far_job_f(int kind, const ImageConsts& c, const Ray& S, double h, Ray& next,
                                          Ray& mid, double& err) {
    err = 0.0;
    if (kind == kRkSD) {
        far_sd_f(c, S, h, next, mid, err);
        return;
    }
    if (kind == kRkRK4) {
        far_chain_f(c, S, h, next);
        mid = next;
        return;
    }
    Ray R2;
    far_chain_f(c, S, 0.5 * h, R2);
    far_chain_f(c, R2, 0.5 * h, next);
    mid = next;
}

// Step-doubling attempt, RK4 step or composed RK4 pair as a stage loop around
// one RHS site.  Out of line: the caller's control state is saved once per
// job and the stage loop has the register file to itself.
template<class P, bool FP32, class SC>
__device__ __noinline__ void rk_job(int kind, const ImageConsts& c, const Ray& S, double h,
                                    Ray& next, Ray& mid, double& err) {
    if (kind == kRkCK) {
        ck_job<P, FP32, SC>(c, S, h, next, mid, err);
        return;
    }
    if constexpr (FP32 && SC::kCksRhs) {
        if (SC::chart_active(c)) {
            far_job_f(kind, c, S, h, next, mid, err);
            return;
        }
    }
    // Stage schedule (see file header): SD = half chain (4), second half
    // chain (4), full chain (3); RK4 = 4; RK4x2 = 4 + 4.
    const int nstage = kind == kRkSD ? 11 : (kind == kRkRK4 ? 4 : 8);
    const double hs = kind == kRkSD ? h * 0.5 : (kind == kRkRK4x2 ? h * 0.5 : h);  // step of the first chain
    const double hh_s = 0.5 * hs;
    const double h6_s = hs / 6.0;
    const double hh_f = 0.5 * h;
    const double h6_f = h / 6.0;
    Ray X = S;   // RHS input
    Ray A;       // stage accumulator
    Ray R1;      // SD: k1 of S, then the two-half endpoint
    Ray R2;      // SD / RK4x2: the first chain's endpoint (half step)
#pragma unroll 1
    for (int st = 0; st < nstage; ++st) {
        const Ray k = policy_rhs<P, FP32, SC>(c, X);
        // position of this stage inside its 4-stage RK4 chain
        const int cs = st < 4 ? st : (st < 8 ? st - 4 : st - 7);
        const bool full_chain = kind == kRkSD && st >= 8;
        const bool second_chain = st >= 4 && st < 8;
        const double hh = full_chain ? hh_f : hh_s;
        const double hl = full_chain ? h : hs;       // last-stage step of the chain
        const double h6 = full_chain ? h6_f : h6_s;
        const Ray& base = second_chain ? R2 : S;
        if (cs == 0) {
            A = k;
            if (st == 0 && kind == kRkSD) R1 = k;
            ray_axpy(X, base, hh, k);
        } else if (cs == 1) {
            ray_acc(A, k, 2.0);
            ray_axpy(X, base, hh, k);
        } else if (cs == 2) {
            ray_acc(A, k, 2.0);
            ray_axpy(X, base, hl, k);
        } else {
            ray_add(A, k);
            if (st == 3) {
                if (kind == kRkRK4) {
                    ray_axpy(next, S, h6, A);
                } else {
                    ray_axpy(R2, S, h6, A);  // half step endpoint
                    X = R2;
                }
            } else if (st == 7) {
                if (kind == kRkRK4x2) {
                    ray_axpy(next, R2, h6, A);
                } else {
                    // two_half = R2 + (hs/6) A; start the full chain from k1 of S
                    Ray two_half;
                    ray_axpy(two_half, R2, h6, A);
                    A = R1;
                    ray_axpy(X, S, hh_f, R1);
                    R1 = two_half;
                    // the full chain's first stage (k1) is already done: advance
                    // its position counter by running stages 8..10 as cs 1..3.
                }
            } else {  // st == 10: full step endpoint
                Ray full;
                ray_axpy(full, S, h6_f, A);
                err = control_error(full, R1, max_val(c.tolerance, kTolFloor));
                next = R1;
                mid = R2;
            }
        }
    }
    if (kind == kRkRK4 || kind == kRkRK4x2) {
        mid = next;
        err = 0.0;
    }
}

}  // namespace kp
