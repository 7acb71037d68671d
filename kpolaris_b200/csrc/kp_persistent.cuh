// kp_persistent.cuh -- the wavefront image kernels.  Lanes claim rays from a
// phase queue (fresh camera rays, then ray ids handed over by other phases),
// advance them one RK job per loop iteration through the pass-A / crossing /
// pass-B control machine, and either finish the pixel or park the ray's
// record in HBM for another phase (or for its own next launch when an iteration
// budget is set).  See kp_engine.cuh for the RK jobs.
//
// Three phases, one kernel each, so that the lanes of a warp run the same
// code and each kernel's instruction working set stays small:
//   far     rays beyond ImageConsts::fp32_radius, pass A and pass B: pure
//           transport (no surface lies within a step, no plasma is sampled);
//   near-A  pass A inside: the surface-crossing search, no radiation;
//   near-B  pass B inside: radiative transfer, Stokes vectors in registers.
//
// Parking happens only at the top of the pass-A or pass-B loop, where the
// whole state is the record: a ray resumed from its record takes exactly the
// arithmetic it would have taken without parking, so results do not depend on
// how rays are distributed over launches, lanes or warps.
#pragma once

#include <cstddef>

#include "kp_engine.cuh"

namespace kp {

enum : int { kEndA = 7 };

// Control state of one ray (17 doubles + 17 ints, 208 bytes), in three
// parts: what every phase uses; what only the pass-A phases (far and
// near-A) use; the surface-crossing search (near-A).  A phase kernel moves
// only the parts it uses between its registers and the record, so the
// others hold no registers there; the record keeps them as the last phase
// that used them left them.
struct LaneState {
    // adaptive attempt sequence (rk4.hpp:108-161)
    double h_try, req_h, ctl_min, ctl_max;
    double h_current;
    // pass B (pass_b.hpp:940-1114)
    double cap, hB, start_r;
    int job, pixel, mode, in_b;
    int attempt, rk_kind;
    int pa_steps, reason;
    int steps, reached;
    // pass A (pass_b.hpp:786-938)
    double old_r;
    // far-phase chart scenes: the FMKS azimuth the ray entered the far
    // phase with, and whether S (here and in a record parked for the far
    // phase itself) holds the far phase's chart
    double x3_ref;
    int n, entered, inside;
    int chart;
    // surface-crossing search (pass_a_core.hpp:94-197)
    double lo, hi, flo, fhi, full_h, surf, trial;
    int cross_reason, iter, use_secant;
};
static_assert(sizeof(LaneState) <= sizeof(((RayRecord*)nullptr)->st), "LaneState must fit its record slot");
static_assert(offsetof(LaneState, old_r) % 8 == 0 && offsetof(LaneState, lo) % 8 == 0, "parts are whole doubles");

// Bytes of LaneState a phase kernel moves: near-B runs no pass-A step and
// never holds a far chart, far runs no crossing search, and near-A's
// crossing search works on the crossing part in the record itself (one
// search per ray, a few iterations).
template<int PHASE>
constexpr size_t kLaneStateBytes = PHASE == kPhaseNearB ? offsetof(LaneState, old_r) : offsetof(LaneState, lo);

template<class LS>
__device__ __forceinline__ void begin_adaptive(LS& L, double requested, double min_step, double max_step) {
    L.req_h = requested;
    L.ctl_min = min_step;
    L.ctl_max = max_step;
    double h = min_val(max_val(abs_val(requested), min_step), max_step);
    if (requested < 0.0) h = -h;
    L.h_try = h;
    L.attempt = 0;
}

// Step growth after an accepted attempt (rk4.hpp:130-142).  With
// tol >= 64 err the factor 0.9 (tol/err)^0.2 is at least 2.07 and clamps to
// 2, so pow is evaluated only below that ratio (same result).
__device__ __forceinline__ double accepted_next_h(double h, double err, double tol, double min_step,
                                                  double max_step, double requested) {
    double factor = 2.0;
    if (err > 0.0 && !(tol >= 64.0 * err)) {
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
template<class LS>
__device__ __forceinline__ int rejected_attempt(LS& L, double err, double tol) {
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

template<class LS>
__device__ __forceinline__ void issue_step(LS& L, const ImageConsts& c, double h, double min_step, double max_step) {
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

// Warp-aggregated append of the ids of the lanes in `mask` to a queue.
__device__ __forceinline__ void queue_push(unsigned* ids, unsigned* count, bool push, unsigned id) {
    const unsigned FULL = 0xffffffffu;
    const unsigned m = __ballot_sync(FULL, push);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(count, unsigned(__popc(m)));
    base = __shfl_sync(FULL, base, leader);
    if (push) ids[base + __popc(m & ((1u << lane) - 1u))] = id;
}

// Initial control state of a camera ray at the top of pass A
// (pass_b.hpp:786-792).
template<class SC>
__device__ __forceinline__ void start_ray(LaneState& st, Ray& S, const JobDesc* J, int job, int pixel) {
    memset(&st, 0, sizeof(st));
    st.job = job;
    st.pixel = pixel;
    S = SC::camera(J->c, J->frame, pixel);
    st.reason = kMaxSteps;
    st.h_current = -abs_val(J->c.step);
    st.mode = kAStep;
    st.rk_kind = -1;
}

// Seeds the rays of newly admitted jobs: one thread per ray writes the ray's
// initial record (pass-A loop top) and appends its id to the far queue.
// entries: (job slot, first ray id, pixel count) with prefix sums of the
// counts in `prefix` (nentries + 1 values).
template<class SC>
__device__ __forceinline__ void seed_body(const JobDesc* jobs, const SeedEntry* entries, const long long* prefix,
                                          int nentries, RayRecord* pool, unsigned* far_ids,
                                          unsigned* far_count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < prefix[nentries];
    unsigned id = 0;
    if (live) {
        int lo = 0, hi = nentries - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= i) lo = mid; else hi = mid - 1;
        }
        const SeedEntry e = entries[lo];
        const int pixel = int(i - prefix[lo]);
        id = unsigned(e.ray_base + pixel);
        LaneState st;
        Ray S;
        start_ray<SC>(st, S, &jobs[e.slot], e.slot, pixel);
        RayRecord& rec = pool[id];
        rec.S = S;
        memcpy(rec.st, &st, sizeof(LaneState));
    }
    queue_push(far_ids, far_count, live, id);
}

// Phase that advances a ray from the top of its pass-A or pass-B loop.
__device__ __forceinline__ int phase_of(const ImageConsts& c, int in_b, double r_bl) {
    if (r_bl > c.fp32_radius) return kPhaseFar;
    return in_b ? kPhaseNearB : kPhaseNearA;
}

// The scene a ray is finished in: a far-phase chart scene hands the ray
// back to the scene its records use.
template<class SC>
struct RecordScene {
    using type = SC;
};
template<class B>
struct RecordScene<SceneFarCks<B>> {
    using type = B;
};

template<class P, int NF, int PHASE, class SC = SceneRiaf>
__device__ __forceinline__ void persistent_body(const WaveDesc& W) {
    constexpr bool kFar = PHASE == kPhaseFar;
    constexpr bool kPassA = PHASE != kPhaseNearB;   // pass-A steps run here
    constexpr bool kPassB = PHASE != kPhaseNearA;   // pass-B steps run here
    constexpr bool kCross = PHASE == kPhaseNearA;   // surface-crossing search
    constexpr bool kRad = PHASE == kPhaseNearB;     // radiative transfer (Stokes in registers)
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    using RT = RadTraits<P, SC>;
    LaneState st;
    st.mode = kIdle;
    st.job = -1;
    st.rk_kind = -1;
    Ray S;
    typename RT::Stokes stokes[NF];
    unsigned my_id = 0;
    // the crossing search's best state (near-A) lives in the record's Stokes
    // slot, which pass A leaves unused: it holds no registers between the
    // search's iterations
    auto best = [&]() -> Ray& { return *reinterpret_cast<Ray*>(W.pool[my_id].stokes); };
    // ... and its bracket, the crossing part of the control state, in the record
    auto cs = [&]() -> LaneState& { return *reinterpret_cast<LaneState*>(W.pool[my_id].st); };
    static_assert(sizeof(((RayRecord*)nullptr)->stokes) >= sizeof(Ray), "the Stokes slot holds a ray");
    int exhausted = 0;
    long long lane_jobs = 0;
    const JobDesc* J = nullptr;
    const long long nfresh = W.fresh_end - W.fresh_begin;
    const long long total_in = nfresh + (long long)(W.in_ids ? *W.in_count : 0u);

#pragma unroll 1
    while (true) {
        // ------------------------------------------------------------ claim
        const bool want = !exhausted && st.mode == kIdle;
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
                    exhausted = 1;
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
                    start_ray<SC>(st, S, J, lo, int(id - J->ray_begin));
                    if constexpr (SC::kFarChart) {
                        if (SC::chart_active(J->c)) {
                            st.x3_ref = S.x.v[3];
                            S = SC::to_phase(J->c, S);
                            st.chart = 1;
                        }
                    }
                } else if (W.budget > 0 && lane_jobs >= W.budget) {
                    // past the budget: hand the id on untouched (below)
                    my_id = W.in_ids[k - nfresh];
                    forward = true;
                } else {
                    // a parked ray: resume from its record
                    my_id = W.in_ids[k - nfresh];
                    const RayRecord& rec = W.pool[my_id];
                    S = rec.S;
                    memcpy(&st, rec.st, kLaneStateBytes<PHASE>);
                    J = &W.jobs[st.job];
                    if constexpr (SC::kFarChart) {
                        // a record parked for this phase already holds its chart
                        if (!st.chart && SC::chart_active(J->c)) {
                            st.x3_ref = S.x.v[3];
                            S = SC::to_phase(J->c, S);
                            st.chart = 1;
                        }
                    }
                    if constexpr (kRad) memcpy(&stokes[0], rec.stokes, sizeof(stokes));
                }
            }
        }
        queue_push(W.out_ids[PHASE], W.out_count[PHASE], forward, my_id);
        const bool active = st.mode != kIdle;
        // The block leaves the loop together, so the barrier below is
        // reached by every thread of the block in every iteration.  A lane
        // that forwarded an id has more input to claim: it keeps the block
        // in the loop like an active lane.
        if (!__syncthreads_or(active || forward)) break;

        // ---------------------------------------------- control before the job
        int dest = -1;  // phase the ray is handed to (PHASE itself: its next launch)
        if constexpr (kPassA) {
            if (active && st.mode == kAStep && st.rk_kind < 0) {
                const ImageConsts& c = J->c;
                const double r_bl = SC::radius(c, S.x);
                const int want_phase = phase_of(c, 0, r_bl);
                if (want_phase != PHASE) {
                    dest = want_phase;
                } else if (W.budget > 0 && lane_jobs >= W.budget) {
                    dest = PHASE;
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
            if (active && dest < 0 && st.mode == kEndA) {
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
                    // pass B starts from zero Stokes, kept in the record until
                    // the ray reaches the radiating phase
#pragma unroll
                    for (int f = 0; f < NF; ++f) RT::zero(stokes[f]);
                    memcpy(W.pool[my_id].stokes, &stokes[0], sizeof(stokes));
                } else {
                    st.mode = kDone;
                }
            }
        }
        if (active && dest < 0 && st.mode == kBStep && st.rk_kind < 0) {
            const ImageConsts& c = J->c;
            if (st.reached || st.steps >= c.max_steps) {
                st.mode = kDone;
            } else {
                const double r_bl = SC::radius(c, S.x);
                const int want_phase = phase_of(c, 1, r_bl);
                if (want_phase != PHASE) {
                    dest = want_phase;
                } else if (W.budget > 0 && lane_jobs >= W.budget) {
                    dest = PHASE;
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
        const bool park = dest >= 0;
        if (park) {
            RayRecord& rec = W.pool[my_id];
            if constexpr (SC::kFarChart) {
                // leaving the phase: back to the records' chart; parked for
                // this phase (a tick budget): kept as is, so the ray resumes
                // bit for bit as if it had not been parked
                if (st.chart && dest != PHASE) {
                    rec.S = SC::to_record(J->c, S, st.x3_ref);
                    st.chart = 0;
                } else {
                    rec.S = S;
                }
            } else {
                rec.S = S;
            }
            memcpy(rec.st, &st, kLaneStateBytes<PHASE>);
            if constexpr (kRad) memcpy(rec.stokes, &stokes[0], sizeof(stokes));
        }
        // A lane past its budget keeps claiming and parks each claimed ray at
        // once, so every input ends the launch finished or in a queue.
#pragma unroll
        for (int d = 0; d < kPhases; ++d) queue_push(W.out_ids[d], W.out_count[d], dest == d, my_id);
        if (park) st.mode = kIdle;

        // ------------------------------------------------------------ RK job
        const bool run = !park && (st.mode == kAStep || st.mode == kACrossHi || st.mode == kACrossTrial ||
                                   st.mode == kBStep || st.mode == kBCamCross);
        // Mixed policy: FP32 stage chains in the far phase only.  Inside the
        // radiating sphere FP32 rounding in dk and de reaches the
        // step-doubling error estimate and reshapes the accepted-step
        // sequence the Faraday-thick transfer is sensitive to.  One RK call
        // site: the crossing search's job differs only in kind and step.
        constexpr bool fp32 = P::kMixed && kFar;
        Ray next, mid;
        double err = 0.0;
        if (run) {
            const bool crossing = kCross && (st.mode == kACrossHi || st.mode == kACrossTrial);
            const int kind = crossing ? (J->c.adaptive ? kRkRK4x2 : kRkRK4) : st.rk_kind;
            const double hj = crossing ? (st.mode == kACrossHi ? cs().full_h : cs().full_h * cs().trial) : st.h_try;
            rk_job<P, fp32, SC>(kind, J->c, S, hj, next, mid, err);
            if (++lane_jobs > (1LL << 30)) {
                st.reason = kInvalidState;
                st.mode = kDone;
                st.in_b = 0;
                atomicExch(W.status, 2);
            }
        }

        // The warps of a block finish their RK jobs together and run the
        // control and radiation code together: one code region at a time
        // per SM keeps it in the instruction cache.
        __syncthreads();

        // ----------------------------------------------- control after the job
        if (kPassA && run && st.mode == kAStep) {
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
                const double next_r = SC::radius(c, next.x);
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
                        if constexpr (kCross) {
                            cs().cross_reason = crossing;
                            cs().surf = crossing == kReachedInner ? c.inner_radius : c.outer_radius;
                            cs().full_h = used_h;
                            best() = S;
                            cs().lo = 0.0;
                            cs().hi = 1.0;
                            cs().flo = SC::radius(c, S.x) - cs().surf;
                            if (cs().flo == 0.0 || !finite_ray(next)) {
                                st.pa_steps += 1;  // the event keeps the first state
                                st.reason = crossing;
                                st.mode = kEndA;
                            } else {
                                st.mode = kACrossHi;
                            }
                        } else {
                            atomicExch(W.status, 3);  // surfaces lie inside the near phase
                            st.reason = kInvalidState;
                            st.mode = kDone;
                        }
                    } else {
                        S = next;
                        st.pa_steps += 1;
                        if (st.entered) st.inside += 1;
                        st.n += 1;
                    }
                }
            }
        } else if (kCross && run && (st.mode == kACrossHi || st.mode == kACrossTrial)) {
            const ImageConsts& c = J->c;
            bool finish = false;
            if (st.mode == kACrossHi) {
                if (!finite_ray(next)) {
                    finish = true;
                } else {
                    const double fhi = SC::radius(c, next.x) - cs().surf;
                    if (!(fhi == fhi) || abs_val(fhi) >= kLarge) {
                        finish = true;
                    } else if (fhi == 0.0) {
                        best() = next;
                        finish = true;
                    } else if ((cs().flo > 0.0) == (fhi > 0.0)) {
                        finish = true;
                    } else {
                        cs().fhi = fhi;
                        cs().iter = 0;
                        cs().use_secant = 1;
                    }
                }
            } else {
                const double ft = finite_ray(next) ? SC::radius(c, next.x) - cs().surf : 0.0;
                if (!finite_ray(next) || !(ft == ft) || abs_val(ft) >= kLarge) {
                    cs().hi = cs().trial;
                    cs().use_secant = 0;
                } else if (ft == 0.0) {
                    best() = next;
                    finish = true;
                } else if ((cs().flo > 0.0) == (ft > 0.0)) {
                    cs().lo = cs().trial;
                    cs().flo = ft;
                    best() = next;
                } else {
                    cs().hi = cs().trial;
                    cs().fhi = ft;
                }
                cs().iter += 1;
            }
            if (!finish && cs().iter >= 12) finish = true;
            if (finish) {
                S = best();
                st.pa_steps += 1;
                st.reason = cs().cross_reason;
                st.mode = kEndA;
            } else {
                const double width = cs().hi - cs().lo;
                double trial = (cs().lo + cs().hi) * 0.5;
                const double denom = cs().flo - cs().fhi;
                if (cs().use_secant && abs_val(denom) > kTiny) {
                    const double secant = cs().lo + width * cs().flo / denom;
                    const double g = width * 0.1;
                    if (secant > cs().lo + g && secant < cs().hi - g) trial = secant;
                }
                cs().trial = trial;
                st.mode = kACrossTrial;
            }
        } else if (kPassB && run && (st.mode == kBStep || st.mode == kBCamCross)) {
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
                            // the slow-light window kernel reports max_steps here
                            // (slow_light_driver.hpp:1172-1177)
                            st.reason = SC::kSlowLight ? kMaxSteps : kAdaptiveUnderflow;
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
                    const double s1 = SC::radius(c, next.x) - c.cam_radius;
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
                bool stopped = false;
                if (proceed) {
                    // radiation at the sample point (pass_b.hpp:1414-1496)
                    const double sample_r = SC::radius(c, sample.x);
                    const double next_r = SC::radius(c, next.x);
                    const double local_max_rs =
                        (c.max_radiation_step > 0.0 &&
                         (st.start_r <= c.outer_radius || sample_r <= c.outer_radius || next_r <= c.outer_radius))
                            ? c.max_radiation_step : 0.0;
                    if constexpr (kRad) {
                        // The frequency loops stay rolled: one copy of the
                        // coefficient and transfer code keeps the kernel's
                        // instruction working set small.
                        typename RT::Co co[NF];
                        typename RT::Sample ps = RT::none();
                        bool radiating = sample_r - c.inner_radius > 0.0 && sample_r < c.outer_radius;
                        if constexpr (SC::kSlowLight) {
                            // slow_light_driver.hpp:1295-1304: a radiating sample
                            // needs its fluid time among the resident snapshots;
                            // otherwise the ray ends where it stands
                            radiating = sample_r >= c.inner_radius && sample_r < c.outer_radius;
                            if (radiating && !SC::time_resident(c, sample)) {
                                st.reason = kSlowLightTimeExhausted;
                                st.mode = kDone;
                                stopped = true;
                            }
                        }
                        if (radiating && !stopped) ps = RT::sample(c, sample);
                        if (!stopped) {
                        const int nf = c.nfreq < NF ? c.nfreq : NF;
#pragma unroll 1
                        for (int f = 0; f < nf; ++f) {
                            co[f] = RT::coeffs(c, ps, f);
                            if (!c.faraday_rotation) co[f].rV = 0.0;
                        }
                        // Substep counts at h (required) and at h_current
                        // (predictive) in one pass: neither test changes h or
                        // h_current.  Over the image's frequencies, or over a
                        // separate step-control list (pass_b.hpp:1787-1833).
                        int required = 1, pred = 1;
                        const bool fused = c.nctl == 0;
#pragma unroll 1
                        for (int g = 0; g < (fused ? nf : c.nctl); ++g) {
                            typename RT::Co cg;
                            double dls;
                            if (fused) {
                                cg = co[g];
                                dls = c.dlambda_scale[g];
                            } else {
                                cg = RT::coeffs_ctl(c, ps, g);
                                if (!c.faraday_rotation) cg.rV = 0.0;
                                dls = c.ctl_dlambda_scale[g];
                            }
                            const int cand = radiation_substep_count(cg, h, dls, local_max_rs, c.max_radiation_depth,
                                                                     c.max_absorption_depth, c.max_faraday_depth);
                            required = cand > required ? cand : required;
                            const int pc = radiation_substep_count(cg, st.h_current, dls, local_max_rs,
                                                                   c.max_radiation_depth, c.max_absorption_depth,
                                                                   c.max_faraday_depth);
                            pred = pc > pred ? pc : pred;
                        }
                        if (required > 1 && h > c.min_step_abs * 1.0001) {
                            st.h_current = max_val(c.min_step_abs, h / double(required));
                            st.cap = st.h_current;
                        } else {
                            if (local_max_rs > 0.0 || c.max_radiation_depth > 0.0 || c.max_absorption_depth > 0.0 ||
                                c.max_faraday_depth > 0.0) {
                                st.cap = pred > 1 ? max_val(c.min_step_abs, st.h_current / double(pred)) : c.max_step;
                            } else {
                                st.cap = c.max_step;
                            }
                            if (h > 0.0) {
#pragma unroll 1
                                for (int f = 0; f < nf; ++f) RT::step(stokes[f], co[f], h, c, f);
                            }
                            S = next;
                            st.steps += 1;
                            if (crosses) st.reached = 1;
                        }
                        }  // !stopped
                    } else {
                        // Far phase: the sample lies outside the radiating
                        // sphere, every coefficient is zero and the transfer
                        // step leaves the Stokes vector unchanged; the step
                        // cap resolves to max_step (pass_b.hpp:1482-1486).
                        if (local_max_rs > 0.0 || (sample_r - c.inner_radius > 0.0 && sample_r < c.outer_radius)) {
                            atomicExch(W.status, 3);
                        }
                        st.cap = c.max_step;
                        S = next;
                        st.steps += 1;
                        if (crosses) st.reached = 1;
                    }
                    if (!stopped) {
                        st.mode = kBStep;
                        st.rk_kind = -1;
                    }
                }
            }
        }

        // ------------------------------------------------------------ finish
        if (!park && st.mode == kDone) {
            const ImageConsts& c = J->c;
            PixelOut o;
            o.pass_a_steps = st.pa_steps;
            o.steps = st.in_b ? st.steps : 0;
            int reason = st.reason;
            if (st.in_b) {
                if (st.reached) {
                    reason = kReachedCamera;
                } else if (reason != kAdaptiveUnderflow && reason != kSlowLightTimeExhausted) {
                    reason = kMaxSteps;
                }
            }
            o.reason = reason;
            const Ray cam = SC::camera(c, J->frame, st.pixel);
            double obs[NF][4];
            Stokes4<double> sd[NF];
            if constexpr (!kRad) {
                // only the radiating phase carries the Stokes vector: it is in the record
                if (st.in_b) memcpy(&stokes[0], W.pool[my_id].stokes, sizeof(stokes));
            }
#pragma unroll
            for (int f = 0; f < NF; ++f)
                sd[f] = st.in_b ? RT::result(stokes[f], c, f) : Stokes4<double>{0.0, 0.0, 0.0, 0.0};
            if constexpr (SC::kFarChart) {
                const Ray S_rec = st.chart ? SC::to_record(c, S, st.x3_ref) : S;
                finish_ray_scene<typename RecordScene<SC>::type, NF>(c, cam, S_rec, st.in_b, sd, o, obs);
            } else {
                finish_ray_scene<SC, NF>(c, cam, S, st.in_b, sd, o, obs);
            }
            store_stokes_n<NF>(J->out, st.pixel, J->npix, c.nfreq, obs);
            store_diagnostics(J->out, st.pixel, o);
            if constexpr (SC::kSlowLight) {
                if (!st.in_b) J->out.basis_identity_error[st.pixel] = 0.0;
            }
            if (W.job_done) atomicAdd(&W.job_done[st.job], 1u);
            st.mode = kIdle;
        }
    }
}

}  // namespace kp
