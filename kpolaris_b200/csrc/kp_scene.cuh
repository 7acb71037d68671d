// kp_scene.cuh -- what the wavefront engine needs of a spacetime and its
// plasma, as compile-time scenes:
//   SceneRiaf:  Cartesian Kerr-Schild metric, analytic RIAF plasma;
//   SceneGrmhd: FMKS metric, GRMHD grid plasma.
// Each scene gives the radial coordinate of the pass logic
// (metric_domain_radius, src/geodesic/metric_domain.hpp:160-172), the
// transport right-hand side, the pinhole camera ray, and the metric at a
// point for the end-of-ray overlaps and diagnostics
// (src/geodesic/pass_b.hpp:87-98, 1096-1113).
#pragma once

#include "kp_bl.cuh"
#include "kp_camera.cuh"
#include "kp_chart.cuh"
#include "kp_fmks.cuh"
#include "kp_geometry_f32.cuh"
#include "kp_grmhd.cuh"
#include "kp_trace_fp64.cuh"

#include <type_traits>

namespace kp {

// Mixed policy marker types live in kp_engine.cuh; the scenes only need to
// know whether FP32 contraction was requested.
template<bool MIXED, bool FP32>
__device__ __forceinline__ Ray riaf_rhs(double mass, double spin, const Ray& X) {
    if constexpr (MIXED && FP32) return ks_rhs_factored<float>(mass, spin, X);
    else if constexpr (MIXED) return ks_rhs_factored<double>(mass, spin, X);
    else return ks_rhs(mass, spin, X);
}

struct SceneRiaf {
    static constexpr bool kSlowLight = false;
    static constexpr bool kCksRhs = true;     // transport is the Cartesian Kerr-Schild RHS
    static constexpr bool kFarChart = false;  // records and integration share one chart
    __device__ static bool chart_active(const ImageConsts&) { return true; }
    struct Metric {
        KSMetricPoint w;
        __device__ double dot(const D4& u, const D4& v) const { return ks_dot_at(w, u, v); }
    };
    __device__ static double radius(const ImageConsts& c, const D4& X) { return ks_radius(c.spin, X); }
    template<bool MIXED, bool FP32>
    __device__ static Ray rhs(const ImageConsts& c, const Ray& X) {
        return riaf_rhs<MIXED, FP32>(c.mass, c.spin, X);
    }
    __device__ static Ray camera(const ImageConsts& c, const CameraFrame& f, int pixel) {
        return camera_ray(c, f, pixel);
    }
    __device__ static Metric metric_at(const ImageConsts& c, const D4& X) { return Metric{ks_point(c.mass, c.spin, X)}; }
};

// initialize_pinhole_camera_ray (camera.hpp:485-513) in Boyer-Lindquist
// coordinates, from the image's precomputed tetrad (normalize_spacelike and
// orthogonalize_spacelike, camera.hpp:207-228).
static __device__ __noinline__ Ray bl_camera_ray(const ImageConsts& c, const CameraFrame& f, int pixel) {
    const BLMetricPoint w = bl_point(c.mass, c.spin, f.x);
    double sx = 0.0, sy = 0.0;
    pixel_offsets(pixel, c, sx, sy);
    const double spatial_norm = sqrt(1.0 + sx * sx + sy * sy);
    const double kt1 = sx / spatial_norm;
    const double kt2 = sy / spatial_norm;
    const double kt3 = 1.0 / spatial_norm;
    D4 sd;
    for (int mu = 0; mu < 4; ++mu)
        sd.v[mu] = f.e1.v[mu] * kt1 + f.e2.v[mu] * kt2 + f.e3.v[mu] * kt3;
    Ray s;
    s.x = f.x;
    for (int mu = 0; mu < 4; ++mu) s.k.v[mu] = f.e0.v[mu] * 1.0 + sd.v[mu];
    D4 e1 = d4_sub_scaled(f.e1, sd, kt1);
    {
        const double n2 = bl_dot_at(w, e1, e1);
        if (!(n2 <= 0.0)) e1 = d4_scale(e1, 1.0 / sqrt(n2));
    }
    D4 e2 = d4_sub_scaled(f.e2, sd, kt2);
    {
        const double denom = bl_dot_at(w, e1, e1);
        if (abs_val(denom) > kTiny) e2 = d4_sub_scaled(e2, e1, bl_dot_at(w, e2, e1) / denom);
        const double n2 = bl_dot_at(w, e2, e2);
        if (!(n2 <= 0.0)) e2 = d4_scale(e2, 1.0 / sqrt(n2));
    }
    s.e1 = e1;
    s.e2 = e2;
    return s;
}

// The analytic RIAF in Boyer-Lindquist coordinates (the reference's RIAF
// backend, src/image/riaf.cpp:21-45, over KerrBoyerLindquistMetric): radius
// x^1 (metric_domain_radius, src/geodesic/metric_domain.hpp:160-172), the
// specialised BL transport in FP64 under both policies, the camera from the
// host's BL tetrad.
struct SceneRiafBL {
    static constexpr bool kSlowLight = false;
    static constexpr bool kCksRhs = false;
    static constexpr bool kFarChart = false;
    __device__ static bool chart_active(const ImageConsts&) { return false; }
    struct Metric {
        BLMetricPoint p;
        __device__ double dot(const D4& u, const D4& v) const { return bl_dot_at(p, u, v); }
    };
    __device__ static double radius(const ImageConsts&, const D4& X) { return X.v[1]; }
    template<bool MIXED, bool FP32>
    __device__ static Ray rhs(const ImageConsts& c, const Ray& X) {
        return bl_rhs(c.mass, c.spin, X);
    }
    __device__ static Ray camera(const ImageConsts& c, const CameraFrame& f, int pixel) {
        return bl_camera_ray(c, f, pixel);
    }
    __device__ static Metric metric_at(const ImageConsts& c, const D4& X) {
        return Metric{bl_point(c.mass, c.spin, X)};
    }
};

// initialize_pinhole_camera_ray (camera.hpp:485-513) in FMKS, from the
// image's precomputed tetrad.
static __device__ __noinline__ Ray fmks_camera_ray(const ImageConsts& c, const CameraFrame& f, int pixel) {
    double g[4][4];
    fmks_gcov(c.fmks, f.x, g);
    double sx = 0.0, sy = 0.0;
    pixel_offsets(pixel, c, sx, sy);
    const double spatial_norm = sqrt(1.0 + sx * sx + sy * sy);
    const double kt1 = sx / spatial_norm, kt2 = sy / spatial_norm, kt3 = 1.0 / spatial_norm;
    Ray s;
    s.x = f.x;
    D4 sd;
    for (int i = 0; i < 4; ++i) sd.v[i] = f.e1.v[i] * kt1 + f.e2.v[i] * kt2 + f.e3.v[i] * kt3;
    for (int i = 0; i < 4; ++i) s.k.v[i] = f.e0.v[i] + sd.v[i];
    for (int i = 0; i < 4; ++i) s.e1.v[i] = f.e1.v[i] - sd.v[i] * kt1;
    {
        const double n2 = dot_gm(g, s.e1, s.e1);
        if (n2 > 0.0) {
            const double inv = 1.0 / sqrt(n2);
            for (int i = 0; i < 4; ++i) s.e1.v[i] *= inv;
        }
    }
    for (int i = 0; i < 4; ++i) s.e2.v[i] = f.e2.v[i] - sd.v[i] * kt2;
    {
        const double denom = dot_gm(g, s.e1, s.e1);
        if (abs_val(denom) > kTiny) {
            const double k = dot_gm(g, s.e2, s.e1) / denom;
            for (int i = 0; i < 4; ++i) s.e2.v[i] -= s.e1.v[i] * k;
        }
        const double n2 = dot_gm(g, s.e2, s.e2);
        if (n2 > 0.0) {
            const double inv = 1.0 / sqrt(n2);
            for (int i = 0; i < 4; ++i) s.e2.v[i] *= inv;
        }
    }
    return s;
}

struct SceneGrmhd {
    static constexpr bool kSlowLight = false;
    static constexpr bool kCksRhs = false;
    static constexpr bool kFarChart = false;
    __device__ static bool chart_active(const ImageConsts&) { return false; }
    struct Metric {
        double g[4][4];
        __device__ double dot(const D4& u, const D4& v) const { return dot_gm(g, u, v); }
    };
    __device__ static double radius(const ImageConsts&, const D4& X) { return fmks_radius(X); }
    // FP64 everywhere (an FP32 FMKS connection puts its rounding noise into
    // the step-doubling error norm); the mixed policy uses the factored form
    template<bool MIXED, bool FP32>
    __device__ static Ray rhs(const ImageConsts& c, const Ray& X) {
        if constexpr (MIXED) {
            return fmks_rhs_factored(c.fmks, X);
        } else {
            return fmks_rhs(c.fmks, X);
        }
    }
    __device__ static Ray camera(const ImageConsts& c, const CameraFrame& f, int pixel) {
        return fmks_camera_ray(c, f, pixel);
    }
    __device__ static Metric metric_at(const ImageConsts& c, const D4& X) {
        Metric m;
        fmks_gcov(c.fmks, X, m.g);
        return m;
    }
};

// Slow light on the GRMHD grid: the same FMKS geometry; the plasma of a
// sample comes from the resident snapshots at t_obs + x^0
// (ImageConsts::series).  A radiating sample whose time lies outside the
// resident snapshots ends the ray (slow_light_time_exhausted).
struct SceneGrmhdSlow : SceneGrmhd {
    static constexpr bool kSlowLight = true;
    __device__ static bool time_resident(const ImageConsts& c, const Ray& sample) {
        return series_holds(c, series_time(c, sample));
    }
};

// A GRMHD scene as the mixed policy's far kernel runs it: beyond the
// radiating sphere no plasma is sampled, so the ray is integrated in
// Cartesian Kerr-Schild (the RIAF scene's FP32 stage chains, with the
// policy's step control) and converted at the phase boundary
// (kp_chart.cuh).  Records, cameras and the end of a ray stay in FMKS:
// to_phase converts a claimed ray, to_record converts it back before it is
// parked or finished.  Phase decisions use the radius its record will hold.
//
// Only step-doubling images change chart: with adaptive steps the far
// field's truncation error stays under the tolerance in either chart, while
// a fixed step's error depends on the chart it is taken in.  Fixed-step and
// Cash-Karp images keep FMKS in the same kernel (chart_active false: the
// base scene's radius and RHS, no conversion).
template<class Base>
struct SceneFarCks : Base {
    static constexpr bool kCksRhs = true;
    static constexpr bool kFarChart = true;
    __device__ static bool chart_active(const ImageConsts& c) { return c.adaptive && c.integrator != 1; }
    __device__ static double radius(const ImageConsts& c, const D4& X) {
        return chart_active(c) ? cks_record_radius(c.spin, X) : Base::radius(c, X);
    }
    // reached only with the chart inactive (the active chart runs far_job_f)
    template<bool MIXED, bool FP32>
    __device__ static Ray rhs(const ImageConsts& c, const Ray& X) {
        return Base::template rhs<MIXED, false>(c, X);
    }
    // out of line: conversions happen a few times per ray, and inlined at
    // each claim, park and finish site they crowd the kernel's registers
    static __device__ __noinline__ Ray to_phase(const ImageConsts& c, const Ray& S) {
        return fmks_to_cks(c.fmks, c.spin, S);
    }
    static __device__ __noinline__ Ray to_record(const ImageConsts& c, const Ray& S, double x3_ref) {
        return cks_to_fmks(c.fmks, c.spin, S, x3_ref);
    }
};

// End of a ray for any scene: screen overlaps with the camera basis,
// observer-basis Stokes (stokes_rotation.hpp:39-57) and the closure
// diagnostics (finish_ray in kp_trace_fp64.cuh for the RIAF plain kernel).
template<class S, int NF>
__device__ __forceinline__ void finish_ray_scene(const ImageConsts& c, const Ray& cam, const Ray& state, int passed_b,
                                                 Stokes4<double> (&stokes)[NF], PixelOut& o,
                                                 double (&obs)[NF][4]) {
    if constexpr (std::is_same<S, SceneRiaf>::value) {
        // the plain kernel's own code, so the FP64 policy stays bit-identical to it
        finish_ray<double, NF>(c, cam, state, passed_b, stokes, o, obs);
        return;
    }
    const typename S::Metric m = S::metric_at(c, state.x);
    if (passed_b) {
        o.r11 = m.dot(cam.e1, state.e1);
        o.r12 = m.dot(cam.e1, state.e2);
        o.r21 = m.dot(cam.e2, state.e1);
        o.r22 = m.dot(cam.e2, state.e2);
    } else if constexpr (S::kSlowLight) {
        // a slow-light ray without pass B keeps zero overlaps
        // (initialize_slow_light_states_metric, slow_light_driver.hpp:393-399)
        o.r11 = o.r12 = o.r21 = o.r22 = 0.0;
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
    o.final_null = m.dot(state.k, state.k);
    double fe = abs_val(m.dot(state.k, state.k));
    fe = max_val(fe, abs_val(m.dot(state.e1, state.k)));
    fe = max_val(fe, abs_val(m.dot(state.e2, state.k)));
    fe = max_val(fe, abs_val(m.dot(state.e1, state.e1) - 1.0));
    fe = max_val(fe, abs_val(m.dot(state.e2, state.e2) - 1.0));
    fe = max_val(fe, abs_val(m.dot(state.e1, state.e2)));
    o.frame_error = fe;
}

}  // namespace kp
