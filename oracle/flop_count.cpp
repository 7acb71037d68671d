// Algorithmic FP64 operation count of the reference's image algorithm
// (test/measurement infrastructure only).
//
// The reference's hot-path templates are instantiated with an op-counting
// scalar `Counted` (a double that tallies every + - * / sqrt and every
// transcendental call).  The RIAF model is wrapped so that the
// frequency-independent plasma state at a sample point (flow, field,
// density, temperature, angles) is counted once per sample and only the
// thermal-synchrotron fit per frequency -- the arithmetic the GPU kernels
// perform.  Output: JSON with totals per image and per category.
//
//   flop_count <config: 1|2> <n> [threads]
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <Kokkos_Core.hpp>

struct OpTally {
    unsigned long long add = 0, mul = 0, div = 0, sqrt = 0, trans = 0;
};
static thread_local OpTally* g_tally = nullptr;

struct Counted {
    double v;
    constexpr Counted() : v(0.0) {}
    constexpr Counted(double x) : v(x) {}
    explicit constexpr operator double() const { return v; }
    explicit constexpr operator int() const { return int(v); }
};
#define KP_T(field) \
    if (g_tally) ++g_tally->field
inline Counted operator+(Counted a, Counted b) { KP_T(add); return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { KP_T(add); return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { KP_T(mul); return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { KP_T(div); return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted& operator-=(Counted& a, Counted b) { a = a - b; return a; }
inline Counted& operator*=(Counted& a, Counted b) { a = a * b; return a; }
inline Counted& operator/=(Counted& a, Counted b) { a = a / b; return a; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }

namespace Kokkos {
inline Counted sqrt(Counted x) { KP_T(sqrt); return Counted(std::sqrt(x.v)); }
#define KP_TR(name) \
    inline Counted name(Counted x) { KP_T(trans); return Counted(std::name(x.v)); }
KP_TR(cbrt) KP_TR(exp) KP_TR(log) KP_TR(sin) KP_TR(cos) KP_TR(tan) KP_TR(tanh) KP_TR(acos)
KP_TR(atan)
inline Counted floor(Counted x) { return Counted(std::floor(x.v)); }
inline Counted ceil(Counted x) { return Counted(std::ceil(x.v)); }
inline Counted atan2(Counted y, Counted x) { KP_T(trans); return Counted(std::atan2(y.v, x.v)); }
inline Counted pow(Counted x, Counted y) { KP_T(trans); return Counted(std::pow(x.v, y.v)); }
#undef KP_TR
}  // namespace Kokkos

inline Counted sqrt(Counted x) { return Kokkos::sqrt(x); }

// Operation count of one transport right-hand side as the GPU kernels
// evaluate it: the CSE'd contraction of kpolaris_b200/csrc/kp_geometry.cuh,
// host-compiled here with `double` standing for the counting scalar.
#include <cstdint>
#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__
#define double Counted
#include "../kpolaris_b200/csrc/kp_geometry.cuh"
#undef double

static OpTally gpu_rhs_ops() {
    OpTally t;
    kp::Ray s;
    const double x[16] = {0, 40, 3, 12, 1, -0.9, 0.1, -0.3, 0, 0.1, 1, 0, 0, 0.2, 0, 1};
    for (int mu = 0; mu < 4; ++mu) {
        s.x.v[mu] = Counted(x[mu]);
        s.k.v[mu] = Counted(x[4 + mu]);
        s.e1.v[mu] = Counted(x[8 + mu]);
        s.e2.v[mu] = Counted(x[12 + mu]);
    }
    g_tally = &t;
    volatile double sink = kp::ks_rhs(Counted(1.0), Counted(0.9375), s).k.v[1].v;
    (void)sink;
    g_tally = nullptr;
    return t;
}

#define KPOLARIS_MAX_FREQUENCIES 4
#include "geodesic/pass_b.hpp"
#include "geometry/kerr_schild_cartesian.hpp"
#include "model/riaf.hpp"

using R = Counted;
using Base = kpolaris::RIAFAnalyticRadiationModel<R>;

// Kerr-Schild metric whose transport_rhs is counted as a call (its arithmetic
// is charged at gpu_rhs_ops()); everything else is the reference's.
struct CountingMetric : kpolaris::KerrSchildInMetric<R> {
    CountingMetric(R m, R a) : kpolaris::KerrSchildInMetric<R>(m, a) {}
};
static thread_local long long t_rhs = 0;

// Engine phases (kpolaris_b200/csrc/kp_common.cuh): 0 far (Boyer-Lindquist
// radius beyond fp32_radius), 1 near-A (pass A inside), 2 near-B (pass B
// inside).  Every RHS call is binned by the radius of its evaluation point;
// the other integration and transfer ops go to the phase of the latest RHS
// call.  Pass B is recognised from the pixel's first plasma sample, so the
// 11 RHS calls of a ray's first pass-B step count as near-A.
static double g_spin = 0.9375;
static double g_fp32_radius = 119.0;
static thread_local int t_in_b = 0;
static thread_local OpTally t_geom_phase[3];
static thread_local long long t_rhs_phase[3] = {0, 0, 0};

static double bl_radius(const kpolaris::TransportState<R>& s) {
    const double x = s.x[1].v, y = s.x[2].v, z = s.x[3].v, a2 = g_spin * g_spin;
    const double R2 = x * x + y * y + z * z;
    const double d = R2 - a2;
    return std::sqrt(0.5 * (d + std::sqrt(d * d + 4.0 * a2 * z * z)));
}

// Found by argument-dependent lookup from the reference's RK templates; as a
// non-template exact match it is preferred over the generic transport_rhs.
kpolaris::TransportState<R> transport_rhs(const CountingMetric& m, const kpolaris::TransportState<R>& s) {
    ++t_rhs;
    const int phase = bl_radius(s) > g_fp32_radius ? 0 : (t_in_b ? 2 : 1);
    ++t_rhs_phase[phase];
    g_tally = nullptr;
    auto d = kpolaris::transport_rhs(static_cast<const kpolaris::KerrSchildInMetric<R>&>(m), s);
    g_tally = &t_geom_phase[phase];
    return d;
}

// Per-thread buckets.
static thread_local OpTally t_geom, t_plasma, t_thermal;
static thread_local long long t_samples = 0, t_coeff = 0;
static thread_local const void* t_last_state = nullptr;
static thread_local double t_last_x[16];
static thread_local double t_last_k0 = 0;

// The RIAF model with the frequency-independent part counted once per
// distinct sample state.  Arithmetic follows riaf.hpp:410-549 through the
// model's own public helpers, so values are the reference's.
struct CountingRIAF : Base {
    template<class Metric>
    kpolaris::TransferCoeffs<R> coefficients(const Metric& metric, const kpolaris::TransportState<R>& state,
                                             R) const {
        t_in_b = 1;
        double cur[16];
        for (int mu = 0; mu < 4; ++mu) {
            cur[mu] = state.x[mu].v;
            cur[4 + mu] = state.k[mu].v;
            cur[8 + mu] = state.e1[mu].v;
            cur[12 + mu] = state.e2[mu].v;
        }
        const bool same = t_samples > 0 && std::memcmp(cur, t_last_x, sizeof(cur)) == 0;
        OpTally* saved = g_tally;
        OpTally scratch;
        g_tally = same ? &scratch : &t_plasma;
        ++t_coeff;
        if (!same) {
            ++t_samples;
            std::memcpy(t_last_x, cur, sizeof(cur));
        }
        kpolaris::TransferCoeffs<R> coeffs;
        R r_coord = R(0), th_coord = R(0), cosphi = R(1), sinphi = R(0);
        this->bl_coordinates_for_metric(metric, state.x, r_coord, th_coord, cosphi, sinphi);
        const R r_bl = kpolaris::max_val(r_coord, this->min_radius);
        const R rh = metric.horizon_radius();
        if (r_bl <= rh + this->horizon_buffer || r_bl < this->r_min || r_bl > this->r_max) {
            g_tally = saved;
            return coeffs;
        }
        const R ne_norm = this->density_profile_bl(r_bl, th_coord);
        if (!(ne_norm > R(0))) {
            g_tally = saved;
            return coeffs;
        }
        const R ne_cgs = ne_norm * this->ne_unit;
        const R thetae = this->thetae_profile(r_bl);
        const R b_cgs = this->magnetic_field_cgs(ne_cgs, r_bl);
        R gcov[4][4];
        metric.gcov_matrix(state.x, gcov);
        const auto ucon = this->fluid_four_velocity_from_bl_coords(metric, state.x, r_bl, th_coord, cosphi,
                                                                   sinphi, gcov);
        const auto ucov = this->lower_vector_with_gcov(gcov, ucon);
        R uk = R(0);
        for (int mu = 0; mu < 4; ++mu) uk += ucov[mu] * state.k[mu];
        const R nu_fluid = kpolaris::max_val(kpolaris::abs_val(-uk), this->min_frequency_scale);
        const auto bcon = this->magnetic_unit_four_vector_with_gcov(metric, state.x, ucon, gcov);
        const auto bcov = this->lower_vector_with_gcov(gcov, bcon);
        R kdotb = R(0);
        for (int mu = 0; mu < 4; ++mu) kdotb += state.k[mu] * bcov[mu];
        const R cos_theta = kpolaris::clamp(kdotb / kpolaris::max_val(nu_fluid, R(1e-30)), R(-1), R(1));
        const R sin_theta = kpolaris::max_val(
            Kokkos::sqrt(kpolaris::max_val(R(0), R(1) - cos_theta * cos_theta)), this->min_sin_theta);
        const R theta = Kokkos::acos(kpolaris::clamp(cos_theta, R(-1), R(1)));
        const R b1 = this->screen_inner_product_with_gcov(gcov, ucon, state.k, state.e1, bcon);
        const R b2 = this->screen_inner_product_with_gcov(gcov, ucon, state.k, state.e2, bcon);
        const R bproj2 = b1 * b1 + b2 * b2;
        R cos2chi = R(0), sin2chi = R(0);
        if (bproj2 > R(1e-30)) {
            cos2chi = (b2 * b2 - b1 * b1) / bproj2;
            sin2chi = -R(2) * b1 * b2 / bproj2;
        }
        // per-frequency part
        g_tally = &t_thermal;
        const R nu = kpolaris::max_val(this->freq_cgs * nu_fluid, R(1));
        kpolaris::ThermalSynchrotronParams<R> tp;
        tp.fit = this->emission_type;
        tp.max_pol_frac = this->max_pol_frac;
        tp.min_sin_theta = this->min_sin_theta;
        kpolaris::LocalThermalSynchrotronState<R> ts;
        ts.nu = nu;
        ts.ne = ne_cgs;
        ts.thetae = thetae;
        ts.b_cgs = b_cgs;
        ts.theta = theta;
        ts.sin_theta = sin_theta;
        ts.cos_theta = cos_theta;
        const auto m = kpolaris::thermal_synchrotron_magnetic_basis_coefficients(ts, tp);
        coeffs.jI = m.jI;
        coeffs.jV = m.jV;
        coeffs.aI = m.aI;
        coeffs.aV = m.aV;
        coeffs.rV = m.rV;
        coeffs.jQ = m.jQ * cos2chi;
        coeffs.jU = m.jQ * sin2chi;
        coeffs.aQ = m.aQ * cos2chi;
        coeffs.aU = m.aQ * sin2chi;
        coeffs.rQ = m.rQ * cos2chi;
        coeffs.rU = m.rQ * sin2chi;
        g_tally = saved;
        return coeffs;
    }
};

static void set_common(kpolaris::PassAParams<R>& p, int n, double step, int adaptive, int max_steps,
                       double tol, double min_step, double max_step, double mrs, double d0, double d1,
                       double d2) {
    const double spin = 0.9375;
    p.camera.nx = n;
    p.camera.ny = n;
    p.camera.radius = R(1000.0);
    p.camera.inclination = R(17.0 * 3.141592653589793238462643383279502884 / 180.0);
    p.camera.fov = R(2.0 * 80.0 / 1000.0);
    p.camera.fov_y = p.camera.fov;
    p.camera.xspan = R(-1);
    p.camera.yspan = R(-1);
    p.mass = R(1);
    p.spin = R(spin);
    p.inner_radius = R((1.0 + std::sqrt(std::max(0.0, 1.0 - spin * spin))) * 1.05);
    p.outer_radius = R(100.0 * 1.15);
    p.step = R(step);
    p.adaptive = adaptive;
    p.max_steps = max_steps;
    p.adaptive_tolerance = R(tol);
    p.min_step = R(min_step);
    p.max_step = R(max_step);
    p.max_radiation_step = R(mrs);
    p.max_radiation_depth = R(d0);
    p.max_absorption_depth = R(d1);
    p.max_faraday_depth = R(d2);
}

int main(int argc, char** argv) {
    const int cfg = argc > 1 ? std::atoi(argv[1]) : 2;
    const int n = argc > 2 ? std::atoi(argv[2]) : 64;
    kpolaris::PassAParams<R> pa;
    std::vector<double> freqs;
    if (cfg == 1) {
        set_common(pa, n, 1.0, 0, 2000, 1e-8, 1e-5, 1.0, 1.0, -1, -1, -1);
        freqs = {230.0e9};
        g_fp32_radius = 115.0 + 2.0 * 1.0;
    } else {
        set_common(pa, n, 0.025, 1, 400000, 1e-8, 1e-10, 2.0, 2.0, 1, 1, 4);
        freqs = {86.0e9, 230.0e9, 345.0e9, 690.0e9};
        g_fp32_radius = 115.0 + 2.0 * 2.0;
    }
    CountingRIAF model;
    model.mbh_solar = R(6.5e9);
    model.ne_unit = R(4.0e6);
    model.te_unit = R(1.5e11);
    model.disk_h = R(0.3);
    model.emission_type = 1;
    const CountingMetric metric(R(1), pa.spin);
    const int npix = n * n;
    OpTally tot_geom, tot_plasma, tot_thermal, tot_phase[3];
    long long samples = 0, coeff = 0, steps_a = 0, steps_b = 0, rhs = 0;
    long long rhs_phase[3] = {0, 0, 0};
#pragma omp parallel reduction(+ : samples, coeff, steps_a, steps_b, rhs)
    {
        for (auto& t : t_geom_phase) t = OpTally();
        for (auto& c : t_rhs_phase) c = 0;
        t_plasma = OpTally();
        t_thermal = OpTally();
        t_samples = 0;
        t_coeff = 0;
        t_rhs = 0;
#pragma omp for schedule(dynamic)
        for (int pixel = 0; pixel < npix; ++pixel) {
            t_in_b = 0;
            g_tally = &t_geom_phase[0];
            R f[KPOLARIS_MAX_FREQUENCIES];
            kpolaris::Stokes<R> st[KPOLARIS_MAX_FREQUENCIES];
            for (size_t i = 0; i < freqs.size(); ++i) f[i] = R(freqs[i]);
            t_samples = std::max<long long>(t_samples, 0);
            auto r = kpolaris::trace_pass_b_segment_model_multifrequency_pixel_metric(
                pixel, pa, model, 1, f, int(freqs.size()), st, metric);
            g_tally = nullptr;
            steps_a += r.pass_a.steps;
            steps_b += r.steps;
        }
        samples += t_samples;
        rhs += t_rhs;
        coeff += t_coeff;
#pragma omp critical
        {
            for (int ph = 0; ph < 3; ++ph) {
                const OpTally& g = t_geom_phase[ph];
                tot_geom.add += g.add; tot_geom.mul += g.mul; tot_geom.div += g.div;
                tot_geom.sqrt += g.sqrt; tot_geom.trans += g.trans;
                tot_phase[ph].add += g.add; tot_phase[ph].mul += g.mul; tot_phase[ph].div += g.div;
                tot_phase[ph].sqrt += g.sqrt; tot_phase[ph].trans += g.trans;
                rhs_phase[ph] += t_rhs_phase[ph];
            }
            tot_plasma.add += t_plasma.add; tot_plasma.mul += t_plasma.mul; tot_plasma.div += t_plasma.div;
            tot_plasma.sqrt += t_plasma.sqrt; tot_plasma.trans += t_plasma.trans;
            tot_thermal.add += t_thermal.add; tot_thermal.mul += t_thermal.mul;
            tot_thermal.div += t_thermal.div; tot_thermal.sqrt += t_thermal.sqrt;
            tot_thermal.trans += t_thermal.trans;
        }
    }
    auto basic = [](const OpTally& t) { return t.add + t.mul + t.div + t.sqrt; };
    std::printf("{\"config\": %d, \"n\": %d, \"pixels\": %d, \"nfreq\": %zu,\n", cfg, n, npix, freqs.size());
    std::printf(" \"pass_a_steps\": %lld, \"pass_b_steps\": %lld, \"coefficient_calls\": %lld, "
                "\"plasma_samples\": %lld,\n", steps_a, steps_b, coeff, samples);
    auto dump = [&](const char* name, const OpTally& t, const char* sep) {
        std::printf(" \"%s\": {\"add\": %llu, \"mul\": %llu, \"div\": %llu, \"sqrt\": %llu, "
                    "\"transcendental\": %llu, \"basic\": %llu}%s\n",
                    name, t.add, t.mul, t.div, t.sqrt, t.trans, basic(t), sep);
    };
    const OpTally per_rhs = gpu_rhs_ops();
    OpTally rhs_tot;
    rhs_tot.add = per_rhs.add * rhs;
    rhs_tot.mul = per_rhs.mul * rhs;
    rhs_tot.div = per_rhs.div * rhs;
    rhs_tot.sqrt = per_rhs.sqrt * rhs;
    std::printf(" \"rhs_calls\": %lld,\n", rhs);
    dump("rhs_each", per_rhs, ",");
    dump("rhs_total", rhs_tot, ",");
    dump("integration_and_transfer", tot_geom, ",");
    dump("plasma", tot_plasma, ",");
    dump("thermal", tot_thermal, ",");
    std::printf(" \"fp32_radius\": %.17g,\n", g_fp32_radius);
    const char* names[3] = {"far", "near_a", "near_b"};
    for (int ph = 0; ph < 3; ++ph) {
        std::printf(" \"phase_%s\": {\"rhs_calls\": %lld, \"rhs_ops\": %llu, \"other_ops\": %llu},\n", names[ph],
                    rhs_phase[ph], basic(per_rhs) * (unsigned long long)rhs_phase[ph], basic(tot_phase[ph]));
    }
    std::printf(" \"fp64_basic_ops\": %llu}\n",
                basic(rhs_tot) + basic(tot_geom) + basic(tot_plasma) + basic(tot_thermal));
    return 0;
}
