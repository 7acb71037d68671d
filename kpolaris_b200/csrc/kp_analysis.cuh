// kp_analysis.cuh -- analysis mode of the RIAF image: the FP64 per-pixel
// pass B with the reference's line-of-sight diagnostics accumulated along
// the ray (src/image/analysis_driver.hpp:16-640):
//   * per radiating sample: path length, emission weight and the
//     emission-weighted radius, optical depth to the camera and plasma
//     state, the brightest sample's radius, region and plasma state,
//     absorption / Faraday depths in total and per logarithmic radial bin
//     (accumulate_physical_analysis_sample, :310-369);
//   * per step: the photon-ring winding estimate from the BL azimuth
//     (accumulate_analysis_phi, :289-307);
//   * one Stokes vector per radial bin, emitting only in its own bin and
//     propagated everywhere else (:576-582), transformed to the observer
//     basis at the end; from them the observer-weighted radii, formation
//     radius quantiles, coherences, contribution closure and foreground
//     depths (finalize_observer_weighted_analysis, :178-262).
// The pass-B loop is the analysis driver's
// (trace_pass_b_segment_model_endpoint_analysis_pixel_metric, :409-621),
// single frequency; it differs from the imaging loop in two places: a
// rejected attempt at the minimum step ends the ray as max_steps, and a
// sample radiates when r >= inner_radius.  With a kp_response_config, the
// source-partition response channels (src/diagnostics/response.hpp) are
// accumulated per radiating sample in global memory.
#pragma once

#include "kp_launch.h"
#include "kp_trace_fp64.cuh"

namespace kp {

// Per-ray accumulators (PassBAnalysisDiagnostics, :25-79).
struct AnalysisAcc {
    double radiating_path_length, emission_weight, emission_weighted_radius, emission_weighted_tau;
    double absorption_depth, absorption_operator_depth, faraday_rotation_depth, faraday_conversion_depth,
        faraday_operator_depth;
    double dominant_radius, dominant_weight, dominant_ne, dominant_thetae, dominant_b, dominant_beta,
        dominant_sigma;
    double w_ne, w_thetae, w_b, w_beta, w_sigma;
    double winding, previous_phi;
    int has_previous_phi, substeps, dominant_region;
    double radial_abs[kMaxRadialBins], radial_rot[kMaxRadialBins], radial_conv[kMaxRadialBins],
        radial_op[kMaxRadialBins];
    Stokes4<double> radial[kMaxRadialBins];
};

__device__ __forceinline__ void analysis_zero(AnalysisAcc& a) {
    a.radiating_path_length = a.emission_weight = a.emission_weighted_radius = a.emission_weighted_tau = 0.0;
    a.absorption_depth = a.absorption_operator_depth = a.faraday_rotation_depth = 0.0;
    a.faraday_conversion_depth = a.faraday_operator_depth = 0.0;
    a.dominant_radius = a.dominant_weight = a.dominant_ne = a.dominant_thetae = a.dominant_b = 0.0;
    a.dominant_beta = a.dominant_sigma = 0.0;
    a.w_ne = a.w_thetae = a.w_b = a.w_beta = a.w_sigma = 0.0;
    a.winding = a.previous_phi = 0.0;
    a.has_previous_phi = a.substeps = a.dominant_region = 0;
    for (int i = 0; i < kMaxRadialBins; ++i) {
        a.radial_abs[i] = a.radial_rot[i] = a.radial_conv[i] = a.radial_op[i] = 0.0;
        a.radial[i] = Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    }
}

// analysis_radial_bin / analysis_radial_bin_center (:88-116): logarithmic
// bins between radial_min and radial_max, the ends clamped.
__device__ __forceinline__ int analysis_radial_bin(const AnalysisConsts& k, double r) {
    if (k.radial_bins <= 1 || !(k.radial_max > k.radial_min) || !(k.radial_min > 0.0) || !(r > k.radial_min))
        return 0;
    if (r >= k.radial_max) return k.radial_bins - 1;
    const double fraction = log(r / k.radial_min) / log(k.radial_max / k.radial_min);
    int bin = int(fraction * double(k.radial_bins));
    if (bin < 0) bin = 0;
    if (bin >= k.radial_bins) bin = k.radial_bins - 1;
    return bin;
}

__device__ __forceinline__ double analysis_bin_center(const AnalysisConsts& k, int bin) {
    if (k.radial_bins <= 0 || !(k.radial_max > k.radial_min) || !(k.radial_min > 0.0)) return 0.0;
    const double lo = log(k.radial_min), hi = log(k.radial_max);
    return exp(lo + (double(bin) + 0.5) / double(k.radial_bins) * (hi - lo));
}

// dominant_emission_region_code (:264-276): 1 inside 5 M, 2 inside 20 M, 3 beyond.
__device__ __forceinline__ int emission_region_code(double r) {
    if (!(r > 0.0)) return 0;
    if (r < 5.0) return 1;
    if (r < 20.0) return 2;
    return 3;
}

// accumulate_analysis_phi (:289-307): winding in turns of the BL azimuth.
__device__ __forceinline__ void analysis_phi(const ImageConsts& c, const Ray& sample, AnalysisAcc& a) {
    const BlCoords q = riaf_bl_coords(c.spin, sample.x);
    const double two_pi = 6.283185307179586476925286766559005768;
    double phi = atan2(q.sphi, q.cphi);
    if (phi < 0.0) phi += two_pi;
    if (a.has_previous_phi) {
        double dphi = phi - a.previous_phi;
        if (dphi > 3.141592653589793238462643383279502884) dphi -= two_pi;
        else if (dphi < -3.141592653589793238462643383279502884) dphi += two_pi;
        a.winding += abs_val(dphi) / two_pi;
    }
    a.previous_phi = phi;
    a.has_previous_phi = 1;
}

// accumulate_physical_analysis_sample (:310-369) for the RIAF plasma
// (analysis_plasma_diagnostics, src/diagnostics/plasma.hpp:22-44: beta and
// sigma are not defined for it and stay 0).
__device__ __forceinline__ void analysis_sample(const ImageConsts& c, const Ray& sample, const Coeffs<double>& co,
                                                double dlambda, double r, int bin, AnalysisAcc& a) {
    const double dl = abs_val(dlambda);
    const double absorption_delta = max_val(co.aI, 0.0) * dl;
    const double absorption_operator_delta =
        (abs_val(co.aI) + sqrt(co.aQ * co.aQ + co.aU * co.aU + co.aV * co.aV)) * dl;
    const double faraday_rotation_delta = co.rV * dl;
    const double faraday_conversion_delta = sqrt(co.rQ * co.rQ + co.rU * co.rU) * dl;
    const double faraday_operator_delta = sqrt(co.rQ * co.rQ + co.rU * co.rU + co.rV * co.rV) * dl;
    const double tau_from_source_mid = a.absorption_depth + 0.5 * absorption_delta;
    const double weight = max_val(co.jI, 0.0) * dl;
    a.radiating_path_length += dl;
    if (weight > 0.0) {
        a.emission_weight += weight;
        a.emission_weighted_radius += weight * r;
        a.emission_weighted_tau += weight * tau_from_source_mid;
        const BlCoords q = riaf_bl_coords(c.spin, sample.x);
        double r_bl, ne = 0.0, thetae = 0.0, b = 0.0;
        const int valid = riaf_plasma(c, q, r_bl, ne, thetae, b) && ne > 0.0 && thetae > 0.0 && b > 0.0;
        if (weight > a.dominant_weight) {
            a.dominant_weight = weight;
            a.dominant_radius = r;
            a.dominant_region = emission_region_code(r);
            if (valid) {
                a.dominant_ne = ne;
                a.dominant_thetae = thetae;
                a.dominant_b = b;
                a.dominant_beta = 0.0;
                a.dominant_sigma = 0.0;
            }
        }
        if (valid) {
            a.w_ne += weight * ne;
            a.w_thetae += weight * thetae;
            a.w_b += weight * b;
            a.w_beta += weight * 0.0;
            a.w_sigma += weight * 0.0;
        }
    }
    a.absorption_depth += absorption_delta;
    a.absorption_operator_depth += absorption_operator_delta;
    a.faraday_rotation_depth += faraday_rotation_delta;
    a.faraday_conversion_depth += faraday_conversion_delta;
    a.faraday_operator_depth += faraday_operator_delta;
    a.radial_abs[bin] += absorption_delta;
    a.radial_rot[bin] += faraday_rotation_delta;
    a.radial_conv[bin] += faraday_conversion_delta;
    a.radial_op[bin] += faraday_operator_delta;
}

// finalize_analysis (:371-388): the weighted sums become means.
__device__ __forceinline__ void analysis_finalize(AnalysisAcc& a) {
    if (a.emission_weight > 0.0) {
        const double inv = 1.0 / a.emission_weight;
        a.emission_weighted_radius *= inv;
        const double mean_tau_from_source = a.emission_weighted_tau * inv;
        a.emission_weighted_tau = max_val(0.0, a.absorption_depth - mean_tau_from_source);
        a.w_ne *= inv;
        a.w_thetae *= inv;
        a.w_b *= inv;
        a.w_beta *= inv;
        a.w_sigma *= inv;
    } else {
        a.emission_weighted_radius = 0.0;
        a.emission_weighted_tau = 0.0;
        a.dominant_radius = 0.0;
        a.dominant_region = 0;
    }
}

// The imaging loop's observer transform (transform_to_observer_basis,
// src/frame/stokes_rotation.hpp:39-57) with the overlaps of finish_ray.
__device__ __forceinline__ Stokes4<double> observer_stokes(const Stokes4<double>& s, const PixelOut& o) {
    const double r11 = o.r11, r12 = o.r12, r21 = o.r21, r22 = o.r22;
    Stokes4<double> out;
    out.I = s.I;
    out.Q = 0.5 * s.Q * (r11 * r11 - r12 * r12 - r21 * r21 + r22 * r22) + s.U * (r11 * r12 - r21 * r22);
    out.U = s.Q * (r11 * r21 - r12 * r22) + s.U * (r11 * r22 + r12 * r21);
    out.V = (r11 * r22 - r12 * r21) * s.V;
    return out;
}

// radial_contribution_weight (:127-138): I+, |linear|, |V|.
__device__ __forceinline__ double contribution_weight(const Stokes4<double>& s, int component) {
    if (component == 0) return max_val(s.I, 0.0);
    if (component == 1) return sqrt(s.Q * s.Q + s.U * s.U);
    return abs_val(s.V);
}

// radial_formation_quantile (:141-162) over observer-basis bin Stokes.
__device__ __forceinline__ double formation_quantile(const AnalysisAcc& a, const AnalysisConsts& k, int component,
                                                     double quantile) {
    double total = 0.0;
    for (int b = 0; b < k.radial_bins; ++b) total += contribution_weight(a.radial[b], component);
    if (!(total > 0.0)) return 0.0;
    const double target = min_val(1.0, max_val(0.0, quantile)) * total;
    double cumulative = 0.0;
    for (int b = 0; b < k.radial_bins; ++b) {
        cumulative += contribution_weight(a.radial[b], component);
        if (cumulative >= target) return analysis_bin_center(k, b);
    }
    return analysis_bin_center(k, k.radial_bins - 1);
}

// radial_weighted_radius (:164-176).
__device__ __forceinline__ double weighted_radius(const AnalysisAcc& a, const AnalysisConsts& k, int component) {
    double weighted = 0.0, total = 0.0;
    for (int b = 0; b < k.radial_bins; ++b) {
        const double w = contribution_weight(a.radial[b], component);
        weighted += w * analysis_bin_center(k, b);
        total += w;
    }
    return total > 0.0 ? weighted / total : 0.0;
}

struct ObserverAnalysis {
    double radius_i, radius_linear, radius_circular;
    double q[3][3];  // formation radius (low, median, high) of I, linear, circular
    double linear_coherence, circular_coherence, closure_max_abs, closure_relative_l1;
    double fg_abs, fg_rot, fg_conv, fg_op, fg_op_fraction;
};

// finalize_observer_weighted_analysis (:178-262); a.radial already holds
// the observer-basis bin Stokes, `observed` the ray's own.
__device__ __forceinline__ ObserverAnalysis observer_analysis(const AnalysisAcc& a, const AnalysisConsts& k,
                                                             const Stokes4<double>& observed) {
    ObserverAnalysis o = {};
    Stokes4<double> sum{0.0, 0.0, 0.0, 0.0};
    double sum_linear = 0.0, sum_abs_v = 0.0, contribution_l1 = 0.0;
    for (int b = 0; b < k.radial_bins; ++b) {
        const Stokes4<double>& s = a.radial[b];
        sum.I += s.I;
        sum.Q += s.Q;
        sum.U += s.U;
        sum.V += s.V;
        sum_linear += sqrt(s.Q * s.Q + s.U * s.U);
        sum_abs_v += abs_val(s.V);
        contribution_l1 += abs_val(s.I) + abs_val(s.Q) + abs_val(s.U) + abs_val(s.V);
    }
    const double di = sum.I - observed.I, dq = sum.Q - observed.Q, du = sum.U - observed.U,
                 dv = sum.V - observed.V;
    o.closure_max_abs = max_val(max_val(abs_val(di), abs_val(dq)), max_val(abs_val(du), abs_val(dv)));
    const double residual_l1 = abs_val(di) + abs_val(dq) + abs_val(du) + abs_val(dv);
    o.closure_relative_l1 = residual_l1 / max_val(contribution_l1, 1e-300);  // tiny_positive<double>
    o.linear_coherence = sum_linear > 0.0 ? sqrt(sum.Q * sum.Q + sum.U * sum.U) / sum_linear : 0.0;
    o.circular_coherence = sum_abs_v > 0.0 ? abs_val(sum.V) / sum_abs_v : 0.0;
    o.radius_i = weighted_radius(a, k, 0);
    o.radius_linear = weighted_radius(a, k, 1);
    o.radius_circular = weighted_radius(a, k, 2);
    const double tail = 0.5 * (1.0 - k.formation_fraction);
    for (int comp = 0; comp < 3; ++comp) {
        o.q[comp][0] = formation_quantile(a, k, comp, tail);
        o.q[comp][1] = formation_quantile(a, k, comp, 0.5);
        o.q[comp][2] = formation_quantile(a, k, comp, 1.0 - tail);
    }
    const double formation_outer = o.q[0][2];
    if (formation_outer > 0.0) {
        for (int b = 0; b < k.radial_bins; ++b) {
            if (analysis_bin_center(k, b) > formation_outer) {
                o.fg_abs += a.radial_abs[b];
                o.fg_rot += a.radial_rot[b];
                o.fg_conv += a.radial_conv[b];
                o.fg_op += a.radial_op[b];
            }
        }
    }
    if (a.faraday_operator_depth > 0.0) o.fg_op_fraction = o.fg_op / a.faraday_operator_depth;
    return o;
}

// ------------------------------------------------ source-partition responses
// Channel c of pixel p: four Stokes components at (4 c + s) npix + p
// (response_read / response_write, response.hpp:12-24).
__device__ __forceinline__ Stokes4<double> resp_read(const double* d, int pixel, int npix, int ch) {
    const size_t base = size_t(4) * size_t(ch) * size_t(npix) + size_t(pixel);
    return Stokes4<double>{d[base], d[base + npix], d[base + 2 * size_t(npix)], d[base + 3 * size_t(npix)]};
}

__device__ __forceinline__ void resp_write(double* d, int pixel, int npix, int ch, const Stokes4<double>& s) {
    const size_t base = size_t(4) * size_t(ch) * size_t(npix) + size_t(pixel);
    d[base] = s.I;
    d[base + npix] = s.Q;
    d[base + 2 * size_t(npix)] = s.U;
    d[base + 3 * size_t(npix)] = s.V;
}

__device__ __forceinline__ Stokes4<double> resp_add(const Stokes4<double>& a, const Stokes4<double>& b) {
    return Stokes4<double>{a.I + b.I, a.Q + b.Q, a.U + b.U, a.V + b.V};
}

// The transfer step as a linear map: its columns are the unit Stokes vectors
// stepped without emission (ResponseStepMatrix, response.hpp:37-55).
struct RespStepMatrix {
    Stokes4<double> col[4];
};

__device__ __forceinline__ RespStepMatrix resp_step_matrix(Coeffs<double> co, double dl) {
    co.jI = co.jQ = co.jU = co.jV = 0.0;
    RespStepMatrix m;
    for (int k = 0; k < 4; ++k) {
        m.col[k] = Stokes4<double>{k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0, k == 3 ? 1.0 : 0.0};
        stokes_step(m.col[k], co, dl);
    }
    return m;
}

__device__ __forceinline__ Stokes4<double> resp_apply(const RespStepMatrix& m, const Stokes4<double>& s) {
    const Stokes4<double>* c = m.col;
    return Stokes4<double>{c[0].I * s.I + c[1].I * s.Q + c[2].I * s.U + c[3].I * s.V,
                           c[0].Q * s.I + c[1].Q * s.Q + c[2].Q * s.U + c[3].Q * s.V,
                           c[0].U * s.I + c[1].U * s.Q + c[2].U * s.U + c[3].U * s.V,
                           c[0].V * s.I + c[1].V * s.Q + c[2].V * s.U + c[3].V * s.V};
}

// response_replace_block (response.hpp:57-70): mechanism 0 emission, 1
// absorption, 2 Faraday rotation, 3 Faraday conversion.
__device__ __forceinline__ Coeffs<double> resp_replace(Coeffs<double> b, const Coeffs<double>& v, int m) {
    if (m == 0) {
        b.jI = v.jI; b.jQ = v.jQ; b.jU = v.jU; b.jV = v.jV;
    } else if (m == 1) {
        b.aI = v.aI; b.aQ = v.aQ; b.aU = v.aU; b.aV = v.aV;
    } else if (m == 2) {
        b.rV = v.rV;
    } else {
        b.rQ = v.rQ; b.rU = v.rU;
    }
    return b;
}

// Source bin of a sample (response_partition_bin, response.hpp:79-111) for
// the RIAF plasma, whose magnetisation is undefined (src/diagnostics/
// plasma.hpp:22-44).
__device__ __forceinline__ int resp_partition_bin(const kp_response_config& R, const ImageConsts& c,
                                                  const BlCoords& q) {
    const double r = q.rc, theta = q.th;
    if (R.partition == KP_PARTITION_RADIAL) {
        int bin = 0;
        while (bin < R.bins - 1 && r >= R.edges[bin + 1]) ++bin;
        return bin;
    }
    if (R.partition == KP_PARTITION_REGION || R.partition == KP_PARTITION_NEAR_FAR) {
        const double sight_dot =
            sin(theta) * sin(R.observer_theta) * (q.cphi * cos(R.observer_phi) + q.sphi * sin(R.observer_phi)) +
            cos(theta) * cos(R.observer_theta);
        const int side = sight_dot >= 0.0 ? 0 : 1;
        if (R.partition == KP_PARTITION_NEAR_FAR) return side;
        const double polar = min_val(theta, 3.14159265358979323846 - theta);
        const int region = polar < R.funnel_angle ? 0 : (polar < R.disk_angle ? 1 : 2);
        return 2 * region + side;
    }
    if (R.partition == KP_PARTITION_PLASMA_REGION) return 3;
    if (R.partition == KP_PARTITION_SIGMA || R.partition == KP_PARTITION_BETA) return R.bins - 1;
    double r_bl, ne = 0.0, thetae = 0.0, b = 0.0;
    const int valid = riaf_plasma(c, q, r_bl, ne, thetae, b) && ne > 0.0 && thetae > 0.0 && b > 0.0;
    if (!valid) return R.bins - 1;
    double value = thetae;
    if (R.partition == KP_PARTITION_NE_CGS) value = ne;
    if (R.partition == KP_PARTITION_B_CGS) value = b;
    int bin = 0;
    while (bin < R.edge_count && value >= R.edges[bin]) ++bin;
    return bin;
}

// The coefficients at the sample with the plasma scaled by e^q
// (PlasmaPerturbation::apply, src/radiation/plasma_perturbation.hpp:14-31,
// inside RIAFAnalyticRadiationModel::coefficients, riaf.hpp:428-432), or
// every coefficient scaled by e^q (response_scale_coefficients,
// response.hpp:72-78).
__device__ __forceinline__ Coeffs<double> resp_variant(const ImageConsts& c, const kp_response_config& R,
                                                       const RiafSample& p, const Coeffs<double>& base, double q) {
    if (R.parameter == KP_RESPONSE_COEFFICIENTS) {
        const double f = exp(q);
        Coeffs<double> o = base;
        o.jI *= f; o.jQ *= f; o.jU *= f; o.jV *= f;
        o.aI *= f; o.aQ *= f; o.aU *= f; o.aV *= f;
        o.rQ *= f; o.rU *= f; o.rV *= f;
        return o;
    }
    RiafSample v = p;
    if (q != 0.0) {
        const double f = exp(q);
        if (R.parameter == KP_RESPONSE_DENSITY_SCALE) {
            v.ne *= f;
            v.b *= exp(q * 0.5);
        } else if (R.parameter == KP_RESPONSE_TEMPERATURE_SCALE) {
            v.thetae *= f;
        } else if (R.parameter == KP_RESPONSE_MAGNETIC_SCALE) {
            v.b *= f;
        }
    }
    Coeffs<double> o = riaf_coefficients(c, v, c.freq[0]);
    if (!c.faraday_rotation) o.rV = 0.0;
    return o;
}

// accumulate_response_sample + response_transfer_step (response.hpp:117-
// 184): `incoming` is the pixel's Stokes vector before this step, `base`
// the step's coefficients, `p` the plasma sample they came from.
__device__ __noinline__ void response_sample(const ImageConsts& c, const kp_response_config& R, const Ray& sample,
                                             const RiafSample& p, const Stokes4<double>& incoming,
                                             const Coeffs<double>& base, double dl, double* data, int pixel,
                                             int npix) {
    const BlCoords q = riaf_bl_coords(c.spin, sample.x);
    const int bin = resp_partition_bin(R, c, q);
    const bool responses = R.parameter != KP_RESPONSE_NONE;
    Coeffs<double> variants[4];
    if (responses) {
        for (int v = 0; v < 4; ++v) {
            const double qv = R.step * (v % 2 == 0 ? 1.0 : -1.0) * (v < 2 ? 1.0 : 0.5);
            variants[v] = resp_variant(c, R, p, base, qv);
        }
    }
    const RespStepMatrix m = resp_step_matrix(base, dl);
    Stokes4<double> emitted{0.0, 0.0, 0.0, 0.0};
    stokes_step(emitted, base, dl);
    for (int k = 0; k < R.bins; ++k) {
        Stokes4<double> s = resp_apply(m, resp_read(data, pixel, npix, k));
        if (k == bin) s = resp_add(s, emitted);
        resp_write(data, pixel, npix, k, s);
    }
    if (!responses) return;
    const double denom = 2.0 * R.step;
    for (int mech = 0; mech < 4; ++mech) {
        Stokes4<double> plus = incoming, minus = incoming;
        stokes_step(plus, resp_replace(base, variants[0], mech), dl);
        stokes_step(minus, resp_replace(base, variants[1], mech), dl);
        const Stokes4<double> forcing{(plus.I - minus.I) / denom, (plus.Q - minus.Q) / denom,
                                      (plus.U - minus.U) / denom, (plus.V - minus.V) / denom};
        for (int k = 0; k < R.bins; ++k) {
            const int ch = R.bins + mech * R.bins + k;
            Stokes4<double> s = resp_apply(m, resp_read(data, pixel, npix, ch));
            if (k == bin) s = resp_add(s, forcing);
            resp_write(data, pixel, npix, ch, s);
        }
    }
    for (int v = 0; v < 4; ++v) {
        const int ch = 5 * R.bins + v;
        Stokes4<double> s = resp_read(data, pixel, npix, ch);
        stokes_step(s, variants[v], dl);
        resp_write(data, pixel, npix, ch, s);
    }
}

// Channels of a configuration (ResponseConfig::channels, response_config.hpp:29).
KP_HD int response_channel_count(const kp_response_config& R) {
    if (R.partition == KP_PARTITION_NONE) return 0;
    const bool responses = R.parameter != KP_RESPONSE_NONE;
    return R.bins * (responses ? 5 : 1) + (responses ? 4 : 0);
}

// The analysis driver's pass B, one frequency (:444-611).
__device__ __forceinline__ void trace_pass_b_analysis(const ImageConsts& c, const AnalysisConsts& k, Ray& state,
                                                      Stokes4<double>& stokes, int& steps, int& reason,
                                                      AnalysisAcc& a, const kp_response_config* resp = nullptr,
                                                      double* resp_data = nullptr, int pixel = 0, int npix = 0) {
    const double mass = c.mass, spin = c.spin;
    StepControl ctl;
    ctl.tolerance = c.tolerance;
    ctl.min_step = c.min_step_abs;
    ctl.max_step = c.max_step;
    stokes = Stokes4<double>{0.0, 0.0, 0.0, 0.0};
    int reached = 0;
    steps = 0;
    double h_current = c.step;
    double cap = c.max_radiation_step > 0.0 ? c.max_radiation_step : c.max_step;
    const double min_step = c.min_step_abs;
    const double dls = c.dlambda_scale[0];
#pragma unroll 1
    while (!reached && steps < c.max_steps) {
        double h = h_current;
        const Ray old = state;
        const double start_r = ks_radius(spin, old.x);
        if (start_r <= c.outer_radius && cap > 0.0) h = min_val(h, cap);
        Ray next, sample;
        if (c.adaptive) {
            AdaptiveStep st;
            adaptive_step(0, mass, spin, old, h, ctl, st);
            if (!st.accepted) {
                h_current = abs_val(st.next_h);
                if (h_current <= min_step * 1.0001) {
                    reason = kMaxSteps;
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
        const double s0 = start_r - c.cam_radius;
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
                    cc.min_step = min_val(min_step, abs_val(h));
                    cc.max_step = max_val(cc.min_step, abs_val(h));
                    AdaptiveStep cs;
                    adaptive_step(0, mass, spin, old, h, cc, cs);
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
        const double old_r = start_r;
        const double sample_r = ks_radius(spin, sample.x);
        const double next_r = ks_radius(spin, next.x);
        const int active = sample_r >= c.inner_radius && sample_r < c.outer_radius;
        Coeffs<double> co = {};
        RiafSample ps;
        ps.emitting = 0;
        if (active) {
            ps = riaf_sample(c, sample);
            co = riaf_coefficients(c, ps, c.freq[0]);
            if (!c.faraday_rotation) co.rV = 0.0;
        }
        const double local_max_rs =
            (c.max_radiation_step > 0.0 &&
             (old_r <= c.outer_radius || sample_r <= c.outer_radius || next_r <= c.outer_radius))
                ? c.max_radiation_step : 0.0;
        const int required = radiation_substep_count(co, h, dls, local_max_rs, c.max_radiation_depth,
                                                     c.max_absorption_depth, c.max_faraday_depth);
        if (required > 1 && h > min_step * 1.0001) {
            h_current = max_val(min_step, h / double(required));
            cap = h_current;
            continue;
        }
        if (local_max_rs > 0.0 || c.max_radiation_depth > 0.0 || c.max_absorption_depth > 0.0 ||
            c.max_faraday_depth > 0.0) {
            const int pred = radiation_substep_count(co, h_current, dls, local_max_rs, c.max_radiation_depth,
                                                     c.max_absorption_depth, c.max_faraday_depth);
            cap = pred > 1 ? max_val(min_step, h_current / double(pred)) : c.max_step;
        } else {
            cap = c.max_step;
        }
        if (h > 0.0) {
            analysis_phi(c, sample, a);
            if (active) {
                const double dlambda = abs_val(h) * dls;
                const double r = riaf_bl_coords(spin, sample.x).rc;
                const int bin = analysis_radial_bin(k, r);
                analysis_sample(c, sample, co, dlambda, r, bin, a);
                Coeffs<double> propagation = co;
                propagation.jI = propagation.jQ = propagation.jU = propagation.jV = 0.0;
                if (resp) response_sample(c, *resp, sample, ps, stokes, co, dlambda, resp_data, pixel, npix);
#pragma unroll 1
                for (int b = 0; b < k.radial_bins; ++b) stokes_step(a.radial[b], b == bin ? co : propagation, dlambda);
                a.substeps += 1;
            }
            stokes_step(stokes, co, abs_val(h) * dls);
        }
        state = next;
        steps += 1;
        if (crosses) reached = 1;
    }
    analysis_finalize(a);
    if (reached) {
        reason = kReachedCamera;
    } else if (reason != kAdaptiveUnderflow) {
        reason = kMaxSteps;
    }
}

}  // namespace kp
