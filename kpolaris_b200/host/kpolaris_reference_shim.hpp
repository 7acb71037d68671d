// kpolaris_reference_shim.hpp -- C++ host shim that gives the reference's
// image entry points their original signatures on top of the C ABI
// (include/kpolaris_b200.h), so the reference's callers
// (tools/kpolaris_model_image.cpp:3416 compute_frequency_image,
//  :3437 compute_multifrequency_images; examples/grrt_batch_benchmark.cpp;
//  tests/test_image_batch.cpp) relink unchanged.
//
// The shim is templated on the reference's own parameter and result types
// (PassAParams<double>, RIAFAnalyticRadiationModel<double>, ImageHostData),
// which it reads field by field; it therefore compiles inside the reference's
// build without this library depending on the reference's headers.  Include it
// after the reference's own headers (they bring in Kokkos, whose mirror views
// the GRMHD entry points use).  Errors
// are rethrown with the reference's exception types: KP_ERR_INVALID as
// std::invalid_argument, everything else as std::runtime_error.
#pragma once

#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "kpolaris_b200.h"

namespace kpolaris_b200 {

inline void throw_on_error(int status) {
    if (status == KP_OK) return;
    const std::string msg = kp_last_error();
    if (status == KP_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// PassAParams<Real> (src/geodesic/pass_a_core.hpp:10-36) -> kp_pass_a_params.
template<class PassA>
kp_pass_a_params to_c(const PassA& p) {
    kp_pass_a_params o;
    std::memset(&o, 0, sizeof(o));
    o.camera.nx = p.camera.nx;
    o.camera.ny = p.camera.ny;
    o.camera.radius = double(p.camera.radius);
    o.camera.inclination = double(p.camera.inclination);
    o.camera.fov = double(p.camera.fov);
    o.camera.fov_y = double(p.camera.fov_y);
    o.camera.xspan = double(p.camera.xspan);
    o.camera.yspan = double(p.camera.yspan);
    o.camera.x_offset = double(p.camera.x_offset);
    o.camera.y_offset = double(p.camera.y_offset);
    o.camera.model = static_cast<int>(p.camera.model);
    o.emission_selection.equatorial_h_over_r = double(p.emission_selection.equatorial_h_over_r);
    o.emission_selection.equatorial_samples = p.emission_selection.equatorial_samples;
    o.emission_selection.faraday_rotation = p.emission_selection.faraday_rotation;
    o.mass = double(p.mass);
    o.spin = double(p.spin);
    o.inner_radius = double(p.inner_radius);
    o.outer_radius = double(p.outer_radius);
    o.step = double(p.step);
    o.max_steps = p.max_steps;
    o.adaptive = p.adaptive;
    o.direct_only = p.direct_only;
    o.adaptive_tolerance = double(p.adaptive_tolerance);
    o.min_step = double(p.min_step);
    o.max_step = double(p.max_step);
    o.max_radiation_step = double(p.max_radiation_step);
    o.max_radiation_depth = double(p.max_radiation_depth);
    o.max_absorption_depth = double(p.max_absorption_depth);
    o.max_faraday_depth = double(p.max_faraday_depth);
    o.fmks_startx1 = double(p.fmks_startx1);
    o.fmks_hslope = double(p.fmks_hslope);
    o.fmks_mks_smooth = double(p.fmks_mks_smooth);
    o.fmks_poly_alpha = double(p.fmks_poly_alpha);
    o.fmks_poly_xt = double(p.fmks_poly_xt);
    o.fmks_poly_norm = double(p.fmks_poly_norm);
    o.coordinate_system = static_cast<int>(p.coordinate_system);
    return o;
}

// RIAFAnalyticRadiationModel<Real> (src/model/riaf.hpp:19-52) -> kp_riaf_model.
template<class Model>
kp_riaf_model to_c_riaf(const Model& m) {
    kp_riaf_model o;
    std::memset(&o, 0, sizeof(o));
    o.nth0 = double(m.nth0);
    o.Te0 = double(m.Te0);
    o.disk_h = double(m.disk_h);
    o.pow_nth = double(m.pow_nth);
    o.pow_T = double(m.pow_T);
    o.ne_unit = double(m.ne_unit);
    o.te_unit = double(m.te_unit);
    o.b_unit = double(m.b_unit);
    o.freq_cgs = double(m.freq_cgs);
    o.mbh_solar = double(m.mbh_solar);
    o.r_min = double(m.r_min);
    o.r_max = double(m.r_max);
    o.horizon_buffer = double(m.horizon_buffer);
    o.emission_scale = double(m.emission_scale);
    o.absorption_scale = double(m.absorption_scale);
    o.faraday_scale = double(m.faraday_scale);
    o.max_pol_frac = double(m.max_pol_frac);
    o.keplerian_factor = double(m.keplerian_factor);
    o.infall_factor = double(m.infall_factor);
    o.emission_type = m.emission_type;
    o.min_frequency_scale = double(m.min_frequency_scale);
    o.min_sin_theta = double(m.min_sin_theta);
    o.min_thetae = double(m.min_thetae);
    o.min_radius = double(m.min_radius);
    return o;
}

// Sizes an ImageHostData (src/image/result.hpp:9-31) and points a
// kp_image_out at its vectors.
template<class HostData>
kp_image_out bind_outputs(HostData& d, int npix, int nfreq) {
    const size_t img = size_t(npix) * size_t(nfreq);
    d.npix = npix;
    d.nfreq = nfreq;
    d.image_i.assign(img, 0.0);
    d.image_q.assign(img, 0.0);
    d.image_u.assign(img, 0.0);
    d.image_v.assign(img, 0.0);
    for (auto* v : {&d.closure_x, &d.closure_k, &d.final_null, &d.frame_error, &d.det_r, &d.overlap_r11,
                    &d.overlap_r12, &d.overlap_r21, &d.overlap_r22, &d.basis_identity_error,
                    &d.basis_rotation_angle})
        v->assign(size_t(npix), 0.0);
    d.pass_a_steps.assign(size_t(npix), 0);
    d.steps.assign(size_t(npix), 0);
    d.reason.assign(size_t(npix), 0);
    d.has_analysis = 0;
    kp_image_out o;
    o.npix = npix;
    o.nfreq = nfreq;
    o.image_i = d.image_i.data();
    o.image_q = d.image_q.data();
    o.image_u = d.image_u.data();
    o.image_v = d.image_v.data();
    o.closure_x = d.closure_x.data();
    o.closure_k = d.closure_k.data();
    o.final_null = d.final_null.data();
    o.frame_error = d.frame_error.data();
    o.det_r = d.det_r.data();
    o.overlap_r11 = d.overlap_r11.data();
    o.overlap_r12 = d.overlap_r12.data();
    o.overlap_r21 = d.overlap_r21.data();
    o.overlap_r22 = d.overlap_r22.data();
    o.basis_identity_error = d.basis_identity_error.data();
    o.basis_rotation_angle = d.basis_rotation_angle.data();
    o.pass_a_steps = reinterpret_cast<int32_t*>(d.pass_a_steps.data());
    o.steps = reinterpret_cast<int32_t*>(d.steps.data());
    o.reason = reinterpret_cast<int32_t*>(d.reason.data());
    return o;
}

// Process-wide launch options used by the shim (FP64 bit-exact path by
// default; set e.g. precision = KP_PRECISION_MIXED to serve the mixed path).
inline kp_run_options& shim_options() {
    static kp_run_options o = [] {
        kp_run_options d;
        kp_default_run_options(&d);
        return d;
    }();
    return o;
}

// run_riaf_image (src/image/riaf.hpp:12-16).
template<class HostData, class PassA, class Model>
HostData run_riaf_image(const PassA& pass_a, Model model, int radiation_substeps, int timing,
                        int split_transport) {
    (void)split_transport;  // one fused launch: identical results to the split pair
    const kp_pass_a_params p = to_c(pass_a);
    const kp_riaf_model m = to_c_riaf(model);
    HostData out;
    kp_image_out o = bind_outputs(out, p.camera.nx * p.camera.ny, 1);
    kp_run_options opt = shim_options();
    opt.timing = timing;
    const double f = m.freq_cgs;
    throw_on_error(kp_image_riaf(&p, &m, radiation_substeps, &f, 1, &opt, &o));
    return out;
}

// run_riaf_analysis_image (src/image/riaf.hpp:22-28, src/image/riaf.cpp:48-75):
// the image plus the analysis block of ImageHostData (src/image/result.hpp:
// 35-92), with the radial-bin edges and centres the reference's analysis
// driver records (src/image/analysis_driver.hpp:1060-1076).  With
// analysis_config.response enabled, the source-partition response channels
// come back in response_data (4 * channels * npix, the driver's view layout,
// :729-730, 1016-1017) through kp_image_riaf_analysis_response.
template<class HostData, class PassA, class AnalysisCfg, class Model>
HostData run_riaf_analysis_image(const PassA& pass_a, const AnalysisCfg& analysis_config, Model model,
                                 int radiation_substeps, int timing, int split_transport) {
    (void)split_transport;
    const kp_pass_a_params p = to_c(pass_a);
    const kp_riaf_model m = to_c_riaf(model);
    const int npix = p.camera.nx * p.camera.ny;
    const int bins = analysis_config.radial_bins;
    if (bins < 1 || bins > KP_MAX_ANALYSIS_RADIAL_BINS)
        throw std::invalid_argument("analysis_radial_bins must lie in [1, KPOLARIS_MAX_ANALYSIS_RADIAL_BINS]");
    HostData out;
    kp_image_out o = bind_outputs(out, npix, 1);
    kp_analysis_out a;
    auto scalar = [&](auto& v) {
        v.assign(size_t(npix), 0);
        return v.data();
    };
    auto radial = [&](auto& v) {
        v.assign(size_t(bins) * size_t(npix), 0);
        return v.data();
    };
    auto as_i32 = [](int* q) { return reinterpret_cast<int32_t*>(q); };
    static_assert(sizeof(int) == sizeof(int32_t), "int arrays are passed as int32");
    a.radiating_path_length = scalar(out.radiating_path_length);
    a.emission_weight = scalar(out.emission_weight);
    a.emission_weighted_radius = scalar(out.emission_weighted_radius);
    a.emission_weighted_optical_depth_to_camera = scalar(out.emission_weighted_optical_depth_to_camera);
    a.absorption_depth = scalar(out.absorption_depth);
    a.absorption_operator_depth = scalar(out.absorption_operator_depth);
    a.faraday_rotation_depth = scalar(out.faraday_rotation_depth);
    a.faraday_conversion_depth = scalar(out.faraday_conversion_depth);
    a.faraday_operator_depth = scalar(out.faraday_operator_depth);
    a.dominant_emission_radius = scalar(out.dominant_emission_radius);
    a.dominant_emission_region = as_i32(scalar(out.dominant_emission_region));
    a.dominant_ne_cgs = scalar(out.dominant_ne_cgs);
    a.dominant_thetae = scalar(out.dominant_thetae);
    a.dominant_b_cgs = scalar(out.dominant_b_cgs);
    a.dominant_beta = scalar(out.dominant_beta);
    a.dominant_sigma = scalar(out.dominant_sigma);
    a.emission_weighted_ne_cgs = scalar(out.emission_weighted_ne_cgs);
    a.emission_weighted_thetae = scalar(out.emission_weighted_thetae);
    a.emission_weighted_b_cgs = scalar(out.emission_weighted_b_cgs);
    a.emission_weighted_beta = scalar(out.emission_weighted_beta);
    a.emission_weighted_sigma = scalar(out.emission_weighted_sigma);
    a.photon_ring_winding_estimate = scalar(out.photon_ring_winding_estimate);
    a.radiation_substeps = as_i32(scalar(out.radiation_substeps));
    a.radial_stokes_i_contribution = radial(out.radial_stokes_i_contribution);
    a.radial_stokes_q_contribution = radial(out.radial_stokes_q_contribution);
    a.radial_stokes_u_contribution = radial(out.radial_stokes_u_contribution);
    a.radial_stokes_v_contribution = radial(out.radial_stokes_v_contribution);
    a.radial_absorption_depth = radial(out.radial_absorption_depth);
    a.radial_faraday_rotation_depth = radial(out.radial_faraday_rotation_depth);
    a.radial_faraday_conversion_depth = radial(out.radial_faraday_conversion_depth);
    a.radial_faraday_operator_depth = radial(out.radial_faraday_operator_depth);
    a.observer_weighted_radius_i = scalar(out.observer_weighted_radius_i);
    a.observer_weighted_radius_linear = scalar(out.observer_weighted_radius_linear);
    a.observer_weighted_radius_circular = scalar(out.observer_weighted_radius_circular);
    a.intensity_formation_radius_low = scalar(out.intensity_formation_radius_low);
    a.intensity_formation_radius_median = scalar(out.intensity_formation_radius_median);
    a.intensity_formation_radius_high = scalar(out.intensity_formation_radius_high);
    a.linear_formation_radius_low = scalar(out.linear_formation_radius_low);
    a.linear_formation_radius_median = scalar(out.linear_formation_radius_median);
    a.linear_formation_radius_high = scalar(out.linear_formation_radius_high);
    a.circular_formation_radius_low = scalar(out.circular_formation_radius_low);
    a.circular_formation_radius_median = scalar(out.circular_formation_radius_median);
    a.circular_formation_radius_high = scalar(out.circular_formation_radius_high);
    a.los_linear_coherence = scalar(out.los_linear_coherence);
    a.los_circular_coherence = scalar(out.los_circular_coherence);
    a.contribution_closure_max_abs = scalar(out.contribution_closure_max_abs);
    a.contribution_closure_relative_l1 = scalar(out.contribution_closure_relative_l1);
    a.foreground_absorption_depth = scalar(out.foreground_absorption_depth);
    a.foreground_faraday_rotation_depth = scalar(out.foreground_faraday_rotation_depth);
    a.foreground_faraday_conversion_depth = scalar(out.foreground_faraday_conversion_depth);
    a.foreground_faraday_operator_depth = scalar(out.foreground_faraday_operator_depth);
    a.foreground_faraday_operator_fraction = scalar(out.foreground_faraday_operator_fraction);
    kp_analysis_config c;
    c.radial_bins = bins;
    c.radial_min = analysis_config.radial_min;
    c.radial_max = analysis_config.radial_max;
    c.formation_fraction = analysis_config.formation_fraction;
    kp_run_options opt = shim_options();
    opt.timing = timing;
    const auto& rc = analysis_config.response;
    if (rc.enabled()) {
        kp_response_config r;
        kp_default_response_config(&r);
        r.parameter = static_cast<int>(rc.parameter);
        r.partition = static_cast<int>(rc.partition);
        r.step = rc.step;
        r.bins = rc.bins;
        r.edge_count = rc.edge_count;
        for (int i = 0; i < KP_MAX_PARTITION_EDGES; ++i) r.edges[i] = rc.edges[i];
        r.funnel_angle = rc.funnel_angle;
        r.disk_angle = rc.disk_angle;
        r.sigma_boundary = rc.sigma_boundary;
        r.beta_boundary = rc.beta_boundary;
        r.observer_theta = rc.observer_theta;
        r.observer_phi = rc.observer_phi;
        const int channels = kp_response_channels(&r);
        throw_on_error(channels < 0 ? channels : KP_OK);
        out.response_data.assign(size_t(4) * size_t(channels) * size_t(npix), 0.0);
        throw_on_error(kp_image_riaf_analysis_response(&p, &m, radiation_substeps, &c, &r, &opt, &o, &a,
                                                       out.response_data.data()));
    } else {
        throw_on_error(kp_image_riaf_analysis(&p, &m, radiation_substeps, &c, &opt, &o, &a));
    }
    out.has_analysis = 1;
    out.response_config = analysis_config.response;
    out.analysis_radial_bins = bins;
    out.analysis_radial_min = analysis_config.radial_min;
    out.analysis_radial_max = analysis_config.radial_max;
    out.analysis_formation_fraction = analysis_config.formation_fraction;
    out.analysis_radial_bin_edges.assign(size_t(bins) + 1, 0.0);
    out.analysis_radial_bin_centers.assign(size_t(bins), 0.0);
    const double lo = std::log(analysis_config.radial_min), hi = std::log(analysis_config.radial_max);
    for (int b = 0; b <= bins; ++b) {
        out.analysis_radial_bin_edges[size_t(b)] = std::exp(lo + double(b) / double(bins) * (hi - lo));
        if (b < bins) {
            const bool valid = analysis_config.radial_max > analysis_config.radial_min &&
                               analysis_config.radial_min > 0.0;
            out.analysis_radial_bin_centers[size_t(b)] =
                valid ? std::exp(lo + (double(b) + 0.5) / double(bins) * (hi - lo)) : 0.0;
        }
    }
    return out;
}

// run_riaf_multifrequency_image (src/image/riaf.hpp:32-39).
template<class HostData, class PassA, class Model>
HostData run_riaf_multifrequency_image(const PassA& pass_a, Model model, int radiation_substeps,
                                       const std::vector<double>& frequencies,
                                       const std::vector<double>& step_control_frequencies,
                                       int timing, int split_transport) {
    (void)split_transport;
    if (step_control_frequencies.empty())
        throw std::invalid_argument("multifrequency step-control frequency list must not be empty");
    const kp_pass_a_params p = to_c(pass_a);
    const kp_riaf_model m = to_c_riaf(model);
    HostData out;
    const int nfreq = int(frequencies.size());
    if (nfreq < 1 || nfreq > KP_MAX_FREQUENCIES)
        throw std::invalid_argument("multifrequency image chunk size must be between 1 and KPOLARIS_MAX_FREQUENCIES");
    kp_image_out o = bind_outputs(out, p.camera.nx * p.camera.ny, nfreq);
    kp_run_options opt = shim_options();
    opt.timing = timing;
    // a list equal to `frequencies` is the plain image inside the library
    throw_on_error(kp_image_riaf_step_control(&p, &m, radiation_substeps, frequencies.data(), nfreq,
                                              step_control_frequencies.data(),
                                              int(step_control_frequencies.size()), &opt, &o));
    return out;
}

// GRMHDGridRadiationModel<Real> scalars (src/model/grmhd_grid.hpp:52-97)
// -> kp_grmhd_model.  Only FMKS data with thermal emission (emission_type 1
// Pandya or 4 Dexter) is built; the library rejects the rest.
template<class Model>
kp_grmhd_model to_c_grmhd(const Model& m) {
    kp_grmhd_model c;
    kp_default_grmhd_model(&c);
    c.n1 = m.n1;
    c.n2 = m.n2;
    c.n3 = m.n3;
    c.spin = double(m.spin);
    c.gam = double(m.gam);
    c.startx1 = double(m.startx1);
    c.startx2 = double(m.startx2);
    c.startx3 = double(m.startx3);
    c.dx1 = double(m.dx1);
    c.dx2 = double(m.dx2);
    c.dx3 = double(m.dx3);
    c.r_in = double(m.r_in);
    c.r_out = double(m.r_out);
    c.hslope = double(m.hslope);
    c.mks_smooth = double(m.mks_smooth);
    c.poly_alpha = double(m.poly_alpha);
    c.poly_xt = double(m.poly_xt);
    c.poly_norm = double(m.poly_norm);
    c.freq_cgs = double(m.freq_cgs);
    c.mbh_solar = double(m.mbh_solar);
    c.M_unit = double(m.M_unit);
    c.trat_small = double(m.trat_small);
    c.trat_large = double(m.trat_large);
    c.beta_crit = double(m.beta_crit);
    c.sigma_cut = double(m.sigma_cut);
    c.sigma_cut_high = double(m.sigma_cut_high);
    c.ne_factor = double(m.ne_factor);
    c.emission_type = m.emission_type;
    c.emission_scale = double(m.emission_scale);
    c.absorption_scale = double(m.absorption_scale);
    c.faraday_scale = double(m.faraday_scale);
    c.max_pol_frac = double(m.max_pol_frac);
    c.has_derived_scalars = m.has_derived_scalars;
    return c;
}

// A resident grid for a reference model, uploaded on first use and kept per
// primitive View (the reference's models share their Views by reference
// counting, so a View's data pointer identifies a snapshot).  The primitives
// are mirrored to the host (device memory in a CUDA build of the reference)
// and narrowed to FP32, the layout the library's grids hold.  Call
// release_grids() when the snapshots go away.
inline std::map<const void*, kp_grid*>& grid_cache() {
    static std::map<const void*, kp_grid*> cache;
    return cache;
}

inline void release_grids() {
    for (auto& kv : grid_cache()) kp_grid_release(kv.second);
    grid_cache().clear();
}

template<class Model>
kp_grid* grid_for(const Model& m) {
    const void* key = m.prims.data();
    auto it = grid_cache().find(key);
    if (it != grid_cache().end()) return it->second;
    auto host = Kokkos::create_mirror_view_and_copy(Kokkos::HostSpace(), m.prims);
    std::vector<float> prims(host.extent(0));
    for (size_t i = 0; i < prims.size(); ++i) prims[i] = float(host(i));
    const kp_grmhd_model c = to_c_grmhd(m);
    kp_grid* g = nullptr;
    throw_on_error(kp_grid_upload(&c, prims.data(), shim_options().device, &g));
    grid_cache()[key] = g;
    return g;
}

// run_grmhd_image (src/image/grmhd.hpp:12-18), FMKS backend.
template<class HostData, class PassA, class Model>
HostData run_grmhd_image(const PassA& pass_a, Model model, int radiation_substeps, int timing,
                         int split_transport) {
    (void)split_transport;
    const kp_pass_a_params p = to_c(pass_a);
    kp_grid* g = grid_for(model);
    HostData out;
    kp_image_out o = bind_outputs(out, p.camera.nx * p.camera.ny, 1);
    kp_run_options opt = shim_options();
    opt.timing = timing;
    const double f = double(model.freq_cgs);
    throw_on_error(kp_image_grmhd(&p, g, radiation_substeps, &f, 1, &opt, &o));
    return out;
}

// run_grmhd_multifrequency_image (src/image/grmhd.hpp:30-37).
template<class HostData, class PassA, class Model, class Real>
HostData run_grmhd_multifrequency_image(const PassA& pass_a, Model model, int radiation_substeps,
                                        const std::vector<Real>& frequencies,
                                        const std::vector<Real>& step_control_frequencies, int timing) {
    if (step_control_frequencies.empty())
        throw std::invalid_argument("multifrequency step-control frequency list must not be empty");
    const int nfreq = int(frequencies.size());
    if (nfreq < 1 || nfreq > KP_MAX_FREQUENCIES)
        throw std::invalid_argument("multifrequency image chunk size must be between 1 and KPOLARIS_MAX_FREQUENCIES");
    const kp_pass_a_params p = to_c(pass_a);
    kp_grid* g = grid_for(model);
    HostData out;
    kp_image_out o = bind_outputs(out, p.camera.nx * p.camera.ny, nfreq);
    kp_run_options opt = shim_options();
    opt.timing = timing;
    std::vector<double> f(frequencies.begin(), frequencies.end());
    std::vector<double> ctl(step_control_frequencies.begin(), step_control_frequencies.end());
    throw_on_error(kp_image_grmhd_step_control(&p, g, radiation_substeps, f.data(), nfreq, ctl.data(), int(ctl.size()),
                                               &opt, &o));
    return out;
}

// A slow-light image over resident snapshots (the images
// run_slow_light_batch_metric produces in its default decoupled step mode,
// src/image/slow_light_batch_driver.hpp:107-368, for one observation time):
// `models` are the loaded snapshots at `times`.
template<class HostData, class PassA, class Model, class Real>
HostData run_slow_light_image(const PassA& pass_a, const std::vector<Model>& models, const std::vector<Real>& times,
                              Real observation_time, const std::vector<Real>& frequencies) {
    if (models.size() != times.size()) throw std::runtime_error("slow-light dump path/time list size mismatch");
    if (models.size() < 2) throw std::runtime_error("slow-light requires at least two dump time slices");
    const int nfreq = int(frequencies.size());
    const kp_pass_a_params p = to_c(pass_a);
    std::vector<const kp_grid*> grids;
    for (const auto& m : models) grids.push_back(grid_for(m));
    std::vector<double> t(times.begin(), times.end()), f(frequencies.begin(), frequencies.end());
    HostData out;
    kp_image_out o = bind_outputs(out, p.camera.nx * p.camera.ny, nfreq);
    kp_run_options opt = shim_options();
    throw_on_error(kp_image_grmhd_slow_light(&p, grids.data(), t.data(), int(grids.size()), double(observation_time),
                                             1, f.data(), nfreq, &opt, &o));
    return out;
}

}  // namespace kpolaris_b200
