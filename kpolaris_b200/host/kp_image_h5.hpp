// kp_image_h5.hpp -- the image tool's HDF5 output: the kpolaris_image schema,
// version 1 (docs/hdf5_schema.md "Image schema"; the writer of
// tools/kpolaris_model_image.cpp:4284-4840 for model=riaf), written through
// the minimal HDF5 writer of kp_hdf5.hpp.
//
// Layout: root provenance and run attributes, /header, /parameters/{camera,
// spacetime,integration,radiation}, /grid (x, y, frequency_hz), /results
// (summary attributes, per-frequency sums and fluxes), /frame_0/freq_<fi>
// (I, Q, U, V and the invariant *_inv images, [ny][nx] float64) and
// /frame_0/diagnostics ([ny][nx] per-pixel diagnostics).  Attribute names,
// types and values follow the reference's writer; string attributes are
// fixed-length ASCII instead of variable-length (readers decode both), and
// the provenance attributes name this library.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "kp_hdf5.hpp"
#include "kpolaris_image_options.hpp"

namespace kpb {

// One frequency of a traced image, packed like the CSV rows.
struct H5Frequency {
    double frequency;
    const double* inv[4];    // I, Q, U, V invariant [npix]
    const double* nu[4];     // I, Q, U, V specific intensity [npix]
    double sum_inv[4];
    double flux_jy[4];
};

// The geometry-level outputs shared by every frequency.
struct H5Diagnostics {
    const int32_t* reason;
    const int32_t* pass_a_steps;
    const int32_t* steps;
    const int32_t* total_steps;  // as packed (pass A + pass B of returned rays)
    const double* diag[11];  // closure_x .. basis_rotation_angle, kp_image_out order
};

inline std::string h5_frequency_list(const std::vector<double>& f) {
    std::ostringstream out;
    out.precision(17);
    for (size_t i = 0; i < f.size(); ++i) {
        if (i) out << ',';
        out << f[i];
    }
    return out.str();
}

// The polarization and camera convention attributes of an image file
// (tools/kpolaris_conventions_output.hpp:8-48).
inline void h5_camera_conventions(kph5::Group& g, const std::string& evpa_0) {
    const bool north = evpa_0 == "N";
    g.attr("polarization_conventions_version", "2");
    g.attr("metric_signature", "-+++");
    g.attr("wavevector_direction", "future_directed; Pass A uses negative affine steps, Pass B positive");
    g.attr("camera_azimuth_convention", "pinhole: native phi=0; parallel: center in Cartesian x-z plane; no camera roll");
    g.attr("sky_orientation", "image north=up, east=left by convention; celestial position angle not assigned");
    g.attr("screen_handedness", "right_handed (e1,e2,photon_direction) in the observer rest frame");
    g.attr("stokes_definition", "I=<|E1|^2+|E2|^2>; Q=<|E1|^2-|E2|^2>; U=2Re<E1 E2*>; V=-2Im<E1 E2*>");
    g.attr("electric_field_phase_convention", "Re[E exp(-i omega t)] in a local right-handed screen");
    g.attr("stokes_basis_definition",
           north ? "output basis (e2,-e1), a passive 90-degree rotation of the internal camera screen"
                 : "output basis (e1,e2), the internal camera screen");
    g.attr("evpa_definition",
           north ? "0.5 atan2(U,Q), modulo pi; zero=image north, increasing toward image east in the distant-observer "
                   "limit; undefined at Q=U=0"
                 : "0.5 atan2(U,Q), modulo pi; zero=horizontal (W), increasing toward vertical (N) in the "
                   "distant-observer limit; undefined at Q=U=0");
    g.attr("image_pixel_order", "pixel=iy*nx+ix; increasing ix right, iy up");
    g.attr("image_axis_geometry", "phi=0 distant-observer limit: +x=+e_phi, +y=-e_theta (projected coordinate +z)");
    g.attr("pinhole_screen_geometry",
           "project tetrad e1,e2 perpendicular to each k, then Gram-Schmidt; gnomonic image chart");
    g.attr("output_stokes_transform", north ? "I,Q,U,V=(I_camera,-Q_camera,-U_camera,V_camera); passive 90-degree basis rotation"
                                            : "identity; I,Q,U,V=(I_camera,Q_camera,U_camera,V_camera)");
    g.attr("image_array_order", "y,x");
    g.attr("image_display_origin", "lower");
}

// The RIAF model's metadata (write_hdf5_model_metadata for
// RIAFAnalyticRadiationModel, tools/kpolaris_model_image.cpp:2888-2917).
inline void h5_riaf_metadata(kph5::Group& g, const kp_riaf_model& m) {
    g.attr("riaf_r_min", m.r_min);
    g.attr("riaf_r_max", m.r_max);
    g.attr("riaf_nth0", m.nth0);
    g.attr("riaf_Te0", m.Te0);
    g.attr("riaf_disk_h", m.disk_h);
    g.attr("riaf_pow_nth", m.pow_nth);
    g.attr("riaf_pow_T", m.pow_T);
    g.attr("riaf_ne_unit", m.ne_unit);
    g.attr("riaf_te_unit", m.te_unit);
    g.attr("riaf_mbh_solar", m.mbh_solar);
    g.attr("riaf_keplerian_factor", m.keplerian_factor);
    g.attr("riaf_infall_factor", m.infall_factor);
    g.attr("emission_type", m.emission_type);
    g.attr("emission_fit", emission_fit_name(m.emission_type));
    const double l_unit = length_unit_cm(m.mbh_solar);
    g.attr("dlambda_scale", l_unit / std::max(m.freq_cgs, 1.0));  // riaf.hpp:76-85
}

// A GRMHD model's metadata (write_model_metadata for GRMHDRadiationModel,
// tools/kpolaris_model_image.cpp:739-787): the shared grmhd_* keys and the
// same under the model's own prefix.  FMKS data, thermal fits.
inline void h5_grmhd_metadata(kph5::Group& g, const kp_grmhd_model& m, const std::string& prefix, double freq) {
    const double l_unit = 6.67430e-8 * m.mbh_solar * 1.98847e33 / (2.99792458e10 * 2.99792458e10);
    const double dls = l_unit / std::max(freq, 1.0);  // grmhd_grid.hpp:159-161
    for (const std::string& pre : {std::string("grmhd"), prefix}) {
        g.attr(pre + "_n1", m.n1);
        g.attr(pre + "_n2", m.n2);
        g.attr(pre + "_n3", m.n3);
        g.attr(pre + "_M_unit", m.M_unit);
        g.attr(pre + "_mbh_solar", m.mbh_solar);
        g.attr(pre + "_trat_small", m.trat_small);
        g.attr(pre + "_trat_large", m.trat_large);
        g.attr(pre + "_beta_crit", m.beta_crit);
        g.attr(pre + "_sigma_cut", m.sigma_cut);
        g.attr(pre + "_sigma_cut_high", m.sigma_cut_high);
        g.attr(pre + "_interpolate_derived_scalars", m.has_derived_scalars);
        g.attr(pre + "_precomputed_fluid_state", 0);
        g.attr(pre + "_data_coordinate_system", int(KP_COORD_FMKS));
        g.attr(pre + "_radial_coordinate_log", 1);
        g.attr(pre + "_dlambda_scale", dls);
    }
    g.attr("emission_type", m.emission_type);
    g.attr("emission_fit", emission_fit_name(m.emission_type));
}

inline void h5_provenance(kph5::Group& g) {
    g.attr("schema", "kpolaris_image");
    g.attr("schema_version", 1);
    g.attr("code", "KPolaris");
    g.attr("code_version", "b200-abi-" + std::to_string(kp_abi_version()));
    g.attr("code_revision", "kpolaris_b200");
    g.attr("code_source_dirty", -1);
    g.attr("code_source_fingerprint", "unknown");
#if defined(__clang__)
    g.attr("compiler_id", "Clang");
#elif defined(__GNUC__)
    g.attr("compiler_id", "GNU");
#else
    g.attr("compiler_id", "unknown");
#endif
#ifdef __VERSION__
    g.attr("compiler_version", __VERSION__);
#else
    g.attr("compiler_version", "unknown");
#endif
    g.attr("build_type", "Release");
    g.attr("image_backend", "KPolaris-B200 (sm_100a C ABI)");
}

// `grmhd`: the model of a GRMHD image (model=iharm), or null for RIAF.
inline void write_image_h5(const std::string& path, const ImageOptions& opt, const std::string& params_path,
                           const kp_pass_a_params& pass_a, const std::vector<double>& freqs,
                           const std::vector<H5Frequency>& images, const H5Diagnostics& dg, const FluxScale& fs,
                           const kp_grmhd_model* grmhd = nullptr) {
    const int nx = opt.nx, ny = opt.ny, npix = nx * ny;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    const double jy = fs.valid ? fs.jy_per_pixel : nan;
    const double sr = fs.valid ? fs.pixel_solid_angle_sr : nan;
    // pixel-centre grid (tools/kpolaris_model_image.cpp:3989-3998, 4124-4130)
    const double x_extent = pass_a.camera.xspan > 0.0 ? 2.0 * pass_a.camera.xspan : pass_a.camera.fov;
    const double y_extent = pass_a.camera.yspan > 0.0 ? 2.0 * pass_a.camera.yspan
                            : (pass_a.camera.xspan > 0.0 ? 2.0 * pass_a.camera.xspan * double(ny) / double(nx)
                               : (pass_a.camera.fov_y > 0.0 ? pass_a.camera.fov_y : pass_a.camera.fov));
    const double dx = x_extent / double(nx), dy = y_extent / double(ny);
    const double xh = 0.5 * x_extent, yh = 0.5 * y_extent;
    const std::string grid_units = opt.camera == "pinhole" ? "dimensionless_slope" : "M";
    std::vector<double> gx(static_cast<size_t>(nx)), gy(static_cast<size_t>(ny));
    for (int i = 0; i < nx; ++i) gx[size_t(i)] = (double(i) + 0.5) * dx - xh + pass_a.camera.x_offset;
    for (int j = 0; j < ny; ++j) gy[size_t(j)] = (double(j) + 0.5) * dy - yh + pass_a.camera.y_offset;
    const kp_riaf_model first_model = to_riaf_model(opt, freqs.front());
    const double mbh = model_mbh_solar(opt);
    auto model_metadata = [&](kph5::Group& g, double freq) {
        if (grmhd) {
            h5_grmhd_metadata(g, *grmhd, opt.model, freq);
        } else {
            h5_riaf_metadata(g, freq == freqs.front() ? first_model : to_riaf_model(opt, freq));
        }
    };
    const int chunk = effective_chunk_size(opt, freqs.size());
    const std::string flist = h5_frequency_list(freqs);
    const std::string metric = metric_name_of(opt.coordinate);
    const std::string eff = params_path;

    kph5::File file;
    kph5::Group& root = file.root();
    h5_provenance(root);
    root.attr("model", opt.model);
    root.attr("parameter_file", opt.parameter_file);
    root.attr("effective_parameter_file", eff);
    root.attr("camera", opt.camera);
    root.attr("coordinate", opt.coordinate);
    root.attr("metric", metric);
    root.attr("stokes_convention", "camera_frame");
    root.attr("polarization_basis", "camera_screen");
    root.attr("evpa_0", opt.evpa_0);
    h5_camera_conventions(root, opt.evpa_0);
    root.attr("nx", nx);
    root.attr("ny", ny);
    root.attr("nfreq", int(freqs.size()));
    root.attr("frequency_list_hz", flist);
    root.attr("frequency_hz", freqs.front());
    root.attr("camera_radius", opt.radius);
    root.attr("inclination_rad", opt.inclination);
    root.attr("fov", opt.fov);
    root.attr("fovy", opt.fovy > 0.0 ? opt.fovy : opt.fov);
    root.attr("dsource", opt.dsource_pc);
    root.attr("fovx_dsource", opt.effective_fovx_dsource);
    root.attr("fovy_dsource", opt.effective_fovy_dsource);
    root.attr("mbh_solar", mbh);
    root.attr("image_width_x_M", opt.image_width_x);
    root.attr("image_width_y_M", opt.image_width_y);
    root.attr("x_offset", pass_a.camera.x_offset);
    root.attr("y_offset", pass_a.camera.y_offset);
    root.attr("use_pinhole_pixel_bias", opt.use_pinhole_pixel_bias);
    root.attr("pinhole_pixel_bias", opt.pinhole_pixel_bias);
    root.attr("grid_units", grid_units);
    root.attr("x_half_extent", xh);
    root.attr("y_half_extent", yh);
    root.attr("dx", dx);
    root.attr("dy", dy);
    root.attr("flux_scale_valid", fs.valid ? 1 : 0);
    root.attr("l_unit_cm", fs.l_unit_cm);
    root.attr("dsource_cm", fs.dsource_cm);
    root.attr("pixel_solid_angle_sr", sr);
    root.attr("intensity_to_flux_jy_per_pixel", jy);
    root.attr("image_stokes_units", "cgs_specific_intensity");
    root.attr("flux_density_unit", "Jy");
    const double yspan_out = opt.yspan > 0.0 ? opt.yspan : opt.xspan * double(ny) / double(nx);
    if (opt.xspan > 0.0) {
        root.attr("xspan", opt.xspan);
        root.attr("yspan", yspan_out);
    }
    root.attr("spin", opt.spin);
    root.attr("step", opt.step);
    root.attr("adaptive", opt.adaptive);
    root.attr("adaptive_tolerance", opt.adaptive_tolerance);
    root.attr("min_step", opt.min_step);
    root.attr("max_step", opt.max_step);
    root.attr("max_radiation_step", opt.max_radiation_step);
    root.attr("max_radiation_depth", opt.max_radiation_depth);
    root.attr("max_absorption_depth", opt.max_absorption_depth);
    root.attr("max_faraday_depth", opt.max_faraday_depth);
    root.attr("closure_x_warning", opt.closure_x_warning);
    root.attr("closure_k_warning", opt.closure_k_warning);
    root.attr("frame_error_warning", opt.frame_error_warning);
    root.attr("basis_identity_warning", opt.basis_identity_warning);
    root.attr("split_transport", opt.split_transport);
    root.attr("multifrequency_chunk_size", opt.multifrequency_chunk_size);
    root.attr("effective_multifrequency_chunk_size", chunk);
    root.attr("analysis_mode", opt.analysis_mode);
    root.attr("analysis_radial_bins", 16);
    root.attr("equatorial_h_over_r", opt.equatorial_h_over_r);
    root.attr("equatorial_samples", opt.equatorial_samples);
    root.attr("faraday_rotation", opt.faraday_rotation);
    root.attr("equatorial_emission_definition",
              "0 disabled; otherwise seed emission only where abs(cos(theta_BL))=abs(z_KS)/r_BL <= h_over_r; h is "
              "half-height; 1 retains all emission");
    root.attr("equatorial_transfer_definition",
              "only jI,jQ,jU,jV are masked; absorption and Faraday conversion remain everywhere in the configured "
              "plasma domain; rhoV is independently controlled by faraday_rotation");
    root.attr("equatorial_sampling",
              "limit accepted-step height-ratio variation to 2*h_over_r/equatorial_samples and refine first crossed "
              "wedge surface with the same RK composition");
    root.attr("direct_only", opt.direct_only);
    root.attr("emission_segment", opt.direct_only ? "n0_vertical_turn" : "all");
    root.attr("slow_light", opt.slow_light);
    root.attr("slow_light_compiled", 0);
    root.attr("slow_light_time_probe", opt.slow_light_time_probe);
    root.attr("analysis_compiled", 0);
    root.attr("radiation_substeps", opt.radiation_substeps);
    root.attr("max_steps", opt.max_steps);
    root.attr("inner_radius", opt.inner_radius);
    root.attr("outer_radius", opt.outer_radius);
    model_metadata(root, freqs.front());

    kph5::Group& header = root.group("header");
    h5_provenance(header);
    header.attr("image_layout", "/frame_0/freq_i");
    header.attr("diagnostics_layout", "/frame_0/diagnostics");
    header.attr("analysis_layout", freqs.size() > 1 ? "/frame_0/freq_N/analysis" : "/frame_0/analysis");
    header.attr("parameter_file", opt.parameter_file);
    header.attr("effective_parameter_file", eff);
    header.attr("stokes_convention", "camera_frame");
    header.attr("polarization_basis", "camera_screen");
    header.attr("evpa_0", opt.evpa_0);

    kph5::Group& params = root.group("parameters");
    params.attr("parameter_file", opt.parameter_file);
    params.attr("effective_parameter_file", eff);
    {
        kph5::Group& g = params.group("camera");
        g.attr("model", opt.camera);
        g.attr("coordinate", opt.coordinate);
        g.attr("nx", nx);
        g.attr("ny", ny);
        g.attr("radius", opt.radius);
        g.attr("inclination_rad", opt.inclination);
        g.attr("fov", opt.fov);
        g.attr("fovy", opt.fovy > 0.0 ? opt.fovy : opt.fov);
        g.attr("dsource", opt.dsource_pc);
        g.attr("fovx_dsource", opt.effective_fovx_dsource);
        g.attr("fovy_dsource", opt.effective_fovy_dsource);
        g.attr("mbh_solar", mbh);
        g.attr("image_width_x_M", opt.image_width_x);
        g.attr("image_width_y_M", opt.image_width_y);
        g.attr("x_offset", pass_a.camera.x_offset);
        g.attr("y_offset", pass_a.camera.y_offset);
        g.attr("grid_units", grid_units);
        g.attr("x_half_extent", xh);
        g.attr("y_half_extent", yh);
        g.attr("dx", dx);
        g.attr("dy", dy);
        g.attr("flux_scale_valid", fs.valid ? 1 : 0);
        g.attr("l_unit_cm", fs.l_unit_cm);
        g.attr("dsource_cm", fs.dsource_cm);
        g.attr("pixel_solid_angle_sr", sr);
        g.attr("intensity_to_flux_jy_per_pixel", jy);
        g.attr("use_pinhole_pixel_bias", opt.use_pinhole_pixel_bias);
        g.attr("pinhole_pixel_bias", opt.pinhole_pixel_bias);
        if (opt.xspan > 0.0) {
            g.attr("xspan", opt.xspan);
            g.attr("yspan", yspan_out);
        }
    }
    {
        kph5::Group& g = params.group("spacetime");
        g.attr("metric", metric);
        g.attr("coordinate", opt.coordinate);
        g.attr("mass", 1.0);
        g.attr("mbh_solar", mbh);
        g.attr("l_unit_cm", fs.l_unit_cm);
        g.attr("spin", opt.spin);
    }
    {
        kph5::Group& g = params.group("integration");
        g.attr("step", opt.step);
        g.attr("adaptive", opt.adaptive);
        g.attr("adaptive_tolerance", opt.adaptive_tolerance);
        g.attr("min_step", opt.min_step);
        g.attr("max_step", opt.max_step);
        g.attr("max_radiation_step", opt.max_radiation_step);
        g.attr("max_radiation_depth", opt.max_radiation_depth);
        g.attr("max_absorption_depth", opt.max_absorption_depth);
        g.attr("max_faraday_depth", opt.max_faraday_depth);
        g.attr("closure_x_warning", opt.closure_x_warning);
        g.attr("closure_k_warning", opt.closure_k_warning);
        g.attr("frame_error_warning", opt.frame_error_warning);
        g.attr("basis_identity_warning", opt.basis_identity_warning);
        g.attr("split_transport", opt.split_transport);
        g.attr("analysis_mode", opt.analysis_mode);
        g.attr("analysis_radial_bins", 16);
        g.attr("slow_light", opt.slow_light);
        g.attr("slow_light_compiled", 0);
        g.attr("slow_light_time_probe", opt.slow_light_time_probe);
        g.attr("max_steps", opt.max_steps);
        g.attr("inner_radius", opt.inner_radius);
        g.attr("outer_radius", opt.outer_radius);
        g.attr("radiation_substeps", opt.radiation_substeps);
    }
    {
        kph5::Group& g = params.group("radiation");
        g.attr("model", opt.model);
        g.attr("mbh_solar", mbh);
        g.attr("slow_light", opt.slow_light);
        g.attr("slow_light_compiled", 0);
        g.attr("slow_light_time_probe", opt.slow_light_time_probe);
        g.attr("equatorial_h_over_r", opt.equatorial_h_over_r);
        g.attr("equatorial_samples", opt.equatorial_samples);
        g.attr("faraday_rotation", opt.faraday_rotation);
        g.attr("nfreq", int(freqs.size()));
        g.attr("multifrequency_chunk_size", opt.multifrequency_chunk_size);
        g.attr("effective_multifrequency_chunk_size", chunk);
        g.attr("frequency_hz", freqs.front());
        g.attr("frequency_list_hz", flist);
        g.attr("freq_spacing", opt.freq_spacing);
        g.attr("stokes_convention", "camera_frame");
        g.dataset("frequencies", {uint64_t(freqs.size())}, freqs.data());
        model_metadata(g, freqs.front());
    }
    {
        kph5::Group& g = root.group("grid");
        g.attr("units", grid_units);
        g.dataset("x", {uint64_t(nx)}, gx.data());
        g.dataset("y", {uint64_t(ny)}, gy.data());
        g.dataset("frequency_hz", {uint64_t(freqs.size())}, freqs.data());
    }
    // /results: diagnostics summary (summarize_diagnostics,
    // tools/kpolaris_model_image_output.cpp:23-60) and step statistics over
    // the image, sums and fluxes per frequency
    {
        kph5::Group& g = root.group("results");
        double mcx = 0.0, mck = 0.0, mfe = 0.0, mbi = 0.0;
        int mcx_p = -1, returned = 0;
        int wx = 0, wk = 0, wf = 0, wb = 0, wany = 0;
        long long sa = 0, sb = 0;
        int ma = 0, mb = 0, mt = 0;
        auto upd = [](double v, int p, double& m, int& mp) {
            if (!std::isfinite(v)) return;
            if (std::fabs(v) > m) {
                m = std::fabs(v);
                mp = p;
            }
        };
        auto warn = [](double v, double thr) { return thr > 0.0 && v > thr; };
        for (int p = 0; p < npix; ++p) {
            sa += dg.pass_a_steps[p];
            sb += dg.steps[p];
            ma = std::max(ma, int(dg.pass_a_steps[p]));
            mb = std::max(mb, int(dg.steps[p]));
            mt = std::max(mt, int(dg.pass_a_steps[p] + dg.steps[p]));
            if (dg.reason[p] != KP_REASON_REACHED_CAMERA) continue;
            ++returned;
            int dummy = -1;
            upd(dg.diag[0][p], p, mcx, mcx_p);
            upd(dg.diag[1][p], p, mck, dummy);
            upd(dg.diag[3][p], p, mfe, dummy);
            upd(dg.diag[9][p], p, mbi, dummy);
            const bool a = warn(std::fabs(dg.diag[0][p]), opt.closure_x_warning);
            const bool b = warn(std::fabs(dg.diag[1][p]), opt.closure_k_warning);
            const bool c = warn(std::fabs(dg.diag[3][p]), opt.frame_error_warning);
            const bool d = warn(std::fabs(dg.diag[9][p]), opt.basis_identity_warning);
            wx += a;
            wk += b;
            wf += c;
            wb += d;
            wany += (a || b || c || d);
        }
        g.attr("pixels", npix);
        g.attr("returned", returned);
        g.attr("nfreq", int(freqs.size()));
        g.attr("max_closure_x", mcx);
        g.attr("max_closure_k", mck);
        g.attr("max_frame_error", mfe);
        g.attr("max_basis_identity_error", mbi);
        g.attr("max_closure_x_ix", mcx_p >= 0 ? mcx_p % nx : -1);
        g.attr("max_closure_x_iy", mcx_p >= 0 ? mcx_p / nx : -1);
        g.attr("closure_x_warning_count", wx);
        g.attr("closure_k_warning_count", wk);
        g.attr("frame_error_warning_count", wf);
        g.attr("basis_identity_warning_count", wb);
        g.attr("diagnostic_warning_count", wany);
        g.attr("mean_pass_a_steps", double(sa) / double(npix));
        g.attr("mean_pass_b_steps", double(sb) / double(npix));
        g.attr("mean_total_steps", double(sa + sb) / double(npix));
        g.attr("max_pass_a_steps", ma);
        g.attr("max_pass_b_steps", mb);
        g.attr("max_total_steps", mt);
        g.attr("sum_I_inv", images.front().sum_inv[0]);
        g.attr("sum_Q_inv", images.front().sum_inv[1]);
        g.attr("sum_U_inv", images.front().sum_inv[2]);
        g.attr("sum_V_inv", images.front().sum_inv[3]);
        g.attr("intensity_to_flux_jy_per_pixel", jy);
        std::vector<double> sums[4], fluxes[4];
        for (const auto& im : images)
            for (int k = 0; k < 4; ++k) {
                sums[k].push_back(im.sum_inv[k]);
                fluxes[k].push_back(im.flux_jy[k]);
            }
        const char* nm[4] = {"I", "Q", "U", "V"};
        for (int k = 0; k < 4; ++k) g.attr(std::string("flux_") + nm[k] + "_Jy", fluxes[k].front());
        g.dataset("frequency_hz", {uint64_t(freqs.size())}, freqs.data());
        for (int k = 0; k < 4; ++k)
            g.dataset(std::string("sum_") + nm[k] + "_inv_by_freq", {uint64_t(images.size())}, sums[k].data());
        for (int k = 0; k < 4; ++k)
            g.dataset(std::string("flux_") + nm[k] + "_Jy_by_freq", {uint64_t(images.size())}, fluxes[k].data());
    }
    {
        kph5::Group& frame = root.group("frame_0");
        frame.attr("index", 0);
        frame.attr("nfreq", int(freqs.size()));
        const std::vector<uint64_t> dims = {uint64_t(ny), uint64_t(nx)};
        const char* nm[4] = {"I", "Q", "U", "V"};
        for (size_t fi = 0; fi < images.size(); ++fi) {
            const H5Frequency& im = images[fi];
            kph5::Group& g = frame.group("freq_" + std::to_string(fi));
            g.attr("index", int(fi));
            g.attr("frequency", im.frequency);
            g.attr("frequency_hz", im.frequency);
            g.attr("stokes_convention", "camera_frame");
            g.attr("polarization_basis", "camera_screen");
            g.attr("evpa_0", opt.evpa_0);
            g.attr("stokes_units", "cgs_specific_intensity");
            g.attr("intensity_to_flux_jy_per_pixel", jy);
            for (int k = 0; k < 4; ++k) g.attr(std::string("flux_") + nm[k] + "_Jy", im.flux_jy[k]);
            model_metadata(g, im.frequency);
            for (int k = 0; k < 4; ++k) g.dataset(nm[k], dims, im.nu[k]);
            for (int k = 0; k < 4; ++k) g.dataset(std::string(nm[k]) + "_inv", dims, im.inv[k]);
        }
        kph5::Group& d = frame.group("diagnostics");
        d.dataset("reason", dims, dg.reason);
        d.dataset("pass_a_steps", dims, dg.pass_a_steps);
        d.dataset("steps", dims, dg.steps);
        d.dataset("total_steps", dims, dg.total_steps);
        const char* dn[11] = {"closure_x", "closure_k", "final_null", "frame_error", "det_r", "overlap_r11",
                              "overlap_r12", "overlap_r21", "overlap_r22", "basis_identity_error",
                              "basis_rotation_angle"};
        for (int k = 0; k < 11; ++k) d.dataset(dn[k], dims, dg.diag[k]);
    }
    file.write(path);
}

}  // namespace kpb
