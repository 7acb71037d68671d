// kp_model_image -- command-line image tool for the RIAF image path and
// iharm and KHARMA GRMHD dumps, the counterpart of the reference's
// kpolaris_model_image for model=riaf, iharm and kharma
// (tools/kpolaris_model_image.cpp:4908-5195 main, :3909-4260 run_model,
// :2561-2800 output packing, :4136-4245 CSV output).  A dump is read by
// kp_iharm_read / kp_kharma_read and kp_grid_load_iharm /
// kp_grid_load_kharma and imaged with kp_image_grmhd_step_control.
//
//   kp_model_image --parameter_file=run.par [--key=value ...]
//
// Reads the reference's parameter files and overrides
// (kpolaris_image_options.hpp), traces the image through the C ABI
// (kp_image_riaf, frequencies in chunks of at most KP_MAX_FREQUENCIES),
// packs each frequency with kp_pack_image, writes the image -- the
// kpolaris_image v1 HDF5 layout (kp_image_h5.hpp) for format=hdf5 or an
// output ending in .h5 with format=auto, else the CSV image format -- and
// <output>.params, and prints the tool's summary lines.
//
// Extra keys: kp_precision=fp64|mixed, kp_schedule=auto|per_pixel|
// persistent|graph (auto: per-pixel kernel for fp64, wavefront engine for
// mixed), kp_device=N, kp_print_resolved=1 (print the resolved settings and
// exit, no GPU), kp_dry_run=1 (resolve and write <output>.params, no GPU).
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "kp_image_h5.hpp"
#include "kpolaris_image_options.hpp"

namespace {

struct HostImage {
    std::vector<double> i, q, u, v;
    std::vector<double> diag[11];
    std::vector<int32_t> pass_a_steps, steps, reason;

    HostImage(int npix, int nfreq)
        : i(size_t(npix) * nfreq), q(i.size()), u(i.size()), v(i.size()), pass_a_steps(npix), steps(npix),
          reason(npix) {
        for (auto& d : diag) d.assign(size_t(npix), 0.0);
    }
    kp_image_out view(int npix, int nfreq) {
        kp_image_out o;
        o.npix = npix;
        o.nfreq = nfreq;
        o.image_i = i.data();
        o.image_q = q.data();
        o.image_u = u.data();
        o.image_v = v.data();
        double** d[11] = {&o.closure_x, &o.closure_k, &o.final_null, &o.frame_error, &o.det_r, &o.overlap_r11,
                          &o.overlap_r12, &o.overlap_r21, &o.overlap_r22, &o.basis_identity_error,
                          &o.basis_rotation_angle};
        for (int k = 0; k < 11; ++k) *d[k] = diag[k].data();
        o.pass_a_steps = pass_a_steps.data();
        o.steps = steps.data();
        o.reason = reason.data();
        return o;
    }
};

struct PackedFrequency {
    double frequency = 0.0;
    std::vector<double> inv[4], nu[4];
    std::vector<int32_t> total_steps;
    kp_packed_image p{};
};

void check(int rc, const char* what) {
    if (rc != KP_OK) throw std::runtime_error(std::string(what) + ": " + kp_last_error());
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void report_timing(const kpb::ImageOptions& o, const char* name, double s) {
    if (o.timing) std::cout << "timing " << name << " " << s << " s\n";
}

int run(const std::vector<std::string>& args) {
    const auto t_start = std::chrono::steady_clock::now();
    kpb::ImageOptions opt = kpb::parse_options(args);
    kpb::finalize_options(opt);
    // model=iharm: the dump's header settles the spin, the radii and the
    // coordinate map (read on the host; no device yet)
    const bool grmhd = kpb::grmhd_model(opt);
    const bool kharma = opt.model == "kharma";
    kp_grmhd_model gm{};
    kp_iharm_options io{};
    if (grmhd) {
        io = kpb::to_iharm_options(opt);
        if (kharma)
            check(kp_kharma_read(opt.kharma_dump.c_str(), &io, opt.kharma_reverse_field, &gm, nullptr, 0),
                  "kp_kharma_read");
        else
            check(kp_iharm_read(opt.iharm_dump.c_str(), &io, &gm, nullptr, 0), "kp_iharm_read");
        kpb::resolve_grmhd_geometry(opt, gm);
    }
    if (opt.kp_print_resolved) {
        kpb::print_resolved(std::cout, opt);
        return 0;
    }
    const std::vector<double> freqs = kpb::build_frequency_grid(opt);
    kp_pass_a_params pass_a = kpb::to_pass_a(opt);
    if (grmhd) kpb::apply_fmks_map(pass_a, gm);
    const bool hdf5 = opt.output_format == "hdf5" ||
                      (opt.output_format == "auto" && opt.output.size() >= 3 &&
                       opt.output.compare(opt.output.size() - 3, 3, ".h5") == 0);
    if (opt.output_format != "auto" && opt.output_format != "hdf5" && opt.output_format != "csv")
        throw std::runtime_error("unknown output format: " + opt.output_format);
    const std::string params_path = kpb::effective_parameter_path(opt);
    kpb::write_effective_parameters(params_path, opt, pass_a, freqs);
    if (opt.kp_dry_run) {
        std::cout << "format " << (hdf5 ? "hdf5" : "csv") << "\nparameters " << params_path << "\n";
        return 0;
    }

    kp_run_options ro;
    kp_default_run_options(&ro);
    ro.device = opt.kp_device;
    ro.timing = opt.timing;
    ro.precision = opt.kp_precision == "mixed" ? KP_PRECISION_MIXED : KP_PRECISION_FP64;
    if (opt.kp_schedule == "per_pixel") ro.schedule = KP_SCHEDULE_PER_PIXEL;
    else if (opt.kp_schedule == "persistent") ro.schedule = KP_SCHEDULE_PERSISTENT;
    else if (opt.kp_schedule == "graph") ro.schedule = KP_SCHEDULE_GRAPH;
    else ro.schedule = ro.precision == KP_PRECISION_MIXED ? KP_SCHEDULE_PERSISTENT : KP_SCHEDULE_PER_PIXEL;

    const int npix = opt.nx * opt.ny;
    const int chunk = kpb::effective_chunk_size(opt, freqs.size());
    const kpb::FluxScale fs = kpb::flux_scale_of(opt);
    const double jy = fs.valid ? fs.jy_per_pixel : -1.0;
    std::vector<PackedFrequency> packed(freqs.size());
    HostImage first_chunk(npix, 1);
    kp_grid* grid = nullptr;
    if (grmhd) {
        const auto t_load = std::chrono::steady_clock::now();
        if (kharma)
            check(kp_grid_load_kharma(opt.kharma_dump.c_str(), &io, opt.kharma_reverse_field, opt.kp_device, &gm,
                                      &grid),
                  "kp_grid_load_kharma");
        else
            check(kp_grid_load_iharm(opt.iharm_dump.c_str(), &io, opt.kp_device, &gm, &grid), "kp_grid_load_iharm");
        report_timing(opt, kharma ? "kharma_load_total" : "iharm_load_total", seconds_since(t_load));
    }
    struct GridGuard {
        kp_grid* g;
        ~GridGuard() {
            if (g) kp_grid_release(g);
        }
    } guard{grid};
    const auto t_transport = std::chrono::steady_clock::now();
    for (size_t c0 = 0; c0 < freqs.size(); c0 += size_t(chunk)) {
        const int nf = int(std::min(freqs.size() - c0, size_t(chunk)));
        HostImage img(npix, nf);
        kp_image_out out = img.view(npix, nf);
        // every chunk's step control runs over the whole frequency grid
        // (tools/kpolaris_model_image.cpp:3432-3446), so all chunks follow
        // one geodesic per pixel; a single chunk is the plain image
        if (grmhd) {
            check(kp_image_grmhd_step_control(&pass_a, grid, opt.radiation_substeps, freqs.data() + c0, nf,
                                              freqs.data(), int(freqs.size()), &ro, &out),
                  "kp_image_grmhd_step_control");
        } else {
            const kp_riaf_model model = kpb::to_riaf_model(opt, freqs[c0]);
            check(kp_image_riaf_step_control(&pass_a, &model, opt.radiation_substeps, freqs.data() + c0, nf,
                                             freqs.data(), int(freqs.size()), &ro, &out),
                  "kp_image_riaf_step_control");
        }
        for (int f = 0; f < nf; ++f) {
            PackedFrequency& pf = packed[c0 + size_t(f)];
            pf.frequency = freqs[c0 + size_t(f)];
            for (int k = 0; k < 4; ++k) {
                pf.inv[k].assign(size_t(npix), 0.0);
                pf.nu[k].assign(size_t(npix), 0.0);
            }
            pf.total_steps.assign(size_t(npix), 0);
            pf.p.i_inv = pf.inv[0].data();
            pf.p.q_inv = pf.inv[1].data();
            pf.p.u_inv = pf.inv[2].data();
            pf.p.v_inv = pf.inv[3].data();
            pf.p.i_nu = pf.nu[0].data();
            pf.p.q_nu = pf.nu[1].data();
            pf.p.u_nu = pf.nu[2].data();
            pf.p.v_nu = pf.nu[3].data();
            pf.p.total_steps = pf.total_steps.data();
            check(kp_pack_image(&out, f, pf.frequency, opt.evpa_0 == "N", jy, &pf.p), "kp_pack_image");
        }
        if (c0 == 0) {
            // one geodesic per pixel: the diagnostics of every chunk match
            for (int k = 0; k < 11; ++k) first_chunk.diag[k].swap(img.diag[k]);
            first_chunk.pass_a_steps.swap(img.pass_a_steps);
            first_chunk.steps.swap(img.steps);
            first_chunk.reason.swap(img.reason);
        }
    }
    report_timing(opt, "image_transport", seconds_since(t_transport));

    const auto t_output = std::chrono::steady_clock::now();
    const bool multi = freqs.size() > 1;
    if (hdf5) {
        std::vector<kpb::H5Frequency> h5f(packed.size());
        for (size_t fi = 0; fi < packed.size(); ++fi) {
            const PackedFrequency& pf = packed[fi];
            kpb::H5Frequency& f = h5f[fi];
            f.frequency = pf.frequency;
            for (int k = 0; k < 4; ++k) {
                f.inv[k] = pf.inv[k].data();
                f.nu[k] = pf.nu[k].data();
                f.sum_inv[k] = pf.p.sum_inv[k];
                f.flux_jy[k] = pf.p.flux_jy[k];
            }
        }
        kpb::H5Diagnostics dg;
        dg.reason = first_chunk.reason.data();
        dg.pass_a_steps = first_chunk.pass_a_steps.data();
        dg.steps = first_chunk.steps.data();
        dg.total_steps = packed.front().total_steps.data();
        for (int k = 0; k < 11; ++k) dg.diag[k] = first_chunk.diag[k].data();
        kpb::write_image_h5(opt.output, opt, params_path, pass_a, freqs, h5f, dg, fs, grmhd ? &gm : nullptr);
    } else {
        std::ofstream out(opt.output);
        if (!out) throw std::runtime_error("failed to open output: " + opt.output);
        out.precision(17);
        out << "# code,KPolaris-B200\n# code_abi_version," << kp_abi_version() << "\n";
        out << "# model," << opt.model << "\n# parameter_file," << opt.parameter_file << "\n";
        out << "# effective_parameter_file," << params_path << "\n";
        out << "# nx," << opt.nx << "\n# ny," << opt.ny << "\n# camera," << opt.camera << "\n";
        out << "# coordinate," << opt.coordinate << "\n# metric," << kpb::metric_name_of(opt.coordinate) << "\n";
        out << "# stokes_convention,camera_frame\n# polarization_basis,camera_screen\n";
        out << "# inner_radius," << opt.inner_radius << "\n# outer_radius," << opt.outer_radius << "\n";
        if (grmhd) {
            // write_model_metadata for GRMHDRadiationModel (:739-787)
            const double l_unit = 6.67430e-8 * gm.mbh_solar * 1.98847e33 / (2.99792458e10 * 2.99792458e10);
            for (const std::string& pre : {std::string("grmhd"), opt.model}) {
                out << "# " << pre << "_n1," << gm.n1 << "\n# " << pre << "_n2," << gm.n2 << "\n# " << pre << "_n3,"
                    << gm.n3 << "\n# " << pre << "_M_unit," << gm.M_unit << "\n# " << pre << "_mbh_solar,"
                    << gm.mbh_solar << "\n# " << pre << "_trat_small," << gm.trat_small << "\n# " << pre
                    << "_trat_large," << gm.trat_large << "\n# " << pre << "_beta_crit," << gm.beta_crit << "\n# "
                    << pre << "_sigma_cut," << gm.sigma_cut << "\n# " << pre << "_sigma_cut_high," << gm.sigma_cut_high
                    << "\n";
            }
            out << "# emission_type," << gm.emission_type << "\n# emission_fit,"
                << kpb::emission_fit_name(gm.emission_type) << "\n";
            out << "# grmhd_interpolate_derived_scalars," << gm.has_derived_scalars << "\n# grmhd_dlambda_scale,"
                << l_unit / std::max(freqs.front(), 1.0) << "\n";
        }
        const kp_riaf_model m = kpb::to_riaf_model(opt, freqs.front());
        if (!grmhd) out << "# riaf_r_min," << m.r_min << "\n# riaf_r_max," << m.r_max << "\n# riaf_nth0," << m.nth0
            << "\n# riaf_Te0," << m.Te0 << "\n# riaf_disk_h," << m.disk_h << "\n# riaf_pow_nth," << m.pow_nth
            << "\n# riaf_pow_T," << m.pow_T << "\n# riaf_ne_unit," << m.ne_unit << "\n# riaf_te_unit," << m.te_unit
            << "\n# riaf_mbh_solar," << m.mbh_solar << "\n# riaf_keplerian_factor," << m.keplerian_factor
            << "\n# riaf_infall_factor," << m.infall_factor << "\n# emission_type," << m.emission_type
            << "\n# emission_fit," << kpb::emission_fit_name(m.emission_type) << "\n";
        if (!grmhd) {
            // riaf.hpp:76-85: length unit over the frequency
            const double l_unit = 6.67430e-8 * m.mbh_solar * 1.98847e33 / (2.99792458e10 * 2.99792458e10);
            out << "# dlambda_scale," << l_unit / std::max(m.freq_cgs, 1.0) << "\n";
        }
        if (multi) out << "freq_index,frequency_hz,";
        out << "ix,iy,I_inv,Q_inv,U_inv,V_inv,I_nu,Q_nu,U_nu,V_nu,reason,pass_a_steps,pass_b_steps,total_steps,"
               "closure_x,closure_k,final_null,frame_error,det_r,overlap_r11,overlap_r12,overlap_r21,overlap_r22,"
               "basis_identity_error,basis_rotation_angle\n";
        for (size_t fi = 0; fi < packed.size(); ++fi) {
            const PackedFrequency& pf = packed[fi];
            for (int p = 0; p < npix; ++p) {
                if (multi) out << fi << ',' << pf.frequency << ',';
                out << p % opt.nx << ',' << p / opt.nx;
                for (int k = 0; k < 4; ++k) out << ',' << pf.inv[k][size_t(p)];
                for (int k = 0; k < 4; ++k) out << ',' << pf.nu[k][size_t(p)];
                out << ',' << first_chunk.reason[size_t(p)] << ',' << first_chunk.pass_a_steps[size_t(p)] << ','
                    << first_chunk.steps[size_t(p)] << ',' << pf.total_steps[size_t(p)];
                for (int k = 0; k < 11; ++k) out << ',' << first_chunk.diag[k][size_t(p)];
                out << '\n';
            }
        }
        if (!out) throw std::runtime_error("failed writing output: " + opt.output);
    }
    report_timing(opt, "image_output", seconds_since(t_output));
    report_timing(opt, "image_run_model_total", seconds_since(t_start));

    std::cout.precision(17);
    std::cout << "KPolaris-B200 model image output\nmodel " << opt.model << "\nformat " << (hdf5 ? "hdf5" : "csv")
              << "\n";
    std::cout << "output " << opt.output << "\n";
    if (!params_path.empty()) std::cout << "parameters " << params_path << "\n";
    std::cout << "pixels " << npix << "\nfrequencies " << freqs.size() << "\n";
    std::cout << "intensity_to_flux_jy_per_pixel "
              << (fs.valid ? fs.jy_per_pixel : std::numeric_limits<double>::quiet_NaN()) << "\n";
    long long sa = 0, sb = 0;
    int ma = 0, mb = 0, mt = 0;
    for (int p = 0; p < npix; ++p) {
        sa += first_chunk.pass_a_steps[size_t(p)];
        sb += first_chunk.steps[size_t(p)];
        ma = std::max(ma, int(first_chunk.pass_a_steps[size_t(p)]));
        mb = std::max(mb, int(first_chunk.steps[size_t(p)]));
        mt = std::max(mt, int(first_chunk.pass_a_steps[size_t(p)] + first_chunk.steps[size_t(p)]));
    }
    for (size_t fi = 0; fi < packed.size(); ++fi) {
        const PackedFrequency& pf = packed[fi];
        std::cout << "freq_index " << fi << "\nfrequency_hz " << pf.frequency << "\nreturned " << pf.p.returned << "\n";
        std::cout << "mean_pass_a_steps " << double(sa) / npix << "\nmean_pass_b_steps " << double(sb) / npix
                  << "\nmean_total_steps " << double(sa + sb) / npix << "\n";
        std::cout << "max_pass_a_steps " << ma << "\nmax_pass_b_steps " << mb << "\nmax_total_steps " << mt << "\n";
        const char* names[4] = {"I", "Q", "U", "V"};
        for (int k = 0; k < 4; ++k) std::cout << names[k] << "_inv " << pf.p.sum_inv[k] << "\n";
        for (int k = 0; k < 4; ++k) std::cout << "flux_" << names[k] << "_Jy " << pf.p.flux_jy[k] << "\n";
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> args;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        if (a == "--help" || a == "-h") {
            std::cout << "usage: kp_model_image --parameter_file=FILE.par [--key=value ...]\n"
                         "RIAF images and iharm / KHARMA GRMHD dumps through the KPolaris-B200 C ABI; HDF5 or CSV "
                         "output and <output>.params.\n";
            return 0;
        }
        args.push_back(a);
    }
    try {
        return run(args);
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
}
