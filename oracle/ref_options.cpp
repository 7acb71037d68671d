// Reference-options oracle: the reference image tool's own option code
// (tools/kpolaris_model_image_options.cpp, compiled unchanged against
// oracle/shim) driven through the steps of its main() that settle an image's
// parameters (tools/kpolaris_model_image.cpp:4916-4960 for model=riaf:
// parse, canonical names, validation, camera extents, inner radius 1.05 r_+,
// outer radius 1.15 riaf_r_max).  Prints the resolved settings as
// "key=value" lines in the order and format of kp_model_image's
// kp_print_resolved, so the two front ends compare line by line.  Test
// infrastructure only.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <iostream>
#include <string>

#include "kpolaris_model_image_options.hpp"

int main(int argc, char** argv) {
    try {
        Options opt = parse_options(argc, argv);
        for (char& c : opt.model) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
        opt.camera = canonical_camera_name(opt.camera);
        opt.coordinate = canonical_coordinate_name(opt.coordinate);
        validate_options(opt);
        resolve_camera_extents(opt);
        validate_resolved_camera(opt);
        const double horizon = 1.0 + std::sqrt(std::max(0.0, 1.0 - opt.spin * opt.spin));
        if (opt.inner_radius <= 0.0) opt.inner_radius = horizon * 1.05;
        if (opt.model != "riaf") throw std::runtime_error("model other than riaf");
        if (opt.outer_radius <= 0.0) opt.outer_radius = opt.riaf_r_max * 1.15;
        std::ostream& out = std::cout;
        out.precision(17);
        out << "model=" << opt.model << "\ncamera=" << opt.camera << "\ncoordinate=" << opt.coordinate << "\n";
        out << "output=" << opt.output << "\nformat=" << opt.output_format << "\nevpa_0=" << opt.evpa_0 << "\n";
        out << "parameter_file=" << opt.parameter_file << "\nparameter_output=" << opt.parameter_output << "\n";
        out << "nx=" << opt.nx << "\nny=" << opt.ny << "\nradius=" << opt.radius << "\ninclination=" << opt.inclination
            << "\n";
        out << "fov=" << opt.fov << "\nfovy=" << opt.fovy << "\nxspan=" << opt.xspan << "\nyspan=" << opt.yspan
            << "\n";
        out << "dsource_pc=" << opt.dsource_pc << "\nfovx_dsource=" << opt.fovx_dsource
            << "\nfovy_dsource=" << opt.fovy_dsource << "\n";
        out << "image_width_x=" << opt.image_width_x << "\nimage_width_y=" << opt.image_width_y << "\n";
        out << "effective_fovx_dsource=" << opt.effective_fovx_dsource
            << "\neffective_fovy_dsource=" << opt.effective_fovy_dsource << "\n";
        out << "x_offset=" << opt.x_offset << "\ny_offset=" << opt.y_offset
            << "\nuse_pinhole_pixel_bias=" << opt.use_pinhole_pixel_bias
            << "\npinhole_pixel_bias=" << opt.pinhole_pixel_bias << "\n";
        out << "spin=" << opt.spin << "\ninner_radius=" << opt.inner_radius << "\nouter_radius=" << opt.outer_radius
            << "\n";
        out << "step=" << opt.step << "\nmax_steps=" << opt.max_steps << "\nadaptive=" << opt.adaptive
            << "\nadaptive_tolerance=" << opt.adaptive_tolerance << "\nmin_step=" << opt.min_step
            << "\nmax_step=" << opt.max_step << "\n";
        out << "max_radiation_step=" << opt.max_radiation_step << "\nmax_radiation_depth=" << opt.max_radiation_depth
            << "\nmax_absorption_depth=" << opt.max_absorption_depth
            << "\nmax_faraday_depth=" << opt.max_faraday_depth << "\n";
        out << "direct_only=" << opt.direct_only << "\nequatorial_h_over_r=" << opt.equatorial_h_over_r
            << "\nequatorial_samples=" << opt.equatorial_samples << "\nfaraday_rotation=" << opt.faraday_rotation
            << "\n";
        out << "radiation_substeps=" << opt.radiation_substeps << "\nsplit_transport=" << opt.split_transport << "\n";
        out << "closure_x_warning=" << opt.closure_x_warning << "\nclosure_k_warning=" << opt.closure_k_warning
            << "\nframe_error_warning=" << opt.frame_error_warning
            << "\nbasis_identity_warning=" << opt.basis_identity_warning << "\n";
        out << "freq=" << opt.freq << "\nfreq_list=" << opt.freq_list << "\nfreq_min=" << opt.freq_min
            << "\nfreq_max=" << opt.freq_max << "\nnfreq=" << opt.nfreq << "\nfreq_spacing=" << opt.freq_spacing
            << "\nmultifrequency_chunk_size=" << opt.multifrequency_chunk_size << "\n";
        out << "riaf_r_min=" << opt.riaf_r_min << "\nriaf_r_max=" << opt.riaf_r_max << "\nriaf_nth0=" << opt.riaf_nth0
            << "\nriaf_Te0=" << opt.riaf_Te0 << "\nriaf_disk_h=" << opt.riaf_disk_h
            << "\nriaf_pow_nth=" << opt.riaf_pow_nth << "\nriaf_pow_T=" << opt.riaf_pow_T
            << "\nriaf_ne_unit=" << opt.riaf_ne_unit << "\nriaf_te_unit=" << opt.riaf_te_unit
            << "\nriaf_mbh_solar=" << opt.riaf_mbh_solar << "\nriaf_keplerian_factor=" << opt.riaf_keplerian_factor
            << "\nriaf_infall_factor=" << opt.riaf_infall_factor << "\n";
        out << "emission_type=" << opt.emission_type << "\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
}
