// kpolaris_image_options.hpp -- the `.par` / `--key=value` front end of the
// image tool for the RIAF image path: parameter files and command-line
// overrides, the reference's key names and aliases, its derived defaults
// (field of view from xspan or from a source-plane width in microarcseconds,
// automatic inner and outer radius, frequency grid) and the effective
// parameter file that replays a run.
//
// Semantics follow the reference's image tool:
//   key normalisation, parameter files       tools/kpolaris_model_image_options.cpp:84-117, 1129-1180
//   option keys and aliases                  tools/kpolaris_model_image_options.cpp:489-1127
//   command line (files first, then every    tools/kpolaris_model_image_options.cpp:1182-1219
//     argument in order)
//   camera extents                           tools/kpolaris_model_image_options.cpp:136-186
//   validation                               tools/kpolaris_model_image_options.cpp:188-422
//   inner / outer radius defaults            tools/kpolaris_model_image.cpp:4920-4960
//   PassAParams from the options             tools/kpolaris_model_image.cpp:3942-3985
//   frequency grid                           tools/kpolaris_model_image.cpp:1186-1266
//   flux scale                               tools/kpolaris_model_image.cpp:539-595
//   effective parameter file                 tools/kpolaris_model_image.cpp:3024-3260
//
// Keys are looked up in one table (name and aliases -> setter) instead of a
// chain of comparisons.  Options of subsystems this library does not build
// (GRMHD file loaders, analysis mode, slow-light dump lists, binary RIAF,
// non-thermal distributions) are accepted so that the reference's own
// effective parameter files replay here, and rejected only when their value
// asks for the subsystem.  Keys beginning with "kp_" are this library's own:
// kp_precision (fp64 | mixed), kp_schedule (per_pixel | persistent | graph),
// kp_device, kp_print_resolved, kp_dry_run.
#pragma once

#include <cctype>
#include <cmath>
#include <fstream>
#include <functional>
#include <limits>
#include <map>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kpolaris_b200.h"

namespace kpb {

struct ImageOptions {
    std::string model = "riaf";
    std::string output = "kpolaris_image.h5";
    std::string output_format = "auto";
    std::string evpa_0 = "N";
    std::string parameter_file;
    std::string parameter_output = "auto";
    std::string camera = "pinhole";
    std::string coordinate = "cartesian_ks";
    int nx = 96;
    int ny = 96;
    double radius = 35.0;
    double inclination = 1.04719755119659774615;
    double fov = 0.08;
    double fovy = -1.0;
    double xspan = -1.0;
    double yspan = -1.0;
    double dsource_pc = -1.0;
    double fovx_dsource = -1.0;
    double fovy_dsource = -1.0;
    double image_width_x = -1.0;
    double image_width_y = -1.0;
    double effective_fovx_dsource = -1.0;
    double effective_fovy_dsource = -1.0;
    double x_offset = 0.0;
    double y_offset = 0.0;
    int use_pinhole_pixel_bias = 0;
    double pinhole_pixel_bias = -0.01;
    double spin = 0.9375;
    double inner_radius = -1.0;
    bool inner_radius_explicit = false;
    double outer_radius = -1.0;
    double step = 0.025;
    int max_steps = 4096;
    int adaptive = 1;
    int direct_only = 0;
    double equatorial_h_over_r = 0.0;
    int equatorial_samples = 8;
    int faraday_rotation = 1;
    double adaptive_tolerance = 1e-10;
    double min_step = 1e-5;
    double max_step = 1.0;
    double max_radiation_step = 1.0;
    double max_radiation_depth = 1.0;
    double max_absorption_depth = 1.0;
    double max_faraday_depth = 4.0;
    int radiation_substeps = 2;
    double closure_x_warning = 1.0;
    double closure_k_warning = 1e-2;
    double frame_error_warning = 1e-2;
    double basis_identity_warning = 1e-2;
    int split_transport = 1;
    double freq = 230.0e9;
    std::string freq_list;
    double freq_min = -1.0;
    double freq_max = -1.0;
    int nfreq = 0;
    std::string freq_spacing = "log";
    int multifrequency_chunk_size = 0;
    double riaf_r_min = 1.0;
    double riaf_r_max = 100.0;
    double riaf_nth0 = 1.0;
    double riaf_Te0 = 1.0;
    double riaf_disk_h = 0.35;
    double riaf_pow_nth = -1.1;
    double riaf_pow_T = -0.84;
    double riaf_ne_unit = 5.0e6;
    double riaf_te_unit = 1.0e11;
    double riaf_mbh_solar = 4.3e6;
    double riaf_keplerian_factor = 1.0;
    double riaf_infall_factor = 0.0;
    int emission_type = 0;
    // model=iharm: the dump and the IHARMLoadOptions the tool passes
    // (tools/kpolaris_model_image_options.hpp:190-201 defaults)
    std::string iharm_dump;
    double iharm_M_unit = 3.0e25;
    double iharm_mbh_solar = 6.2e9;
    double iharm_trat_small = 1.0;
    double iharm_trat_large = 20.0;
    double iharm_beta_crit = 1.0;
    double iharm_sigma_cut = 1.0;
    double iharm_sigma_cut_high = -1.0;
    int iharm_interpolate_derived_scalars = 1;
    // model=kharma (tools/kpolaris_model_image_options.hpp:210-227 defaults)
    std::string kharma_dump;
    double kharma_M_unit = 3.0e25;
    double kharma_mbh_solar = 6.2e9;
    double kharma_trat_small = 1.0;
    double kharma_trat_large = 20.0;
    double kharma_beta_crit = 1.0;
    double kharma_sigma_cut = 1.0;
    double kharma_sigma_cut_high = -1.0;
    int kharma_interpolate_derived_scalars = 1;
    int kharma_reverse_field = 0;
    int timing = 0;
    int repeat_images = 1;
    // requests for subsystems that are not built (checked by validate_options)
    int analysis_mode = 0;
    int slow_light = 0;
    int slow_light_time_probe = 0;
    // this library's own keys
    std::string kp_precision = "fp64";
    std::string kp_schedule = "auto";
    int kp_device = 0;
    int kp_print_resolved = 0;
    int kp_dry_run = 0;
};

inline std::string trim_copy(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
    while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
    return s.substr(a, b - a);
}

// Leading "--" (any number) dropped, '-' read as '_'; case is kept.
inline std::string normalize_key(const std::string& raw) {
    std::string key = trim_copy(raw);
    while (key.size() >= 2 && key[0] == '-' && key[1] == '-') key.erase(0, 2);
    for (char& c : key)
        if (c == '-') c = '_';
    return key;
}

inline std::string lowercase_copy(std::string v) {
    for (char& c : v) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return v;
}

inline std::string canonical_camera_name(const std::string& name) {
    if (name == "pinhole" || name == "parallel_plane") return name;
    throw std::runtime_error("unknown camera: " + name);
}

inline std::string canonical_coordinate_name(const std::string& name) {
    static const std::vector<std::pair<std::string, std::vector<std::string>>> table = {
        {"cartesian_ks", {"cartesian_ks", "cartesian-kerr-schild", "ks"}},
        {"spherical_ks", {"spherical_ks", "spherical-kerr-schild", "ks_spherical", "kerr_schild_spherical", "sks"}},
        {"mks", {"mks", "modified_ks", "modified-kerr-schild", "native_mks"}},
        {"fmks", {"fmks", "funky_modified_ks", "funky-modified-kerr-schild", "native_fmks", "mmks"}},
        {"boyer_lindquist", {"boyer_lindquist", "boyer-lindquist", "bl"}},
    };
    for (const auto& row : table)
        for (const auto& alias : row.second)
            if (name == alias) return row.first;
    throw std::runtime_error("unknown coordinate: " + name);
}

inline int coordinate_system_of(const std::string& canonical) {
    if (canonical == "boyer_lindquist") return KP_COORD_BOYER_LINDQUIST;
    if (canonical == "spherical_ks") return KP_COORD_SPHERICAL_KS;
    if (canonical == "fmks") return KP_COORD_FMKS;
    if (canonical == "mks") return KP_COORD_MKS;
    return KP_COORD_CARTESIAN_KS;
}

inline std::string metric_name_of(const std::string& canonical) {
    if (canonical == "boyer_lindquist") return "Kerr-Boyer-Lindquist";
    if (canonical == "spherical_ks") return "Kerr-Spherical-Kerr-Schild";
    if (canonical == "fmks") return "Kerr-Funky-Modified-Kerr-Schild";
    if (canonical == "mks") return "Kerr-Spherical-Kerr-Schild with native MKS fluid grid";
    return "Kerr-Cartesian-Kerr-Schild";
}

// emission_fit names (1 Pandya thermal, 2 kappa, 3 power law, 4 Dexter thermal).
inline int emission_type_from_name(const std::string& name) {
    static const std::vector<std::pair<int, std::vector<std::string>>> table = {
        {1, {"symphony", "pandya", "thermal", "symphony_pandya_thermal"}},
        {2, {"kappa", "symphony_kappa"}},
        {3, {"powerlaw", "power_law", "symphony_powerlaw", "symphony_power_law"}},
        {4, {"dexter", "dexter_thermal"}},
    };
    for (const auto& row : table)
        for (const auto& alias : row.second)
            if (name == alias) return row.first;
    throw std::runtime_error("unknown emission fit: " + name);
}

inline std::string emission_fit_name(int type) {
    switch (type) {
    case 1: return "symphony_pandya_thermal";
    case 2: return "symphony_kappa";
    case 3: return "symphony_power_law";
    case 4: return "dexter_thermal";
    default: return "unspecified";
    }
}

inline std::string parse_evpa_zero(const std::string& v) {
    if (v == "N" || v == "n") return "N";
    if (v == "W" || v == "w") return "W";
    throw std::invalid_argument("evpa_0 must be N or W");
}

namespace detail {

using Setter = std::function<void(ImageOptions&, const std::string&)>;

inline double to_real(const std::string& v) { return std::stod(v); }
inline int to_int(const std::string& v) { return std::stoi(v); }

inline Setter real_field(double ImageOptions::*f) {
    return [f](ImageOptions& o, const std::string& v) { o.*f = to_real(v); };
}
inline Setter int_field(int ImageOptions::*f) {
    return [f](ImageOptions& o, const std::string& v) { o.*f = to_int(v); };
}
inline Setter text_field(std::string ImageOptions::*f) {
    return [f](ImageOptions& o, const std::string& v) { o.*f = v; };
}
inline Setter zero_or_one(int ImageOptions::*f, const char* what) {
    return [f, what](ImageOptions& o, const std::string& v) {
        if (v != "0" && v != "1") throw std::runtime_error(std::string(what) + " must be 0 or 1");
        o.*f = to_int(v);
    };
}

struct KeyTable {
    std::map<std::string, Setter> set;
    void add(std::initializer_list<const char*> names, Setter s) {
        for (const char* n : names) set[n] = s;
    }
};

inline const KeyTable& key_table() {
    static const KeyTable table = [] {
        KeyTable t;
        using O = ImageOptions;
        const double pi = 3.141592653589793238462643383279502884;
        t.add({"parameter_file", "input", "input_file", "params", "config"}, text_field(&O::parameter_file));
        t.add({"parameter_output", "params_output", "effective_parameters", "effective_parameter_file"},
              text_field(&O::parameter_output));
        t.add({"model"}, text_field(&O::model));
        t.add({"output"}, text_field(&O::output));
        t.add({"evpa_0"}, [](O& o, const std::string& v) { o.evpa_0 = parse_evpa_zero(v); });
        t.add({"format"}, text_field(&O::output_format));
        t.add({"camera"}, text_field(&O::camera));
        t.add({"coordinate"}, text_field(&O::coordinate));
        t.add({"nx"}, int_field(&O::nx));
        t.add({"ny"}, int_field(&O::ny));
        t.add({"radius"}, real_field(&O::radius));
        t.add({"inclination_rad"}, real_field(&O::inclination));
        t.add({"inclination_deg"}, [pi](O& o, const std::string& v) { o.inclination = to_real(v) * pi / 180.0; });
        // a later field-of-view setting replaces the earlier conventions
        t.add({"fov"}, [](O& o, const std::string& v) {
            o.fov = to_real(v);
            o.fovy = o.xspan = o.yspan = o.fovx_dsource = o.fovy_dsource = -1.0;
        });
        t.add({"fovy", "fov_y"}, [](O& o, const std::string& v) {
            o.fovy = to_real(v);
            o.fovy_dsource = -1.0;
        });
        t.add({"xspan"}, [](O& o, const std::string& v) {
            o.xspan = to_real(v);
            o.fovx_dsource = -1.0;
        });
        t.add({"yspan"}, [](O& o, const std::string& v) {
            o.yspan = to_real(v);
            o.fovy_dsource = -1.0;
        });
        t.add({"dsource", "dsource_pc"}, real_field(&O::dsource_pc));
        t.add({"fovx_dsource", "fovx_muas", "fovx_uas"}, [](O& o, const std::string& v) {
            o.fovx_dsource = to_real(v);
            o.xspan = -1.0;
        });
        t.add({"fovy_dsource", "fovy_muas", "fovy_uas"}, [](O& o, const std::string& v) {
            o.fovy_dsource = to_real(v);
            o.yspan = -1.0;
        });
        t.add({"x_offset"}, real_field(&O::x_offset));
        t.add({"y_offset"}, real_field(&O::y_offset));
        t.add({"use_pinhole_pixel_bias"}, int_field(&O::use_pinhole_pixel_bias));
        t.add({"pinhole_pixel_bias"}, real_field(&O::pinhole_pixel_bias));
        t.add({"spin"}, real_field(&O::spin));
        t.add({"inner_radius"}, [](O& o, const std::string& v) {
            o.inner_radius = to_real(v);
            o.inner_radius_explicit = true;
        });
        t.add({"outer_radius"}, real_field(&O::outer_radius));
        t.add({"max_steps"}, int_field(&O::max_steps));
        t.add({"equatorial_h_over_r"}, [](O& o, const std::string& v) {
            size_t used = 0;
            o.equatorial_h_over_r = std::stod(v, &used);
            if (used != v.size()) throw std::runtime_error("invalid equatorial_h_over_r");
        });
        t.add({"equatorial_samples"}, [](O& o, const std::string& v) {
            size_t used = 0;
            o.equatorial_samples = std::stoi(v, &used);
            if (used != v.size()) throw std::runtime_error("equatorial_samples must be an integer");
        });
        t.add({"faraday_rotation"}, zero_or_one(&O::faraday_rotation, "faraday_rotation"));
        t.add({"direct_only"}, zero_or_one(&O::direct_only, "direct_only"));
        t.add({"adaptive"}, int_field(&O::adaptive));
        t.add({"adaptive_tolerance"}, real_field(&O::adaptive_tolerance));
        t.add({"min_step"}, real_field(&O::min_step));
        t.add({"max_step"}, real_field(&O::max_step));
        t.add({"max_radiation_step", "radiation_sampling_interval"}, real_field(&O::max_radiation_step));
        // one depth for both limits; a later separate value overrides it
        t.add({"max_radiation_depth", "radiation_sampling_depth"}, [](O& o, const std::string& v) {
            o.max_radiation_depth = to_real(v);
            o.max_absorption_depth = o.max_radiation_depth;
            o.max_faraday_depth = o.max_radiation_depth;
        });
        t.add({"max_absorption_depth", "absorption_sampling_depth"}, real_field(&O::max_absorption_depth));
        t.add({"max_faraday_depth", "faraday_sampling_depth"}, real_field(&O::max_faraday_depth));
        t.add({"step"}, real_field(&O::step));
        t.add({"substeps", "radiation_substeps"}, int_field(&O::radiation_substeps));
        t.add({"closure_x_warning", "warn_closure_x"}, real_field(&O::closure_x_warning));
        t.add({"closure_k_warning", "warn_closure_k"}, real_field(&O::closure_k_warning));
        t.add({"frame_error_warning", "warn_frame_error"}, real_field(&O::frame_error_warning));
        t.add({"basis_identity_warning", "warn_basis_identity"}, real_field(&O::basis_identity_warning));
        t.add({"split_transport", "split_passes", "separate_passes"}, int_field(&O::split_transport));
        t.add({"freq", "frequency_hz"}, real_field(&O::freq));
        t.add({"freq_list", "frequency_list", "frequencies"}, text_field(&O::freq_list));
        t.add({"freq_min", "frequency_min"}, real_field(&O::freq_min));
        t.add({"freq_max", "frequency_max"}, real_field(&O::freq_max));
        t.add({"nfreq", "frequency_count"}, int_field(&O::nfreq));
        t.add({"freq_spacing", "frequency_spacing"}, text_field(&O::freq_spacing));
        t.add({"multifrequency_chunk_size", "frequency_chunk_size", "freq_chunk_size"},
              int_field(&O::multifrequency_chunk_size));
        t.add({"riaf_r_min"}, real_field(&O::riaf_r_min));
        t.add({"riaf_r_max"}, real_field(&O::riaf_r_max));
        t.add({"riaf_nth0"}, real_field(&O::riaf_nth0));
        t.add({"riaf_Te0", "riaf_te0"}, real_field(&O::riaf_Te0));
        t.add({"riaf_disk_h"}, real_field(&O::riaf_disk_h));
        t.add({"riaf_pow_nth"}, real_field(&O::riaf_pow_nth));
        t.add({"riaf_pow_T", "riaf_pow_t"}, real_field(&O::riaf_pow_T));
        t.add({"riaf_ne_unit"}, real_field(&O::riaf_ne_unit));
        t.add({"riaf_te_unit"}, real_field(&O::riaf_te_unit));
        t.add({"riaf_mbh_solar"}, real_field(&O::riaf_mbh_solar));
        t.add({"riaf_keplerian_factor"}, real_field(&O::riaf_keplerian_factor));
        t.add({"riaf_infall_factor"}, real_field(&O::riaf_infall_factor));
        // GRMHD dump options (kpolaris_model_image_options.cpp:827-970): the
        // prefixed forms set one loader's value, the unprefixed forms both
        auto both = [](double O::*a, double O::*b) {
            return [a, b](O& o, const std::string& v) { o.*a = o.*b = to_real(v); };
        };
        t.add({"iharm_dump"}, text_field(&O::iharm_dump));
        t.add({"kharma_dump", "phdf"}, text_field(&O::kharma_dump));
        t.add({"dump"}, [](O& o, const std::string& v) { o.iharm_dump = o.kharma_dump = v; });
        t.add({"iharm_M_unit", "iharm_m_unit"}, real_field(&O::iharm_M_unit));
        t.add({"kharma_M_unit", "kharma_m_unit"}, real_field(&O::kharma_M_unit));
        t.add({"M_unit"}, both(&O::iharm_M_unit, &O::kharma_M_unit));
        t.add({"iharm_mbh_solar"}, real_field(&O::iharm_mbh_solar));
        t.add({"kharma_mbh_solar"}, real_field(&O::kharma_mbh_solar));
        t.add({"MBH"}, both(&O::iharm_mbh_solar, &O::kharma_mbh_solar));
        t.add({"iharm_trat_small"}, real_field(&O::iharm_trat_small));
        t.add({"kharma_trat_small"}, real_field(&O::kharma_trat_small));
        t.add({"trat_small"}, both(&O::iharm_trat_small, &O::kharma_trat_small));
        t.add({"iharm_trat_large"}, real_field(&O::iharm_trat_large));
        t.add({"kharma_trat_large"}, real_field(&O::kharma_trat_large));
        t.add({"trat_large"}, both(&O::iharm_trat_large, &O::kharma_trat_large));
        t.add({"iharm_beta_crit"}, real_field(&O::iharm_beta_crit));
        t.add({"kharma_beta_crit"}, real_field(&O::kharma_beta_crit));
        t.add({"beta_crit"}, both(&O::iharm_beta_crit, &O::kharma_beta_crit));
        t.add({"iharm_sigma_cut"}, real_field(&O::iharm_sigma_cut));
        t.add({"kharma_sigma_cut"}, real_field(&O::kharma_sigma_cut));
        t.add({"sigma_cut"}, both(&O::iharm_sigma_cut, &O::kharma_sigma_cut));
        t.add({"iharm_sigma_cut_high"}, real_field(&O::iharm_sigma_cut_high));
        t.add({"kharma_sigma_cut_high"}, real_field(&O::kharma_sigma_cut_high));
        t.add({"sigma_cut_high"}, both(&O::iharm_sigma_cut_high, &O::kharma_sigma_cut_high));
        t.add({"iharm_interpolate_derived_scalars"}, int_field(&O::iharm_interpolate_derived_scalars));
        t.add({"kharma_interpolate_derived_scalars"}, int_field(&O::kharma_interpolate_derived_scalars));
        t.add({"interpolate_derived_scalars"}, [](O& o, const std::string& v) {
            o.iharm_interpolate_derived_scalars = o.kharma_interpolate_derived_scalars = to_int(v);
        });
        t.add({"kharma_reverse_field", "reverse_field"}, int_field(&O::kharma_reverse_field));
        t.add({"emission_type"}, int_field(&O::emission_type));
        t.add({"emission_fit"}, [](O& o, const std::string& v) { o.emission_type = emission_type_from_name(v); });
        t.add({"timing", "profile"}, int_field(&O::timing));
        t.add({"repeat_images"}, int_field(&O::repeat_images));
        t.add({"analysis_mode", "analysis", "physical_diagnostics"}, int_field(&O::analysis_mode));
        t.add({"slow_light", "slowlight"}, int_field(&O::slow_light));
        t.add({"slow_light_time_probe", "slowlight_time_probe", "time_probe"}, int_field(&O::slow_light_time_probe));
        t.add({"kp_precision"}, [](O& o, const std::string& v) {
            const std::string p = lowercase_copy(trim_copy(v));
            if (p != "fp64" && p != "mixed") throw std::runtime_error("kp_precision must be fp64 or mixed");
            o.kp_precision = p;
        });
        t.add({"kp_schedule"}, [](O& o, const std::string& v) {
            const std::string s = lowercase_copy(trim_copy(v));
            if (s != "auto" && s != "per_pixel" && s != "persistent" && s != "graph")
                throw std::runtime_error("kp_schedule must be auto, per_pixel, persistent or graph");
            o.kp_schedule = s;
        });
        t.add({"kp_device"}, int_field(&O::kp_device));
        t.add({"kp_print_resolved"}, int_field(&O::kp_print_resolved));
        t.add({"kp_dry_run"}, int_field(&O::kp_dry_run));
        return t;
    }();
    return table;
}

// Options this library does not use: loader settings beyond the table's
// iharm/KHARMA entries, the other loaders, and subsystems not built here.
// Their values enter no image; the requests that would (analysis_mode,
// slow_light, slow_light_time_probe, repeat_images) are table entries above.
inline bool inert_key(const std::string& key) {
    static const char* const prefixes[] = {"iharm_", "kharma_", "athenak_", "bhac_", "hamr_", "torus_",
                                           "binary_", "slow_light_", "slowlight_", "analysis_", "formation_",
                                           "resample_", "variable_kappa", "powerlaw_", "power_law_", "dump_"};
    for (const char* p : prefixes)
        if (key.rfind(p, 0) == 0) return true;
    static const char* const exact[] = {"kappa", "nonthermal_kappa", "scalar_transport", "M_unit", "MBH",
                                        "trat_small", "trat_large", "beta_crit", "sigma_cut", "sigma_cut_high",
                                        "interpolate_derived_scalars", "prefetch", "t_obs"};
    for (const char* e : exact)
        if (key == e) return true;
    return false;
}

}  // namespace detail

inline void apply_option(ImageOptions& opt, const std::string& raw_key, const std::string& value,
                         const std::string& source) {
    const std::string key = normalize_key(raw_key);
    const auto& table = detail::key_table().set;
    const auto it = table.find(key);
    if (it == table.end()) {
        if (detail::inert_key(key)) return;
        throw std::runtime_error("unknown option '" + key + "' in " + source);
    }
    try {
        it->second(opt, value);
    } catch (const std::exception& e) {
        throw std::runtime_error("invalid value for option '" + key + "' in " + source + ": " + value + " (" +
                                 e.what() + ")");
    }
}

inline bool is_parameter_file_key(const std::string& key) {
    return key == "parameter_file" || key == "input" || key == "input_file" || key == "params" || key == "config";
}

// "key=value" or "key value" per line, '#' starts a comment.
inline void apply_parameter_text(ImageOptions& opt, std::istream& in, const std::string& name) {
    std::string line;
    int line_no = 0;
    while (std::getline(in, line)) {
        ++line_no;
        const std::string where = name + ":" + std::to_string(line_no);
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        line = trim_copy(line);
        if (line.empty()) continue;
        std::string key, value;
        const size_t eq = line.find('=');
        if (eq != std::string::npos) {
            key = trim_copy(line.substr(0, eq));
            value = trim_copy(line.substr(eq + 1));
        } else {
            std::istringstream words(line);
            std::string extra;
            words >> key >> value;
            if (words >> extra) throw std::runtime_error(where + ": expected key=value or key value");
        }
        if (key.empty()) throw std::runtime_error(where + ": empty key");
        if (value.empty()) {
            const std::string k = normalize_key(key);
            // empty partition edges select the built-in boundaries; an empty
            // parameter-file entry names no file
            if (k == "analysis_partition_edges" || is_parameter_file_key(k)) continue;
            throw std::runtime_error(where + ": empty value");
        }
        apply_option(opt, key, value, where);
    }
}

inline void apply_parameter_file(ImageOptions& opt, const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("failed to open parameter file: " + path);
    apply_parameter_text(opt, in, path);
}

// Every argument is --key=value.  Parameter files named on the command line
// are applied first, in order; then every argument, in order, overrides.
inline ImageOptions parse_options(const std::vector<std::string>& args) {
    ImageOptions opt;
    std::vector<std::string> files;
    for (const std::string& arg : args) {
        const size_t eq = arg.find('=');
        if (eq == std::string::npos || arg.rfind("--", 0) != 0)
            throw std::runtime_error("expected --key=value option: " + arg);
        if (is_parameter_file_key(normalize_key(arg.substr(0, eq)))) files.push_back(arg.substr(eq + 1));
    }
    for (const std::string& f : files) apply_parameter_file(opt, f);
    for (const std::string& arg : args) {
        const size_t eq = arg.find('=');
        apply_option(opt, arg.substr(0, eq), arg.substr(eq + 1), "command line");
    }
    return opt;
}

// The black-hole mass of the model's length unit (camera_mbh_solar /
// output_mbh_solar, kpolaris_model_image_options.cpp:126-134).
inline double model_mbh_solar(const ImageOptions& o) {
    return o.model == "iharm" ? o.iharm_mbh_solar : o.model == "kharma" ? o.kharma_mbh_solar : o.riaf_mbh_solar;
}

// The GRMHD dump models the tool images.
inline bool grmhd_model(const ImageOptions& o) { return o.model == "iharm" || o.model == "kharma"; }

inline double length_unit_cm(double mbh_solar) {
    // the tool's constants (kpolaris_model_image_options.cpp:119-124)
    return 6.6742e-8 * mbh_solar * 1.989e33 / (2.99792458e10 * 2.99792458e10);
}

inline void validate_options(const ImageOptions& o) {
    auto positive = [](double v, const char* name) {
        if (!std::isfinite(v) || !(v > 0.0)) throw std::runtime_error(std::string(name) + " must be finite and positive");
    };
    if (o.repeat_images < 1) throw std::runtime_error("repeat_images must be positive");
    if (o.repeat_images > 1) throw std::runtime_error("repeat_images > 1 is not built: run the tool once per image");
    if (o.analysis_mode) throw std::runtime_error("analysis_mode is not built in this library");
    if (o.slow_light || o.slow_light_time_probe)
        throw std::runtime_error("slow_light from dump lists is not built in this tool (see kp_image_grmhd_slow_light)");
    if (!std::isfinite(o.equatorial_h_over_r) || o.equatorial_h_over_r < 0.0 || o.equatorial_h_over_r > 1.0 ||
        (o.equatorial_h_over_r > 0.0 && o.equatorial_h_over_r < 1e-6))
        throw std::runtime_error("equatorial_h_over_r must be 0 (disabled) or in [1e-6,1]");
    if (o.equatorial_samples < 2 || o.equatorial_samples > 1024)
        throw std::runtime_error("equatorial_samples must be an integer in [2,1024]");
    if (o.faraday_rotation != 0 && o.faraday_rotation != 1) throw std::runtime_error("faraday_rotation must be 0 or 1");
    if (o.direct_only != 0 && o.direct_only != 1) throw std::runtime_error("direct_only must be 0 or 1");
    if (o.nx <= 0 || o.ny <= 0) throw std::runtime_error("nx and ny must be positive");
    if (o.nx > std::numeric_limits<int>::max() / o.ny)
        throw std::runtime_error("nx*ny exceeds the supported integer pixel count");
    positive(o.radius, "radius");
    if (!std::isfinite(o.outer_radius))
        throw std::runtime_error("outer_radius must be finite (use a non-positive value for automatic resolution)");
    if (!std::isfinite(o.inclination)) throw std::runtime_error("inclination must be finite");
    if (!std::isfinite(o.spin) || std::fabs(o.spin) > 1.0) throw std::runtime_error("spin must be finite and lie in [-1, 1]");
    positive(o.step, "step");
    if (o.max_steps <= 0) throw std::runtime_error("max_steps must be positive");
    if (o.adaptive != 0 && o.adaptive != 1) throw std::runtime_error("adaptive must be 0 or 1");
    positive(o.adaptive_tolerance, "adaptive_tolerance");
    positive(o.min_step, "min_step");
    positive(o.max_step, "max_step");
    if (o.max_step < o.min_step) throw std::runtime_error("max_step must be greater than or equal to min_step");
    if (!std::isfinite(o.max_radiation_step) || !std::isfinite(o.max_radiation_depth) ||
        !std::isfinite(o.max_absorption_depth) || !std::isfinite(o.max_faraday_depth))
        throw std::runtime_error("radiation step/depth controls must be finite");
    if (o.radiation_substeps <= 0) throw std::runtime_error("radiation_substeps must be positive");
    if (o.multifrequency_chunk_size < 0) throw std::runtime_error("multifrequency_chunk_size must be non-negative");
    if (o.output.empty()) throw std::runtime_error("output path must not be empty");
}

// Field of view: a source-plane width in microarcseconds (with dsource)
// wins; else a pinhole's xspan/yspan half-widths set the slopes; the image
// widths in M follow, and the effective source-plane widths when dsource
// is known.
inline void resolve_camera_extents(ImageOptions& o) {
    const double pc_cm = 3.085678e18;
    const double muas_per_rad = 2.06265e11;
    const bool pinhole = o.camera != "parallel_plane";
    if (o.fovx_dsource > 0.0 || o.fovy_dsource > 0.0) {
        if (o.dsource_pc <= 0.0) throw std::runtime_error("fovx_dsource/fovy_dsource require dsource in parsec");
        if (o.fovx_dsource <= 0.0) o.fovx_dsource = o.fovy_dsource;
        if (o.fovy_dsource <= 0.0) o.fovy_dsource = o.fovx_dsource;
        const double m_per_muas = o.dsource_pc * pc_cm / length_unit_cm(model_mbh_solar(o)) / muas_per_rad;
        o.image_width_x = o.fovx_dsource * m_per_muas;
        o.image_width_y = o.fovy_dsource * m_per_muas;
        o.effective_fovx_dsource = o.fovx_dsource;
        o.effective_fovy_dsource = o.fovy_dsource;
        o.fov = o.image_width_x / o.radius;
        o.fovy = o.image_width_y / o.radius;
        o.xspan = pinhole ? -1.0 : o.image_width_x / 2.0;
        o.yspan = pinhole ? -1.0 : o.image_width_y / 2.0;
        return;
    }
    if (pinhole && o.xspan > 0.0) {
        o.fov = 2.0 * o.xspan / o.radius;
        if (o.yspan > 0.0) o.fovy = 2.0 * o.yspan / o.radius;
    }
    if (o.fovy <= 0.0) o.fovy = o.fov;
    if (pinhole) {
        o.image_width_x = o.fov * o.radius;
        o.image_width_y = o.fovy * o.radius;
    } else {
        if (o.xspan > 0.0 && o.yspan <= 0.0) o.yspan = o.xspan * double(o.ny) / double(o.nx);
        o.image_width_x = o.xspan > 0.0 ? 2.0 * o.xspan : o.fov;
        o.image_width_y = o.yspan > 0.0 ? 2.0 * o.yspan : o.fovy;
    }
    if (o.dsource_pc > 0.0 && o.image_width_x > 0.0 && o.image_width_y > 0.0) {
        const double m_per_muas = o.dsource_pc * pc_cm / length_unit_cm(model_mbh_solar(o)) / muas_per_rad;
        o.effective_fovx_dsource = o.image_width_x / m_per_muas;
        o.effective_fovy_dsource = o.image_width_y / m_per_muas;
    }
}

inline void validate_resolved_camera(const ImageOptions& o) {
    auto ok = [](double v) { return std::isfinite(v) && v > 0.0; };
    if (!ok(o.fov) || !ok(o.fovy) || !ok(o.image_width_x) || !ok(o.image_width_y))
        throw std::runtime_error("resolved camera field of view must be finite and positive");
}

// The tool's order: names canonicalised, options checked, camera extents
// resolved and checked, then the radius defaults (inner: 1.05 r_+; outer
// for the RIAF model: 1.15 riaf_r_max).
inline void finalize_options(ImageOptions& o) {
    o.model = lowercase_copy(o.model);
    o.camera = canonical_camera_name(o.camera);
    o.coordinate = canonical_coordinate_name(o.coordinate);
    validate_options(o);
    resolve_camera_extents(o);
    validate_resolved_camera(o);
    if (grmhd_model(o)) {
        // the radii and the spin come from the dump (resolve_grmhd_geometry)
        if (o.coordinate != "fmks")
            throw std::runtime_error(o.model + " images are built for --coordinate=fmks (the dump's native grid)");
        if (o.camera != "pinhole") throw std::runtime_error(o.model + " images are built for the pinhole camera");
        return;
    }
    const double horizon = 1.0 + std::sqrt(std::max(0.0, 1.0 - o.spin * o.spin));
    if (o.inner_radius <= 0.0) o.inner_radius = horizon * 1.05;
    if (o.model != "riaf")
        throw std::runtime_error("model '" + o.model +
                                 "' is not built in this tool: riaf, iharm and kharma only (other GRMHD grids go "
                                 "through "
                                 "kp_grid_upload / kp_image_grmhd)");
    if (o.outer_radius <= 0.0) o.outer_radius = o.riaf_r_max * 1.15;
}

// A GRMHD model's spin and radii once its dump header is read
// (tools/kpolaris_model_image.cpp:5113-5125, safe_inner_radius :468-475):
// the dump's spin; outer radius min(r_out, 0.9 camera radius) unless set;
// inner radius the larger of the grid's r_in and 1.05 r_+, or an explicit
// request no closer than 1.05 r_+.
inline void resolve_grmhd_geometry(ImageOptions& o, const kp_grmhd_model& m) {
    o.spin = m.spin;
    if (o.outer_radius <= 0.0) o.outer_radius = std::min(m.r_out, o.radius * 0.9);
    const double horizon = 1.0 + std::sqrt(std::max(0.0, 1.0 - m.spin * m.spin));
    if (o.inner_radius_explicit && o.inner_radius > 0.0)
        o.inner_radius = std::max(o.inner_radius, horizon * 1.05);
    else
        o.inner_radius = std::max(m.r_in, horizon * 1.05);
}

// The FMKS coordinate map of a GRMHD grid in the pass-A parameters.
inline void apply_fmks_map(kp_pass_a_params& p, const kp_grmhd_model& m) {
    p.fmks_startx1 = m.startx1;
    p.fmks_hslope = m.hslope;
    p.fmks_mks_smooth = m.mks_smooth;
    p.fmks_poly_alpha = m.poly_alpha;
    p.fmks_poly_xt = m.poly_xt;
    p.fmks_poly_norm = m.poly_norm;
}

// The load options of an iharm or KHARMA run (make_iharm_load_options,
// tools/kpolaris_model_image.cpp:1734-1767, and the KHARMA block of main,
// :5130-5175); the fit defaults to Dexter.
inline kp_iharm_options to_iharm_options(const ImageOptions& o) {
    kp_iharm_options io;
    kp_default_iharm_options(&io);
    const bool k = o.model == "kharma";
    io.freq_cgs = o.freq;
    io.M_unit = k ? o.kharma_M_unit : o.iharm_M_unit;
    io.mbh_solar = k ? o.kharma_mbh_solar : o.iharm_mbh_solar;
    io.trat_small = k ? o.kharma_trat_small : o.iharm_trat_small;
    io.trat_large = k ? o.kharma_trat_large : o.iharm_trat_large;
    io.beta_crit = k ? o.kharma_beta_crit : o.iharm_beta_crit;
    io.sigma_cut = k ? o.kharma_sigma_cut : o.iharm_sigma_cut;
    io.sigma_cut_high = k ? o.kharma_sigma_cut_high : o.iharm_sigma_cut_high;
    io.emission_type = o.emission_type > 0 ? o.emission_type : KP_FIT_DEXTER;
    io.interpolate_derived_scalars =
        k ? o.kharma_interpolate_derived_scalars : o.iharm_interpolate_derived_scalars;
    return io;
}

inline std::vector<double> parse_frequency_list(const std::string& text) {
    std::string t = text;
    for (char& c : t)
        if (c == ';') c = ',';
    std::vector<double> out;
    std::stringstream ss(t);
    std::string item;
    while (std::getline(ss, item, ',')) {
        item = trim_copy(item);
        if (!item.empty()) out.push_back(std::stod(item));
    }
    if (out.empty()) throw std::runtime_error("freq_list did not contain any valid frequencies");
    for (double f : out)
        if (!(f > 0.0)) throw std::runtime_error("all frequencies must be positive");
    return out;
}

// freq_list, else freq_min..freq_max with nfreq points (log or linear),
// else freq.
inline std::vector<double> build_frequency_grid(const ImageOptions& o) {
    if (!o.freq_list.empty()) return parse_frequency_list(o.freq_list);
    if (o.nfreq > 0 || o.freq_min > 0.0 || o.freq_max > 0.0) {
        if (o.nfreq <= 0) throw std::runtime_error("freq_min/freq_max range requires nfreq > 0");
        if (!(o.freq_min > 0.0) || !(o.freq_max > 0.0)) throw std::runtime_error("freq_min and freq_max must be positive");
        if (o.nfreq == 1) return {o.freq_min};
        if (!(o.freq_max > o.freq_min))
            throw std::runtime_error("freq_max must be greater than freq_min when nfreq > 1");
        std::vector<double> f(static_cast<size_t>(o.nfreq));
        const std::string spacing = lowercase_copy(o.freq_spacing);
        const bool linear = spacing == "linear" || spacing == "lin";
        if (!linear && spacing != "log" && spacing != "logarithmic")
            throw std::runtime_error("unknown freq_spacing: " + o.freq_spacing);
        const double a = linear ? o.freq_min : std::log(o.freq_min);
        const double b = linear ? o.freq_max : std::log(o.freq_max);
        for (int i = 0; i < o.nfreq; ++i) {
            const double t = double(i) / double(o.nfreq - 1);
            f[static_cast<size_t>(i)] = linear ? a + t * (b - a) : std::exp(a + t * (b - a));
        }
        return f;
    }
    if (!(o.freq > 0.0)) throw std::runtime_error("freq must be positive");
    return {o.freq};
}

inline std::string frequency_list_string(const std::vector<double>& f) {
    std::ostringstream out;
    out.precision(17);
    for (size_t i = 0; i < f.size(); ++i) out << (i ? "," : "") << f[i];
    return out.str();
}

// Frequencies per image call: the compiled capacity, or a smaller chunk
// size when one is set.
inline int effective_chunk_size(const ImageOptions& o, size_t nfreq) {
    int cap = KP_MAX_FREQUENCIES;
    if (o.multifrequency_chunk_size > 0 && o.multifrequency_chunk_size < cap) cap = o.multifrequency_chunk_size;
    if (nfreq < size_t(cap)) cap = int(nfreq);
    return cap < 1 ? 1 : cap;
}

// The requested emission fit, Pandya thermal when none was given.
inline int effective_emission_type(const ImageOptions& o) { return o.emission_type > 0 ? o.emission_type : 1; }

inline kp_pass_a_params to_pass_a(const ImageOptions& o) {
    kp_pass_a_params p;
    kp_default_pass_a_params(&p);
    p.camera.nx = o.nx;
    p.camera.ny = o.ny;
    p.camera.radius = o.radius;
    p.camera.inclination = o.inclination;
    p.camera.fov = o.fov;
    p.camera.fov_y = o.fovy > 0.0 ? o.fovy : o.fov;
    p.camera.x_offset = o.x_offset;
    p.camera.y_offset = o.y_offset;
    const bool pinhole = o.camera == "pinhole";
    if (pinhole && o.use_pinhole_pixel_bias) p.camera.x_offset += o.pinhole_pixel_bias / double(o.nx) * o.fov;
    p.camera.xspan = pinhole ? -1.0 : o.xspan;
    p.camera.yspan = (!pinhole && o.xspan > 0.0) ? (o.yspan > 0.0 ? o.yspan : o.xspan * double(o.ny) / double(o.nx))
                                                 : -1.0;
    p.camera.model = pinhole ? KP_CAMERA_PINHOLE : KP_CAMERA_PARALLEL_PLANE;
    p.coordinate_system = coordinate_system_of(o.coordinate);
    if (p.coordinate_system != KP_COORD_CARTESIAN_KS && !pinhole)
        throw std::runtime_error("parallel_plane camera is currently defined only with cartesian_ks coordinates");
    p.mass = 1.0;
    p.spin = o.spin;
    p.inner_radius = o.inner_radius;
    p.outer_radius = o.outer_radius;
    p.step = o.step;
    p.max_steps = o.max_steps;
    p.adaptive = o.adaptive;
    p.direct_only = o.direct_only;
    p.emission_selection.equatorial_h_over_r = o.equatorial_h_over_r;
    p.emission_selection.equatorial_samples = o.equatorial_samples;
    p.emission_selection.faraday_rotation = o.faraday_rotation;
    p.adaptive_tolerance = o.adaptive_tolerance;
    p.min_step = o.min_step;
    p.max_step = o.max_step;
    p.max_radiation_step = o.max_radiation_step;
    p.max_radiation_depth = o.max_radiation_depth;
    p.max_absorption_depth = o.max_absorption_depth;
    p.max_faraday_depth = o.max_faraday_depth;
    return p;
}

inline kp_riaf_model to_riaf_model(const ImageOptions& o, double freq) {
    kp_riaf_model m;
    kp_default_riaf_model(&m);
    m.freq_cgs = freq;
    m.r_min = o.riaf_r_min;
    m.r_max = o.riaf_r_max;
    m.nth0 = o.riaf_nth0;
    m.Te0 = o.riaf_Te0;
    m.disk_h = o.riaf_disk_h;
    m.pow_nth = o.riaf_pow_nth;
    m.pow_T = o.riaf_pow_T;
    m.ne_unit = o.riaf_ne_unit;
    m.te_unit = o.riaf_te_unit;
    m.mbh_solar = o.riaf_mbh_solar;
    m.keplerian_factor = o.riaf_keplerian_factor;
    m.infall_factor = o.riaf_infall_factor;
    m.emission_type = effective_emission_type(o);
    return m;
}

// Camera grid of the output: extents, pixel pitch and units.
struct ImageGrid {
    double x_half_extent, y_half_extent, dx, dy;
    std::string units;
};

inline ImageGrid image_grid(const ImageOptions& o, const kp_pass_a_params& p) {
    const kp_camera_params& c = p.camera;
    const double xe = c.xspan > 0.0 ? 2.0 * c.xspan : c.fov;
    const double ye = c.yspan > 0.0 ? 2.0 * c.yspan
                                    : (c.xspan > 0.0 ? 2.0 * c.xspan * double(o.ny) / double(o.nx)
                                                     : (c.fov_y > 0.0 ? c.fov_y : c.fov));
    return ImageGrid{0.5 * xe, 0.5 * ye, xe / double(o.nx), ye / double(o.ny),
                     o.camera == "pinhole" ? "dimensionless_slope" : "M"};
}

struct FluxScale {
    double l_unit_cm, dsource_cm, pixel_solid_angle_sr, jy_per_pixel;
    bool valid;
};

inline FluxScale flux_scale_of(const ImageOptions& o) {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    FluxScale s{length_unit_cm(model_mbh_solar(o)), o.dsource_pc * 3.085678e18, nan, nan, false};
    if (o.dsource_pc > 0.0 && o.image_width_x > 0.0 && o.image_width_y > 0.0 && o.nx > 0 && o.ny > 0) {
        const double px = o.image_width_x * s.l_unit_cm / double(o.nx);
        const double py = o.image_width_y * s.l_unit_cm / double(o.ny);
        s.pixel_solid_angle_sr = px * py / (s.dsource_cm * s.dsource_cm);
        s.jy_per_pixel = s.pixel_solid_angle_sr / 1.0e-23;
        s.valid = std::isfinite(s.jy_per_pixel) && s.jy_per_pixel > 0.0;
    }
    return s;
}

inline std::string effective_parameter_path(const ImageOptions& o) {
    if (o.parameter_output == "none" || o.parameter_output == "off" || o.parameter_output == "0") return {};
    if (o.parameter_output.empty() || o.parameter_output == "auto") return o.output + ".params";
    return o.parameter_output;
}

// The resolved settings as "key=value" lines (doubles at 17 digits), the
// same set for every run: what kp_print_resolved prints.
inline void print_resolved(std::ostream& out, const ImageOptions& o) {
    out.precision(17);
    out << "model=" << o.model << "\ncamera=" << o.camera << "\ncoordinate=" << o.coordinate << "\n";
    out << "output=" << o.output << "\nformat=" << o.output_format << "\nevpa_0=" << o.evpa_0 << "\n";
    out << "parameter_file=" << o.parameter_file << "\nparameter_output=" << o.parameter_output << "\n";
    out << "nx=" << o.nx << "\nny=" << o.ny << "\nradius=" << o.radius << "\ninclination=" << o.inclination << "\n";
    out << "fov=" << o.fov << "\nfovy=" << o.fovy << "\nxspan=" << o.xspan << "\nyspan=" << o.yspan << "\n";
    out << "dsource_pc=" << o.dsource_pc << "\nfovx_dsource=" << o.fovx_dsource << "\nfovy_dsource=" << o.fovy_dsource
        << "\n";
    out << "image_width_x=" << o.image_width_x << "\nimage_width_y=" << o.image_width_y << "\n";
    out << "effective_fovx_dsource=" << o.effective_fovx_dsource
        << "\neffective_fovy_dsource=" << o.effective_fovy_dsource << "\n";
    out << "x_offset=" << o.x_offset << "\ny_offset=" << o.y_offset
        << "\nuse_pinhole_pixel_bias=" << o.use_pinhole_pixel_bias << "\npinhole_pixel_bias=" << o.pinhole_pixel_bias
        << "\n";
    out << "spin=" << o.spin << "\ninner_radius=" << o.inner_radius << "\nouter_radius=" << o.outer_radius << "\n";
    out << "step=" << o.step << "\nmax_steps=" << o.max_steps << "\nadaptive=" << o.adaptive
        << "\nadaptive_tolerance=" << o.adaptive_tolerance << "\nmin_step=" << o.min_step
        << "\nmax_step=" << o.max_step << "\n";
    out << "max_radiation_step=" << o.max_radiation_step << "\nmax_radiation_depth=" << o.max_radiation_depth
        << "\nmax_absorption_depth=" << o.max_absorption_depth << "\nmax_faraday_depth=" << o.max_faraday_depth
        << "\n";
    out << "direct_only=" << o.direct_only << "\nequatorial_h_over_r=" << o.equatorial_h_over_r
        << "\nequatorial_samples=" << o.equatorial_samples << "\nfaraday_rotation=" << o.faraday_rotation << "\n";
    out << "radiation_substeps=" << o.radiation_substeps << "\nsplit_transport=" << o.split_transport << "\n";
    out << "closure_x_warning=" << o.closure_x_warning << "\nclosure_k_warning=" << o.closure_k_warning
        << "\nframe_error_warning=" << o.frame_error_warning << "\nbasis_identity_warning=" << o.basis_identity_warning
        << "\n";
    out << "freq=" << o.freq << "\nfreq_list=" << o.freq_list << "\nfreq_min=" << o.freq_min
        << "\nfreq_max=" << o.freq_max << "\nnfreq=" << o.nfreq << "\nfreq_spacing=" << o.freq_spacing
        << "\nmultifrequency_chunk_size=" << o.multifrequency_chunk_size << "\n";
    out << "riaf_r_min=" << o.riaf_r_min << "\nriaf_r_max=" << o.riaf_r_max << "\nriaf_nth0=" << o.riaf_nth0
        << "\nriaf_Te0=" << o.riaf_Te0 << "\nriaf_disk_h=" << o.riaf_disk_h << "\nriaf_pow_nth=" << o.riaf_pow_nth
        << "\nriaf_pow_T=" << o.riaf_pow_T << "\nriaf_ne_unit=" << o.riaf_ne_unit << "\nriaf_te_unit="
        << o.riaf_te_unit << "\nriaf_mbh_solar=" << o.riaf_mbh_solar << "\nriaf_keplerian_factor="
        << o.riaf_keplerian_factor << "\nriaf_infall_factor=" << o.riaf_infall_factor << "\n";
    out << "emission_type=" << o.emission_type << "\n";
}

// <output>.params: the effective settings after parameter files, overrides
// and derived defaults, in a form this tool and the reference's tool both
// read back (derived quantities as comments).
inline void write_effective_parameters(const std::string& path, const ImageOptions& o, const kp_pass_a_params& p,
                                       const std::vector<double>& freqs) {
    if (path.empty()) return;
    std::ofstream out(path);
    if (!out) throw std::runtime_error("failed to open effective parameter output: " + path);
    out.precision(17);
    const ImageGrid g = image_grid(o, p);
    const FluxScale fs = flux_scale_of(o);
    out << "# KPolaris-B200 effective parameter file\n";
    out << "# Written by kp_model_image after applying parameter files, command-line overrides, and derived "
           "defaults.\n";
    out << "# code_abi_version=" << kp_abi_version() << "\n";
    if (!o.parameter_file.empty()) out << "# source_parameter_file=" << o.parameter_file << "\n";
    out << "parameter_output=" << path << "\n";
    out << "model=" << o.model << "\noutput=" << o.output << "\nformat=" << o.output_format << "\n";
    out << "evpa_0=" << o.evpa_0 << "\n";
    out << "camera=" << o.camera << "\ncoordinate=" << o.coordinate << "\n";
    out << "# derived_metric=" << metric_name_of(o.coordinate) << "\n";
    out << "nx=" << o.nx << "\nny=" << o.ny << "\nradius=" << o.radius << "\ninclination_rad=" << o.inclination
        << "\n";
    out << "fov=" << p.camera.fov << "\nfovy=" << p.camera.fov_y << "\n";
    if (p.camera.model == KP_CAMERA_PARALLEL_PLANE)
        out << "xspan=" << p.camera.xspan << "\nyspan=" << p.camera.yspan << "\n";
    if (o.dsource_pc > 0.0) out << "dsource=" << o.dsource_pc << "\n";
    if (o.effective_fovx_dsource > 0.0) out << "fovx_dsource=" << o.effective_fovx_dsource << "\n";
    if (o.effective_fovy_dsource > 0.0) out << "fovy_dsource=" << o.effective_fovy_dsource << "\n";
    out << "# derived_image_width_x_M=" << o.image_width_x << "\n# derived_image_width_y_M=" << o.image_width_y
        << "\n";
    out << "x_offset=" << o.x_offset << "\ny_offset=" << o.y_offset << "\n";
    out << "use_pinhole_pixel_bias=" << o.use_pinhole_pixel_bias << "\npinhole_pixel_bias=" << o.pinhole_pixel_bias
        << "\n";
    out << "# effective_x_offset=" << p.camera.x_offset << "\n# effective_y_offset=" << p.camera.y_offset << "\n";
    out << "# derived_grid_units=" << g.units << "\n# derived_x_half_extent=" << g.x_half_extent
        << "\n# derived_y_half_extent=" << g.y_half_extent << "\n# derived_dx=" << g.dx << "\n# derived_dy=" << g.dy
        << "\n";
    out << "# derived_l_unit_cm=" << fs.l_unit_cm << "\n# derived_dsource_cm=" << fs.dsource_cm
        << "\n# derived_pixel_solid_angle_sr=" << fs.pixel_solid_angle_sr
        << "\n# derived_intensity_to_flux_jy_per_pixel=" << fs.jy_per_pixel << "\n";
    out << "spin=" << o.spin << "\ninner_radius=" << o.inner_radius << "\nouter_radius=" << o.outer_radius << "\n";
    out << "step=" << o.step << "\nadaptive=" << o.adaptive << "\nadaptive_tolerance=" << o.adaptive_tolerance
        << "\nmin_step=" << o.min_step << "\nmax_step=" << o.max_step << "\n";
    out << "max_radiation_step=" << o.max_radiation_step << "\nmax_radiation_depth=" << o.max_radiation_depth
        << "\nmax_absorption_depth=" << o.max_absorption_depth << "\nmax_faraday_depth=" << o.max_faraday_depth
        << "\n";
    out << "closure_x_warning=" << o.closure_x_warning << "\nclosure_k_warning=" << o.closure_k_warning
        << "\nframe_error_warning=" << o.frame_error_warning << "\nbasis_identity_warning=" << o.basis_identity_warning
        << "\n";
    out << "split_transport=" << o.split_transport << "\ndirect_only=" << o.direct_only
        << "\nequatorial_h_over_r=" << o.equatorial_h_over_r << "\nequatorial_samples=" << o.equatorial_samples
        << "\nfaraday_rotation=" << o.faraday_rotation << "\n";
    out << "max_steps=" << o.max_steps << "\nsubsteps=" << o.radiation_substeps << "\nfreq=" << o.freq << "\n";
    if (!o.freq_list.empty()) out << "freq_list=" << o.freq_list << "\n";
    if (o.nfreq > 0 || o.freq_min > 0.0 || o.freq_max > 0.0)
        out << "freq_min=" << o.freq_min << "\nfreq_max=" << o.freq_max << "\nnfreq=" << o.nfreq
            << "\nfreq_spacing=" << o.freq_spacing << "\n";
    out << "multifrequency_chunk_size=" << o.multifrequency_chunk_size << "\n";
    out << "# derived_nfreq=" << freqs.size() << "\n# effective_multifrequency_chunk_size="
        << effective_chunk_size(o, freqs.size()) << "\n# derived_freq_list=" << frequency_list_string(freqs) << "\n";
    out << "# compile_KP_MAX_FREQUENCIES=" << KP_MAX_FREQUENCIES << "\n";
    if (o.model == "iharm") {
        out << "iharm_dump=" << o.iharm_dump << "\niharm_M_unit=" << o.iharm_M_unit
            << "\niharm_mbh_solar=" << o.iharm_mbh_solar << "\niharm_trat_small=" << o.iharm_trat_small
            << "\niharm_trat_large=" << o.iharm_trat_large << "\niharm_beta_crit=" << o.iharm_beta_crit
            << "\niharm_sigma_cut=" << o.iharm_sigma_cut << "\niharm_sigma_cut_high=" << o.iharm_sigma_cut_high
            << "\niharm_interpolate_derived_scalars=" << o.iharm_interpolate_derived_scalars << "\n";
    } else if (o.model == "kharma") {
        out << "kharma_dump=" << o.kharma_dump << "\nkharma_M_unit=" << o.kharma_M_unit
            << "\nkharma_mbh_solar=" << o.kharma_mbh_solar << "\nkharma_trat_small=" << o.kharma_trat_small
            << "\nkharma_trat_large=" << o.kharma_trat_large << "\nkharma_beta_crit=" << o.kharma_beta_crit
            << "\nkharma_sigma_cut=" << o.kharma_sigma_cut << "\nkharma_sigma_cut_high=" << o.kharma_sigma_cut_high
            << "\nkharma_interpolate_derived_scalars=" << o.kharma_interpolate_derived_scalars
            << "\nkharma_reverse_field=" << o.kharma_reverse_field << "\n";
    }
    if (grmhd_model(o)) {
        const int fit = o.emission_type > 0 ? o.emission_type : KP_FIT_DEXTER;
        out << "emission_type=" << fit << "\nemission_fit=" << emission_fit_name(fit) << "\n";
    } else {
        out << "riaf_r_min=" << o.riaf_r_min << "\nriaf_r_max=" << o.riaf_r_max << "\nriaf_nth0=" << o.riaf_nth0
            << "\nriaf_Te0=" << o.riaf_Te0 << "\nriaf_disk_h=" << o.riaf_disk_h << "\nriaf_pow_nth=" << o.riaf_pow_nth
            << "\nriaf_pow_T=" << o.riaf_pow_T << "\nriaf_ne_unit=" << o.riaf_ne_unit << "\nriaf_te_unit="
            << o.riaf_te_unit << "\nriaf_mbh_solar=" << o.riaf_mbh_solar << "\nriaf_keplerian_factor="
            << o.riaf_keplerian_factor << "\nriaf_infall_factor=" << o.riaf_infall_factor << "\n";
        out << "emission_type=" << effective_emission_type(o) << "\nemission_fit="
            << emission_fit_name(effective_emission_type(o)) << "\n";
    }
    out << "# kp_precision=" << o.kp_precision << "\n# kp_schedule=" << o.kp_schedule << "\n";
}

}  // namespace kpb
