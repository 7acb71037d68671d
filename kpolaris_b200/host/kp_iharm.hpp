// kp_iharm.hpp -- the iharm GRMHD dump reader: header, FMKS/MMKS coordinate
// map and the /prims array of an iharm HDF5 dump into a kp_grmhd_model and
// FP32 primitives [8][n1][n2][n3], with the reference loader's checks and
// messages (load_iharm_model_from_hdf5 and read_iharm_dump_time,
// src/grmhd/iharm_loader.cpp:240-370 in the reference).  The file is read by
// kp_hdf5_read.hpp; the derived scalars the reference precomputes after the
// read (:402-520) are computed on the device by kp_grid_upload.
#pragma once

#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "kp_hdf5_read.hpp"
#include "kpolaris_b200.h"

namespace kpb {

struct IharmDump {
    kp_grmhd_model model;
    std::vector<float> prims;  // [8][n1][n2][n3]
};

namespace iharm_detail {

template <class T>
T scalar_value(kph5::Reader& f, const std::string& path) {
    if (!f.exists(path)) throw std::runtime_error("HDF5 object not found: " + path);
    return f.scalar<T>(path);
}

}  // namespace iharm_detail

// /t, else /header/t (iharm_loader.cpp:240-252).
inline double read_iharm_dump_time(const std::string& path) {
    if (path.empty()) throw std::runtime_error("empty iharm dump path");
    kph5::Reader f(path);
    if (f.exists("/t")) return f.scalar<double>("/t");
    if (f.exists("/header/t")) return f.scalar<double>("/header/t");
    throw std::runtime_error("iharm dump has no /t or /header/t time dataset: " + path);
}

// `read_prims` false reads and checks the header only (model filled, prims
// empty).
inline IharmDump load_iharm_dump(const std::string& path, const kp_iharm_options& opt, bool read_prims = true) {
    using iharm_detail::scalar_value;
    if (path.empty()) throw std::runtime_error("--iharm_dump is required for --model=iharm");
    kph5::Reader f(path);
    IharmDump out;
    kp_grmhd_model& m = out.model;
    kp_default_grmhd_model(&m);
    m.n1 = scalar_value<int>(f, "/header/n1");
    m.n2 = scalar_value<int>(f, "/header/n2");
    m.n3 = scalar_value<int>(f, "/header/n3");
    m.spin = scalar_value<double>(f, "/header/a");
    m.gam = f.exists("/header/gam") ? scalar_value<double>(f, "/header/gam") : scalar_value<double>(f, "/header/gamma");
    m.startx1 = scalar_value<double>(f, "/header/geom/startx1");
    m.startx2 = scalar_value<double>(f, "/header/geom/startx2");
    m.startx3 = scalar_value<double>(f, "/header/geom/startx3");
    m.dx1 = scalar_value<double>(f, "/header/geom/dx1");
    m.dx2 = scalar_value<double>(f, "/header/geom/dx2");
    m.dx3 = scalar_value<double>(f, "/header/geom/dx3");
    auto finite = [](double v) { return std::isfinite(v); };
    if (m.n1 <= 0 || m.n2 <= 0 || m.n3 <= 0) throw std::runtime_error("iharm header dimensions must be positive");
    if (!finite(m.spin) || std::abs(m.spin) > 1.0)
        throw std::runtime_error("iharm header spin must be finite and lie in [-1, 1]");
    if (!finite(m.gam) || m.gam <= 1.0)
        throw std::runtime_error("iharm header gamma must be finite and greater than 1");
    if (!finite(m.startx1) || !finite(m.startx2) || !finite(m.startx3))
        throw std::runtime_error("iharm grid starts must be finite");
    if (!finite(m.dx1) || !finite(m.dx2) || !finite(m.dx3) || m.dx1 <= 0.0 || m.dx2 <= 0.0 || m.dx3 <= 0.0)
        throw std::runtime_error("iharm grid spacings must be finite and positive");
    const std::string geom = f.exists("/header/geom/fmks/hslope") ? "/header/geom/fmks" : "/header/geom/mmks";
    m.hslope = scalar_value<double>(f, geom + "/hslope");
    m.mks_smooth = scalar_value<double>(f, geom + "/mks_smooth");
    m.poly_alpha = scalar_value<double>(f, geom + "/poly_alpha");
    m.poly_xt = scalar_value<double>(f, geom + "/poly_xt");
    m.r_in = scalar_value<double>(f, geom + "/r_in");
    m.r_out = scalar_value<double>(f, geom + "/r_out");
    if (!finite(m.hslope) || !finite(m.mks_smooth) || !finite(m.poly_alpha) || !finite(m.poly_xt) ||
        m.poly_alpha <= -1.0 || m.poly_xt <= 0.0)
        throw std::runtime_error(
            "iharm FMKS/MMKS mapping parameters must be finite with poly_alpha > -1 and poly_xt > 0");
    if (!finite(m.r_in) || !finite(m.r_out) || m.r_in <= 0.0 || m.r_out <= m.r_in)
        throw std::runtime_error("iharm radial bounds must be finite, positive, and increasing");
    const double pi = 3.141592653589793238462643383279502884;
    m.poly_norm = 0.5 * pi / (1.0 + 1.0 / (m.poly_alpha + 1.0) / std::pow(m.poly_xt, m.poly_alpha));
    if (!finite(m.poly_norm) || m.poly_norm <= 0.0)
        throw std::runtime_error("iharm FMKS/MMKS mapping normalization must be finite and positive");

    m.freq_cgs = opt.freq_cgs;
    m.M_unit = opt.M_unit;
    m.mbh_solar = opt.mbh_solar;
    m.trat_small = opt.trat_small;
    m.trat_large = opt.trat_large;
    m.beta_crit = opt.beta_crit;
    m.sigma_cut = opt.sigma_cut;
    m.sigma_cut_high = opt.sigma_cut_high;
    m.emission_type = opt.emission_type;
    m.has_derived_scalars = opt.interpolate_derived_scalars;

    if (!f.exists("/prims")) throw std::runtime_error("HDF5 object not found: /prims");
    const kph5::DatasetInfo d = f.info("/prims");
    if (d.dims.size() != 4) throw std::runtime_error("iharm /prims dataset must be rank 4");
    if (d.dims[0] != uint64_t(m.n1) || d.dims[1] != uint64_t(m.n2) || d.dims[2] != uint64_t(m.n3) || d.dims[3] < 8)
        throw std::runtime_error("iharm /prims dimensions do not match header or have fewer than 8 primitives");
    const uint64_t cells = d.dims[0] * d.dims[1] * d.dims[2];
    if (cells > uint64_t(std::numeric_limits<int>::max()))
        throw std::runtime_error("iharm grid cell count exceeds the supported int index range");
    if (!read_prims) return out;
    const size_t nprim = size_t(d.dims[3]);
    const std::vector<float> raw = f.read<float>(d, "/prims");
    const size_t ncell = size_t(cells);
    for (size_t c = 0; c < ncell; ++c)
        for (size_t v = 0; v < 8; ++v)
            if (!std::isfinite(raw[c * nprim + v]))
                throw std::runtime_error("iharm /prims first eight primitive fields must be finite");
    // file order [n1][n2][n3][nprim] -> [8][n1][n2][n3]
    out.prims.resize(8 * ncell);
    for (size_t c = 0; c < ncell; ++c)
        for (size_t v = 0; v < 8; ++v) out.prims[v * ncell + c] = raw[c * nprim + v];
    return out;
}

}  // namespace kpb
