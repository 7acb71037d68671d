// kp_kharma.hpp -- the KHARMA GRMHD dump reader: a Parthenon .phdf file
// (Info / Input attributes, Blocks/loc.lx123, prims.rho, prims.u,
// prims.uvec, prims.B in meshblock order) into a kp_grmhd_model and FP32
// primitives [8][n1][n2][n3], with the reference loader's checks and
// messages (read_kharma_staged_dump, initialize_kharma_staged_metadata,
// validate_kharma_staged_layout, assemble_kharma_primitives and
// read_kharma_dump_time, src/grmhd/kharma_loader.cpp:44-262, 556-823 in the
// reference).  The geometry comes from the run's parameter text (the
// Input/File attribute); fmks and mmks transforms are built (the wavefront
// engine's FMKS grid), the plain mks transform is refused.  The derived
// scalars are computed on the device by kp_grid_upload.
#pragma once

#include <cctype>
#include <cmath>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "kp_hdf5_read.hpp"
#include "kp_iharm.hpp"
#include "kpolaris_b200.h"

namespace kpb {

namespace kharma_detail {

inline std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
    while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
    return s.substr(a, b - a);
}

// `key = value` in the `<block>` section of Parthenon parameter text: the
// section runs to the next '<'; '#' starts a comment; the key must be
// followed by blank or '=' (kharma_loader.cpp:60-91).
inline bool block_value(const std::string& text, const std::string& block, const std::string& key,
                        std::string& value) {
    const std::string tag = "<" + block + ">";
    const size_t at = text.find(tag);
    if (at == std::string::npos) return false;
    const size_t begin = at + tag.size();
    size_t end = text.find('<', begin);
    if (end == std::string::npos) end = text.size();
    std::istringstream in(text.substr(begin, end - begin));
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        line = trim(line);
        if (line.empty() || line.rfind(key, 0) != 0) continue;
        if (line.size() > key.size()) {
            const char next = line[key.size()];
            if (!(std::isspace(static_cast<unsigned char>(next)) || next == '=')) continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        value = trim(line.substr(eq + 1));
        return !value.empty();
    }
    return false;
}

inline int par_int(const std::string& t, const std::string& b, const std::string& k, int def) {
    std::string v;
    return block_value(t, b, k, v) ? std::stoi(v) : def;
}

inline double par_double(const std::string& t, const std::string& b, const std::string& k, double def) {
    std::string v;
    return block_value(t, b, k, v) ? std::stod(v) : def;
}

inline std::string par_string(const std::string& t, const std::string& b, const std::string& k,
                              const std::string& def) {
    std::string v;
    return block_value(t, b, k, v) ? v : def;
}

inline size_t checked_product(size_t a, size_t b, const char* what) {
    if (a != 0 && b > std::numeric_limits<size_t>::max() / a)
        throw std::runtime_error(std::string("KHARMA ") + what + " overflows size_t");
    return a * b;
}

}  // namespace kharma_detail

// /Info Time (or time) (kharma_loader.cpp:726-749).
inline double read_kharma_dump_time(const std::string& path) {
    kph5::Reader f(path);
    if (f.exists("/Info")) {
        if (f.has_attr("/Info", "Time")) return f.attr_values<double>("/Info", "Time").at(0);
        if (f.has_attr("/Info", "time")) return f.attr_values<double>("/Info", "time").at(0);
    }
    throw std::runtime_error("KHARMA dump does not contain /Info Time attribute: " + path);
}

// `read_prims` false reads and checks the metadata only.
inline IharmDump load_kharma_dump(const std::string& path, const kp_iharm_options& opt, int reverse_field,
                                  bool read_prims = true) {
    using namespace kharma_detail;
    if (path.empty()) throw std::runtime_error("--kharma_dump is required for --model=kharma");
    IharmDump out;
    kp_grmhd_model& m = out.model;
    kp_default_grmhd_model(&m);
    try {
        kph5::Reader f(path);
        for (const char* g : {"/Info", "/Input"})
            if (!f.exists(g)) throw kph5::FormatError(std::string("group ") + g + " not found");
        const std::vector<long long> nmb_v = f.attr_values<long long>("/Info", "NumMeshBlocks");
        const std::vector<long long> mbs = f.attr_values<long long>("/Info", "MeshBlockSize");
        const long long nmb = nmb_v.empty() ? 0 : nmb_v[0];
        if (mbs.empty()) throw std::runtime_error("empty KHARMA attribute: MeshBlockSize");
        const long long imax = std::numeric_limits<int>::max();
        if (mbs.size() < 3 || nmb <= 0 || mbs[0] <= 0 || mbs[1] <= 0 || mbs[2] <= 0 || mbs[0] > imax ||
            mbs[1] > imax || mbs[2] > imax)
            throw std::runtime_error("invalid KHARMA Info NumMeshBlocks/MeshBlockSize");
        const int nx1_mb = int(mbs[0]), nx2_mb = int(mbs[1]), nx3_mb = int(mbs[2]);
        const std::string par = f.attr_string("/Input", "File");
        if (par.empty()) throw std::runtime_error("KHARMA /Input File attribute is empty");

        // initialize_kharma_staged_metadata (kharma_loader.cpp:562-661)
        m.n1 = par_int(par, "parthenon/mesh", "nx1", 0);
        m.n2 = par_int(par, "parthenon/mesh", "nx2", 0);
        m.n3 = par_int(par, "parthenon/mesh", "nx3", 0);
        if (m.n1 <= 0 || m.n2 <= 0 || m.n3 <= 0)
            throw std::runtime_error("failed to parse KHARMA mesh dimensions from /Input/File parameter text");
        m.startx1 = par_double(par, "parthenon/mesh", "x1min", 0.0);
        m.startx2 = par_double(par, "parthenon/mesh", "x2min", 0.0);
        m.startx3 = par_double(par, "parthenon/mesh", "x3min", 0.0);
        const double x1max = par_double(par, "parthenon/mesh", "x1max", 0.0);
        const double x2max = par_double(par, "parthenon/mesh", "x2max", 1.0);
        const double x3max = par_double(par, "parthenon/mesh", "x3max", 6.2831853071795864769);
        m.dx1 = (x1max - m.startx1) / double(m.n1);
        m.dx2 = (x2max - m.startx2) / double(m.n2);
        m.dx3 = (x3max - m.startx3) / double(m.n3);
        m.spin = par_double(par, "coordinates", "a", 0.0);
        m.gam = par_double(par, "GRMHD", "gamma", 1.666666666666667);
        m.r_in = par_double(par, "coordinates", "r_in", std::exp(m.startx1));
        m.r_out = par_double(par, "coordinates", "r_out", std::exp(x1max));
        m.hslope = par_double(par, "coordinates", "hslope", 1.0);
        auto finite = [](double v) { return std::isfinite(v); };
        if (!finite(m.startx1) || !finite(m.startx2) || !finite(m.startx3))
            throw std::runtime_error("KHARMA grid starts must be finite");
        if (!finite(m.dx1) || !finite(m.dx2) || !finite(m.dx3) || m.dx1 <= 0.0 || m.dx2 <= 0.0 || m.dx3 <= 0.0)
            throw std::runtime_error("KHARMA grid spacings must be finite and positive");
        if (!finite(m.spin) || std::abs(m.spin) > 1.0)
            throw std::runtime_error("KHARMA spin must be finite and lie in [-1, 1]");
        if (!finite(m.gam) || m.gam <= 1.0) throw std::runtime_error("KHARMA gamma must be finite and greater than 1");
        if (!finite(m.r_in) || !finite(m.r_out) || m.r_in <= 0.0 || m.r_out <= m.r_in)
            throw std::runtime_error("KHARMA radial bounds must be finite, positive, and increasing");
        if (!finite(m.hslope)) throw std::runtime_error("KHARMA coordinate hslope must be finite");
        std::string transform = par_string(par, "coordinates", "transform", "mks");
        for (char& c : transform) c = char(std::tolower(static_cast<unsigned char>(c)));
        if (transform.find("fmks") != std::string::npos || transform.find("mmks") != std::string::npos) {
            m.mks_smooth = par_double(par, "coordinates", "mks_smooth", 0.5);
            m.poly_xt = par_double(par, "coordinates", "poly_xt", 0.82);
            m.poly_alpha = par_double(par, "coordinates", "poly_alpha", 14.0);
            if (!finite(m.mks_smooth) || !finite(m.poly_xt) || !finite(m.poly_alpha) || m.poly_xt <= 0.0 ||
                m.poly_alpha <= -1.0)
                throw std::runtime_error(
                    "KHARMA FMKS/MMKS mapping parameters must be finite with poly_alpha > -1 and poly_xt > 0");
            const double pi = 3.141592653589793238462643383279502884;
            m.poly_norm = 0.5 * pi / (1.0 + 1.0 / (m.poly_alpha + 1.0) / std::pow(m.poly_xt, m.poly_alpha));
            if (!finite(m.poly_norm) || m.poly_norm <= 0.0)
                throw std::runtime_error("KHARMA FMKS/MMKS mapping normalization must be finite and positive");
        } else if (transform.find("mks") != std::string::npos) {
            throw std::runtime_error(
                "KHARMA mks transform is not built (the FMKS grid is; fmks and mmks dumps load)");
        } else {
            throw std::runtime_error("unsupported KHARMA coordinate transform: " + transform);
        }
        // apply_common_options (kharma_loader.cpp:201-223)
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

        for (const char* d : {"/Blocks/loc.lx123", "/prims.rho", "/prims.u", "/prims.uvec", "/prims.B"})
            if (!f.exists(d))
                throw std::runtime_error("KHARMA new-format phdf requires Blocks/loc.lx123 and prims.rho/u/uvec/B");
        const kph5::DatasetInfo loc = f.info("/Blocks/loc.lx123");
        const kph5::DatasetInfo rho = f.info("/prims.rho"), uu = f.info("/prims.u");
        const kph5::DatasetInfo uvec = f.info("/prims.uvec"), bvec = f.info("/prims.B");
        const uint64_t n = uint64_t(nmb), a = uint64_t(nx1_mb), b = uint64_t(nx2_mb), c = uint64_t(nx3_mb);
        using D = std::vector<uint64_t>;
        if (loc.dims != D{n, 3} || rho.dims != D{n, c, b, a} || uu.dims != D{n, c, b, a} ||
            uvec.dims != D{n, 3, c, b, a} || bvec.dims != D{n, 3, c, b, a})
            throw std::runtime_error("KHARMA dataset dimensions do not match the documented meshblock layout");

        // validate_kharma_staged_layout (kharma_loader.cpp:663-723)
        const size_t cells_mb = checked_product(checked_product(size_t(a), size_t(b), "meshblock cell count"),
                                                size_t(c), "meshblock cell count");
        const size_t global = checked_product(checked_product(size_t(m.n1), size_t(m.n2), "global cell count"),
                                              size_t(m.n3), "global cell count");
        if (global > size_t(std::numeric_limits<int>::max()))
            throw std::runtime_error("KHARMA global cell count exceeds the supported int index range");
        const size_t staged = checked_product(size_t(nmb), cells_mb, "staged cell count");
        if (m.n1 % nx1_mb != 0 || m.n2 % nx2_mb != 0 || m.n3 % nx3_mb != 0 || staged != global)
            throw std::runtime_error("KHARMA meshblocks must tile the declared uniform global grid exactly");
        const std::vector<long long> order = f.read<long long>(loc, "/Blocks/loc.lx123");
        const int blocks1 = m.n1 / nx1_mb, blocks2 = m.n2 / nx2_mb, blocks3 = m.n3 / nx3_mb;
        std::vector<unsigned char> occupied(size_t(nmb), 0);
        for (size_t mb = 0; mb < size_t(nmb); ++mb) {
            const long long l1 = order[mb * 3], l2 = order[mb * 3 + 1], l3 = order[mb * 3 + 2];
            if (l1 < 0 || l1 >= blocks1 || l2 < 0 || l2 >= blocks2 || l3 < 0 || l3 >= blocks3)
                throw std::runtime_error("KHARMA logical meshblock location lies outside the global grid");
            const size_t slot = (size_t(l1) * size_t(blocks2) + size_t(l2)) * size_t(blocks3) + size_t(l3);
            if (slot >= occupied.size() || occupied[slot])
                throw std::runtime_error("KHARMA logical meshblock locations contain a duplicate");
            occupied[slot] = 1;
        }
        if (!read_prims) return out;
        const std::vector<float> r = f.read<float>(rho, "/prims.rho");
        const std::vector<float> u = f.read<float>(uu, "/prims.u");
        const std::vector<float> uv = f.read<float>(uvec, "/prims.uvec");
        const std::vector<float> bv = f.read<float>(bvec, "/prims.B");
        auto finite_all = [](const std::vector<float>& v, const char* name) {
            for (float x : v)
                if (!std::isfinite(x))
                    throw std::runtime_error(std::string("KHARMA dataset contains nonfinite primitive values: ") +
                                             name);
        };
        finite_all(r, "/prims.rho");
        finite_all(u, "/prims.u");
        finite_all(uv, "/prims.uvec");
        finite_all(bv, "/prims.B");
        // assemble_kharma_primitives (kharma_loader.cpp:226-259): meshblock
        // cell (kb, jb, ib) at logical location (lx1, lx2, lx3) -> global
        // (i, j, k) = (lx1 nx1 + ib, lx2 nx2 + jb, lx3 nx3 + kb)
        const size_t ncell = global;
        out.prims.assign(8 * ncell, 0.0f);
        const float sign = reverse_field ? -1.0f : 1.0f;
        for (size_t mb = 0; mb < size_t(nmb); ++mb) {
            const size_t l1 = size_t(order[mb * 3]), l2 = size_t(order[mb * 3 + 1]), l3 = size_t(order[mb * 3 + 2]);
            for (size_t local = 0; local < cells_mb; ++local) {
                const size_t ib = local % size_t(nx1_mb);
                const size_t jb = (local / size_t(nx1_mb)) % size_t(nx2_mb);
                const size_t kb = local / (size_t(nx1_mb) * size_t(nx2_mb));
                const size_t i = l1 * size_t(nx1_mb) + ib, j = l2 * size_t(nx2_mb) + jb, k = l3 * size_t(nx3_mb) + kb;
                const size_t cell = (i * size_t(m.n2) + j) * size_t(m.n3) + k;
                const size_t s = mb * cells_mb + local;
                const size_t vb = mb * 3 * cells_mb + local;
                out.prims[0 * ncell + cell] = r[s];
                out.prims[1 * ncell + cell] = u[s];
                out.prims[2 * ncell + cell] = uv[vb];
                out.prims[3 * ncell + cell] = uv[vb + cells_mb];
                out.prims[4 * ncell + cell] = uv[vb + 2 * cells_mb];
                out.prims[5 * ncell + cell] = sign * bv[vb];
                out.prims[6 * ncell + cell] = sign * bv[vb + cells_mb];
                out.prims[7 * ncell + cell] = sign * bv[vb + 2 * cells_mb];
            }
        }
    } catch (const kph5::FormatError& e) {
        throw std::runtime_error("Failed to read KHARMA dump '" + path + "': " + e.what());
    }
    return out;
}

}  // namespace kpb
