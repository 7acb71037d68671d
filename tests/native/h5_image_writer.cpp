// Test program (test infrastructure): writes a synthetic kpolaris_image v1
// file through the image tool's HDF5 output (kpolaris_b200/host/
// kp_image_h5.hpp), from a parameter file resolved as the tool resolves it
// and image arrays given by closed forms the test recomputes:
//   inv[k][p] = (k + 1) * 1e-40 * (1 + p % 7) * (fi + 1),  nu = inv * f^3,
//   diag[d][p] = d + p * 1e-3, reason = 1 unless p % 5 == 4 (then 3),
//   pass_a_steps = 100 + p, steps = 50 + 2 p.
// Also prints lookup3 of the published test strings, one hex value a line.
//   h5_image_writer PARFILE OUT.h5
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "kp_image_h5.hpp"

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    const char* kat = "Four score and seven years ago";
    std::printf("%08x\n%08x\n%08x\n%08x\n", kph5::lookup3(nullptr, 0, 0), kph5::lookup3(nullptr, 0, 0xdeadbeefu),
                kph5::lookup3(reinterpret_cast<const uint8_t*>(kat), 30, 0),
                kph5::lookup3(reinterpret_cast<const uint8_t*>(kat), 30, 1));
    try {
        kpb::ImageOptions opt = kpb::parse_options({std::string("--parameter_file=") + argv[1]});
        kpb::finalize_options(opt);
        const std::vector<double> freqs = kpb::build_frequency_grid(opt);
        const kp_pass_a_params pass_a = kpb::to_pass_a(opt);
        const kpb::FluxScale fs = kpb::flux_scale_of(opt);
        const int npix = opt.nx * opt.ny;
        std::vector<std::vector<double>> inv(freqs.size() * 4), nu(freqs.size() * 4);
        std::vector<kpb::H5Frequency> images(freqs.size());
        for (size_t fi = 0; fi < freqs.size(); ++fi) {
            kpb::H5Frequency& im = images[fi];
            im.frequency = freqs[fi];
            for (int k = 0; k < 4; ++k) {
                auto& a = inv[fi * 4 + k];
                auto& b = nu[fi * 4 + k];
                a.resize(size_t(npix));
                b.resize(size_t(npix));
                double s = 0.0;
                for (int p = 0; p < npix; ++p) {
                    a[size_t(p)] = (k + 1) * 1e-40 * (1 + p % 7) * double(fi + 1);
                    b[size_t(p)] = a[size_t(p)] * freqs[fi] * freqs[fi] * freqs[fi];
                    s += a[size_t(p)];
                }
                im.inv[k] = a.data();
                im.nu[k] = b.data();
                im.sum_inv[k] = s;
                im.flux_jy[k] = 1.5 * (k + 1) * double(fi + 1);
            }
        }
        const size_t n = static_cast<size_t>(npix);
        std::vector<int32_t> reason(n), pa(n), st(n), tot(n);
        std::vector<std::vector<double>> diag(11, std::vector<double>(size_t(npix)));
        for (int p = 0; p < npix; ++p) {
            reason[size_t(p)] = p % 5 == 4 ? 3 : 1;
            pa[size_t(p)] = 100 + p;
            st[size_t(p)] = 50 + 2 * p;
            tot[size_t(p)] = pa[size_t(p)] + st[size_t(p)];
            for (int d = 0; d < 11; ++d) diag[size_t(d)][size_t(p)] = d + p * 1e-3;
        }
        kpb::H5Diagnostics dg;
        dg.reason = reason.data();
        dg.pass_a_steps = pa.data();
        dg.steps = st.data();
        dg.total_steps = tot.data();
        for (int d = 0; d < 11; ++d) dg.diag[d] = diag[size_t(d)].data();
        kpb::write_image_h5(argv[2], opt, "run.params", pass_a, freqs, images, dg, fs);
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
