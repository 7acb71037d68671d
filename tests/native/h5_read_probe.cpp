// Test program (test infrastructure): reads datasets through
// kpolaris_b200/host/kp_hdf5_read.hpp.
//   h5_read_probe FILE OUTDIR PATH...
// For each PATH prints "exists 0|1" and, for a dataset, "rank d0 d1 ..." and
// writes its values converted to float64 to OUTDIR/<i>.f64 (and to int64,
// OUTDIR/<i>.i64).  A reader error prints "error: <message>" and exits 1.
#include <cstdint>
#include <cstdio>
#include <exception>
#include <string>
#include <vector>

#include "kp_hdf5_read.hpp"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    try {
        kph5::Reader f(argv[1]);
        for (int i = 3; i < argc; ++i) {
            const std::string path = argv[i];
            const bool ex = f.exists(path);
            std::printf("exists %d\n", ex ? 1 : 0);
            if (!ex) continue;
            const kph5::DatasetInfo d = f.info(path);
            std::printf("rank %zu", d.dims.size());
            for (uint64_t n : d.dims) std::printf(" %llu", static_cast<unsigned long long>(n));
            std::printf("\n");
            const std::vector<double> v = f.read<double>(d, path);
            const std::vector<int64_t> w = f.read<int64_t>(d, path);
            const std::string base = std::string(argv[2]) + "/" + std::to_string(i - 3);
            std::FILE* o = std::fopen((base + ".f64").c_str(), "wb");
            std::fwrite(v.data(), sizeof(double), v.size(), o);
            std::fclose(o);
            o = std::fopen((base + ".i64").c_str(), "wb");
            std::fwrite(w.data(), sizeof(int64_t), w.size(), o);
            std::fclose(o);
        }
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 1;
    }
    return 0;
}
