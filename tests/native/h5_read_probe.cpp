// Test program (test infrastructure): reads datasets through
// kpolaris_b200/host/kp_hdf5_read.hpp.
//   h5_read_probe FILE OUTDIR PATH...
// For each PATH prints "exists 0|1" and, for a dataset, "rank d0 d1 ..." and
// writes its values converted to float64 to OUTDIR/<i>.f64 (and to int64,
// OUTDIR/<i>.i64).  PATH "@object@name" names an attribute: "exists 0|1",
// then "text" and OUTDIR/<i>.txt for a string, or "rank ..." and the value
// files for numbers.  A reader error prints "error: <message>" and exits 1.
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
            const std::string base = std::string(argv[2]) + "/" + std::to_string(i - 3);
            if (!path.empty() && path[0] == '@') {
                const size_t at = path.find('@', 1);
                const std::string obj = path.substr(1, at - 1), name = path.substr(at + 1);
                const bool ex = f.has_attr(obj, name);
                std::printf("exists %d\n", ex ? 1 : 0);
                if (!ex) continue;
                const kph5::Reader::AttrValue a = f.attr(obj, name);
                if (a.type.type == kph5::ElemType::String || a.type.type == kph5::ElemType::VarString) {
                    std::printf("text\n");
                    std::FILE* o = std::fopen((base + ".txt").c_str(), "wb");
                    std::fwrite(a.text.data(), 1, a.text.size(), o);
                    std::fclose(o);
                    continue;
                }
                std::printf("rank %zu", a.dims.size());
                for (uint64_t n : a.dims) std::printf(" %llu", static_cast<unsigned long long>(n));
                std::printf("\n");
                const std::vector<double> v = f.attr_values<double>(obj, name);
                const std::vector<int64_t> w = f.attr_values<int64_t>(obj, name);
                std::FILE* o = std::fopen((base + ".f64").c_str(), "wb");
                std::fwrite(v.data(), sizeof(double), v.size(), o);
                std::fclose(o);
                o = std::fopen((base + ".i64").c_str(), "wb");
                std::fwrite(w.data(), sizeof(int64_t), w.size(), o);
                std::fclose(o);
                continue;
            }
            const bool ex = f.exists(path);
            std::printf("exists %d\n", ex ? 1 : 0);
            if (!ex) continue;
            const kph5::DatasetInfo d = f.info(path);
            std::printf("rank %zu", d.dims.size());
            for (uint64_t n : d.dims) std::printf(" %llu", static_cast<unsigned long long>(n));
            std::printf("\n");
            const std::vector<double> v = f.read<double>(d, path);
            const std::vector<int64_t> w = f.read<int64_t>(d, path);
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
