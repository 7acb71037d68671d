// Compiles the C++ host shim (kpolaris_b200/host/kpolaris_reference_shim.hpp)
// against the reference's own parameter, model and result types and
// instantiates every entry point, the way a maintainer's translation unit in
// the reference's build would.  Linked against the library, it runs no GPU
// work: main only checks that each instantiation exists.
#include "geodesic/pass_a_core.hpp"
#include "image/analysis_driver.hpp"
#include "image/result.hpp"
#include "model/grmhd.hpp"
#include "model/riaf.hpp"

#include "kpolaris_b200/host/kpolaris_reference_shim.hpp"

using PassA = kpolaris::PassAParams<double>;
using Riaf = kpolaris::RIAFAnalyticRadiationModel<double>;
using Grmhd = kpolaris::GRMHDGridRadiationModel<double>;

template ImageHostData kpolaris_b200::run_riaf_image<ImageHostData, PassA, Riaf>(const PassA&, Riaf, int, int, int);
template ImageHostData kpolaris_b200::run_riaf_analysis_image<ImageHostData, PassA,
                                                               kpolaris::AnalysisConfig<double>, Riaf>(
    const PassA&, const kpolaris::AnalysisConfig<double>&, Riaf, int, int, int);
template ImageHostData kpolaris_b200::run_riaf_multifrequency_image<ImageHostData, PassA, Riaf>(
    const PassA&, Riaf, int, const std::vector<double>&, const std::vector<double>&, int, int);
template ImageHostData kpolaris_b200::run_grmhd_image<ImageHostData, PassA, Grmhd>(const PassA&, Grmhd, int, int, int);
template ImageHostData kpolaris_b200::run_grmhd_multifrequency_image<ImageHostData, PassA, Grmhd, double>(
    const PassA&, Grmhd, int, const std::vector<double>&, const std::vector<double>&, int);
template ImageHostData kpolaris_b200::run_slow_light_image<ImageHostData, PassA, Grmhd, double>(
    const PassA&, const std::vector<Grmhd>&, const std::vector<double>&, double, const std::vector<double>&);

int main() {
    const kp_pass_a_params p = kpolaris_b200::to_c(PassA{});
    const kp_grmhd_model m = kpolaris_b200::to_c_grmhd(Grmhd{});
    return (p.camera.nx > 0 && m.emission_type == 4) ? 0 : 1;
}
