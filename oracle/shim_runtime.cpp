// Runtime check of the C++ host shim (kpolaris_b200/host/
// kpolaris_reference_shim.hpp) as a KPolaris translation unit would use it:
// compiled against the reference's own headers (unchanged, with oracle/shim),
// it calls the shim's run_riaf_image and run_riaf_analysis_image -- which run
// on the GPU through the C ABI -- and the reference's own per-pixel functions
// on the CPU for the same image, and compares them field by field.  Test
// infrastructure: built by `make -C oracle ref` into oracle/_ref/, run by
// tests/test_gpu_host_shim.py.  Prints one line per check and exits non-zero
// if any check failed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "geodesic/pass_b.hpp"
#include "geometry/kerr_schild_cartesian.hpp"
#include "image/analysis_driver.hpp"
#include "image/result.hpp"
#include "model/riaf.hpp"

#include "kpolaris_b200/host/kpolaris_reference_shim.hpp"

namespace {

using Real = double;

int g_fail = 0;

void check(bool ok, const char* what, double got, double want) {
    std::printf("%s %s got=%.17g want=%.17g\n", ok ? "ok" : "FAIL", what, got, want);
    if (!ok) g_fail = 1;
}

// max |a - b| over the arrays, against `rel` of max |b|
void close(const char* what, const std::vector<Real>& a, const std::vector<Real>& b, double rel) {
    double scale = 0.0, diff = 0.0;
    for (size_t i = 0; i < b.size(); ++i) {
        scale = std::max(scale, std::fabs(b[i]));
        if (!(std::isnan(a[i]) && std::isnan(b[i]))) diff = std::max(diff, std::fabs(a[i] - b[i]));
    }
    check(a.size() == b.size() && diff <= rel * std::max(scale, 1e-300), what, diff, rel * scale);
}

void equal(const char* what, const std::vector<int>& a, const std::vector<int>& b) {
    size_t bad = a.size() == b.size() ? 0 : 1;
    for (size_t i = 0; !bad && i < b.size(); ++i) bad += a[i] != b[i];
    check(bad == 0, what, double(bad), 0.0);
}

}  // namespace

int main() {
    // config-2 controls on a 12 x 10 pinhole image (RIAF, Cartesian Kerr-Schild)
    kpolaris::PassAParams<Real> pa;
    pa.camera.nx = 12;
    pa.camera.ny = 10;
    pa.camera.radius = 1000.0;
    pa.camera.inclination = 17.0 * 3.141592653589793238462643383279502884 / 180.0;
    pa.camera.fov = 2.0 * 80.0 / 1000.0;
    pa.camera.fov_y = pa.camera.fov;
    pa.coordinate_system = kpolaris::CoordinateSystem::CartesianKS;
    pa.mass = 1.0;
    pa.spin = 0.9375;
    pa.inner_radius = (1.0 + std::sqrt(1.0 - pa.spin * pa.spin)) * 1.05;
    pa.outer_radius = 115.0;
    pa.step = 0.025;
    pa.adaptive = 1;
    pa.max_steps = 400000;
    pa.adaptive_tolerance = 1e-8;
    pa.min_step = 1e-10;
    pa.max_step = 2.0;
    pa.max_radiation_step = 2.0;
    pa.max_radiation_depth = 1.0;
    pa.max_absorption_depth = 1.0;
    pa.max_faraday_depth = 4.0;
    kpolaris::RIAFAnalyticRadiationModel<Real> model;
    model.freq_cgs = 230e9;
    model.mbh_solar = 6.5e9;
    model.ne_unit = 4e6;
    model.te_unit = 1.5e11;
    model.disk_h = 0.3;
    const int npix = pa.camera.nx * pa.camera.ny;
    const kpolaris::KerrSchildInMetric<Real> metric(pa.mass, pa.spin);

    // imaging path
    const ImageHostData gpu = kpolaris_b200::run_riaf_image<ImageHostData>(pa, model, 1, 0, 1);
    std::vector<Real> ri(npix), rq(npix), rv(npix);
    std::vector<int> rreason(npix), rsteps(npix), rpa(npix);
    for (int p = 0; p < npix; ++p) {
        const auto r = kpolaris::trace_pass_b_segment_model_pixel_metric(p, pa, model, 1, metric);
        ri[p] = r.observed_stokes.I;
        rq[p] = r.observed_stokes.Q;
        rv[p] = r.observed_stokes.V;
        rreason[p] = static_cast<int>(r.reason);
        rsteps[p] = r.steps;
        rpa[p] = r.pass_a.steps;
    }
    equal("image reason", gpu.reason, rreason);
    equal("image steps", gpu.steps, rsteps);
    equal("image pass_a_steps", gpu.pass_a_steps, rpa);
    close("image I", gpu.image_i, ri, 1e-9);
    close("image Q", gpu.image_q, rq, 1e-6);
    close("image V", gpu.image_v, rv, 1e-6);

    // analysis path (field mapping: every block the shim fills, against the
    // reference's per-pixel analysis function)
    kpolaris::AnalysisConfig<Real> cfg;
    cfg.radial_bins = 10;
    cfg.radial_min = 2.0;
    cfg.radial_max = 110.0;
    cfg.formation_fraction = 0.8;
    const ImageHostData an = kpolaris_b200::run_riaf_analysis_image<ImageHostData>(pa, cfg, model, 1, 0, 1);
    check(an.has_analysis == 1 && an.analysis_radial_bins == 10, "analysis metadata", an.analysis_radial_bins, 10);
    std::vector<Real> path(npix), weight(npix), radius(npix), winding(npix), fmed(npix), radial_i(size_t(10) * npix);
    std::vector<int> subs(npix), region(npix), areason(npix);
    for (int p = 0; p < npix; ++p) {
        const auto r = kpolaris::trace_pass_b_segment_model_analysis_pixel_metric(p, pa, cfg, model, 1, metric);
        path[p] = r.analysis.radiating_path_length;
        weight[p] = r.analysis.emission_weight;
        radius[p] = r.analysis.emission_weighted_radius;
        winding[p] = r.analysis.photon_ring_winding_estimate;
        fmed[p] = r.analysis.intensity_formation_radius_median;
        subs[p] = r.analysis.radiation_substeps;
        region[p] = r.analysis.dominant_emission_region;
        areason[p] = static_cast<int>(r.transport.reason);
        for (int b = 0; b < 10; ++b) radial_i[size_t(b) * npix + p] = r.observer_radial_stokes[b].I;
    }
    equal("analysis reason", an.reason, areason);
    equal("analysis radiation_substeps", an.radiation_substeps, subs);
    equal("analysis dominant_emission_region", an.dominant_emission_region, region);
    close("analysis radiating_path_length", an.radiating_path_length, path, 1e-6);
    close("analysis emission_weight", an.emission_weight, weight, 1e-6);
    close("analysis emission_weighted_radius", an.emission_weighted_radius, radius, 1e-6);
    close("analysis photon_ring_winding_estimate", an.photon_ring_winding_estimate, winding, 1e-6);
    close("analysis intensity_formation_radius_median", an.intensity_formation_radius_median, fmed, 1e-9);
    close("analysis radial_stokes_i_contribution", an.radial_stokes_i_contribution, radial_i, 1e-6);
    const double e0 = std::exp(std::log(2.0)), e10 = std::exp(std::log(110.0));
    check(std::fabs(an.analysis_radial_bin_edges.front() - e0) <= 1e-12 &&
              std::fabs(an.analysis_radial_bin_edges.back() - e10) <= 1e-9,
          "analysis bin edges", an.analysis_radial_bin_edges.back(), e10);

    // response channels through the same signature: a density response on
    // four radial bins, against the reference's own accumulation into a
    // zeroed view of the driver's layout (analysis_driver.hpp:729-730)
    kpolaris::AnalysisConfig<Real> rcfg = cfg;
    auto& rc = rcfg.response;
    rc.parameter = kpolaris::PlasmaParameter::density_scale;
    rc.partition = kpolaris::SourcePartition::radial;
    rc.bins = 4;
    rc.edge_count = 5;
    for (int k = 0; k <= 4; ++k) rc.edges[k] = std::exp(std::log(2.0) + Real(k) / 4 * std::log(110.0 / 2.0));
    const ImageHostData rs = kpolaris_b200::run_riaf_analysis_image<ImageHostData>(pa, rcfg, model, 1, 0, 1);
    const size_t nresp = size_t(4) * size_t(rc.channels()) * size_t(npix);
    std::vector<Real> want(nresp, 0.0);
    struct View {
        Real* q;
        Real& operator()(size_t i) const { return q[i]; }
    } view{want.data()};
    for (int p = 0; p < npix; ++p)
        (void)kpolaris::trace_pass_b_segment_model_analysis_pixel_metric(p, pa, rcfg, model, 1, metric, view);
    check(rs.response_data.size() == nresp, "response channel count", double(rs.response_data.size()),
          double(nresp));
    // the emission channels (4 bins) and the derivative and rerun channels
    std::vector<Real> g_emit(rs.response_data.begin(), rs.response_data.begin() + size_t(16) * npix);
    std::vector<Real> w_emit(want.begin(), want.begin() + size_t(16) * npix);
    close("response emission channels", g_emit, w_emit, 1e-6);
    close("response all channels", rs.response_data, want, 1e-5);
    return g_fail;
}
