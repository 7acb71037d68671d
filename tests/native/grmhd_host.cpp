// Host build of the GRMHD/FMKS device code (kpolaris_b200/csrc) as a shared
// library, so the CPU tests can compare each piece with the reference's own
// templates point by point: the FMKS transport RHS, the FMKS pinhole camera
// ray, the per-cell derived-scalar precompute, and the grid plasma sample +
// transfer coefficients at a transport state.  Arrays use the layouts of the
// C ABI (prims [8][n1][n2][n3] FP32, derived [5][n1][n2][n3] FP64, transport
// states x[4] k[4] e1[4] e2[4]).
#include <cmath>
#include <cstring>
#include <vector>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __noinline__
#include "kp_scene.cuh"
#include "kp_grmhd_setup.h"

namespace {

// the library stores grids cell-major; these turn the C-ABI layouts into it
std::vector<float> prim_cells(const kp_grmhd_model* m, const float* prims) {
    const size_t ncell = size_t(m->n1) * size_t(m->n2) * size_t(m->n3);
    std::vector<float> cells(ncell * kp::kPrimStride);
    for (size_t p = 0; p < ncell; ++p)
        for (int f = 0; f < 8; ++f) cells[p * kp::kPrimStride + size_t(f)] = prims[size_t(f) * ncell + p];
    return cells;
}

std::vector<double> derived_cells(const kp_grmhd_model* m, const double* derived) {
    const size_t ncell = size_t(m->n1) * size_t(m->n2) * size_t(m->n3);
    std::vector<double> cells(ncell * kp::kDerStride, 0.0);
    for (size_t p = 0; p < ncell; ++p)
        for (int v = 0; v < kp::kNumDerived; ++v) cells[p * kp::kDerStride + size_t(v)] = derived[size_t(v) * ncell + p];
    return cells;
}

kp::Ray ray_of(const double* s) {
    kp::Ray r;
    for (int m = 0; m < 4; ++m) {
        r.x.v[m] = s[m];
        r.k.v[m] = s[4 + m];
        r.e1.v[m] = s[8 + m];
        r.e2.v[m] = s[12 + m];
    }
    return r;
}

void store(const kp::Ray& r, double* s) {
    for (int m = 0; m < 4; ++m) {
        s[m] = r.x.v[m];
        s[4 + m] = r.k.v[m];
        s[8 + m] = r.e1.v[m];
        s[12 + m] = r.e2.v[m];
    }
}

kp::FmksParams fmks_of(const kp_pass_a_params* p) {
    return kp::FmksParams{p->mass, p->spin, p->fmks_startx1, p->fmks_hslope, p->fmks_mks_smooth,
                          p->fmks_poly_alpha, p->fmks_poly_xt, p->fmks_poly_norm};
}

}  // namespace

extern "C" {

// The far phase's change of chart (kp_chart.cuh) and the two metrics' dot
// products, for the round-trip and invariance checks.
void h_fmks_to_cks(const kp_pass_a_params* p, const double* s16, double* o16) {
    store(kp::fmks_to_cks(fmks_of(p), p->spin, ray_of(s16)), o16);
}

void h_cks_to_fmks(const kp_pass_a_params* p, const double* s16, double x3_ref, double* o16) {
    store(kp::cks_to_fmks(fmks_of(p), p->spin, ray_of(s16), x3_ref), o16);
}

double h_cks_record_radius(double spin, const double* x4) {
    kp::D4 x{{x4[0], x4[1], x4[2], x4[3]}};
    return kp::cks_record_radius(spin, x);
}

double h_dot_fmks(const kp_pass_a_params* p, const double* x4, const double* u4, const double* v4) {
    kp::D4 x{{x4[0], x4[1], x4[2], x4[3]}}, u{{u4[0], u4[1], u4[2], u4[3]}}, v{{v4[0], v4[1], v4[2], v4[3]}};
    double g[4][4];
    kp::fmks_gcov(fmks_of(p), x, g);
    return kp::dot_gm(g, u, v);
}

double h_dot_cks(double spin, const double* x4, const double* u4, const double* v4) {
    kp::D4 x{{x4[0], x4[1], x4[2], x4[3]}}, u{{u4[0], u4[1], u4[2], u4[3]}}, v{{v4[0], v4[1], v4[2], v4[3]}};
    return kp::ks_dot_at(kp::ks_point(1.0, spin, x), u, v);
}

void h_fmks_rhs(const kp_pass_a_params* p, const double* s16, double* d16) {
    store(kp::fmks_rhs(fmks_of(p), ray_of(s16)), d16);
}

void h_fmks_rhs_factored(const kp_pass_a_params* p, const double* s16, double* d16) {
    store(kp::fmks_rhs_factored(fmks_of(p), ray_of(s16)), d16);
}

void h_camera_ray_fmks(const kp_pass_a_params* p, int pixel, double* s16) {
    kp_grmhd_model m;
    std::memset(&m, 0, sizeof(m));
    const kp::ImageConsts c = kp::image_consts_fmks(p, m, kp::GridConsts{}, nullptr, 1, 0);
    kp::CameraFrame f;
    kp::fmks_camera_frame(c.fmks, p->camera.radius, p->camera.inclination, f.x, f.e0, f.e1, f.e2, f.e3);
    store(kp::fmks_camera_ray(c, f, pixel), s16);
}

void h_grmhd_derived(const kp_grmhd_model* m, const float* prims, double* out) {
    const std::vector<float> pc = prim_cells(m, prims);
    const kp::GridConsts g = kp::grid_consts_of(*m, pc.data(), nullptr);
    const size_t ncell = size_t(m->n1) * size_t(m->n2) * size_t(m->n3);
    for (int i = 0; i < m->n1; ++i)
        for (int j = 0; j < m->n2; ++j)
            for (int k = 0; k < m->n3; ++k) {
                double v[kp::kNumDerived];
                kp::grid_derived_cell(g, i, j, k, v);
                const size_t cell = (size_t(i) * size_t(m->n2) + size_t(j)) * size_t(m->n3) + size_t(k);
                for (int q = 0; q < kp::kNumDerived; ++q) out[size_t(q) * ncell + cell] = v[q];
            }
}

void h_grmhd_coefficients(const kp_pass_a_params* p, const kp_grmhd_model* m, const float* prims,
                          const double* derived, const double* s16, double freq, double* out11) {
    const std::vector<float> pc = prim_cells(m, prims);
    const std::vector<double> dc = derived ? derived_cells(m, derived) : std::vector<double>();
    const kp::GridConsts g = kp::grid_consts_of(*m, pc.data(), derived ? dc.data() : nullptr);
    const kp::ImageConsts c = kp::image_consts_fmks(p, *m, g, &freq, 1, 0);
    const kp::GrmhdSample smp = kp::grmhd_sample(c, ray_of(s16));
    const kp::Coeffs<double> o = kp::grmhd_coefficients(c, smp, freq);
    const double v[11] = {o.jI, o.jQ, o.jU, o.jV, o.aI, o.aQ, o.aU, o.aV, o.rQ, o.rU, o.rV};
    std::memcpy(out11, v, sizeof(v));
}

}  // extern "C"
