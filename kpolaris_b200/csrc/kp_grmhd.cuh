// kp_grmhd.cuh -- GRMHD grid plasma in FMKS native coordinates, FP64: the
// trilinear gather of primitives and derived scalars, the fluid four-velocity
// and magnetic four-vector, the R-beta electron temperature, and the
// thermal-synchrotron coefficients rotated into the transported screen
// basis.  Also the per-cell derived-scalar precompute.
//
// Reference: GRMHDGridRadiationModel (src/model/grmhd_grid.hpp): cell lookup
// native_indices_from_native_coords (:271-296), ghost mapping (:309-321),
// stencils (:379-441), native_fluid_metric (:721-766), fluid_state for FMKS
// data on an FMKS metric (:883-1080), coefficients (:1091-1240), unit
// conversions (:144-161); the loaders' precompute_derived_scalars
// (src/grmhd/kharma_loader.cpp:261-362).
#pragma once

#include "kp_fmks.cuh"
#include "kp_radiation.cuh"

namespace kp {

// Primitive indices of the grid ([8][n1][n2][n3], FP32) and the derived
// scalars ([5][n1][n2][n3], FP64).
enum : int { kPrimRho = 0, kPrimU = 1, kPrimU1 = 2, kPrimB1 = 5 };
enum : int { kDerNe = 0, kDerThetae = 1, kDerB = 2, kDerSigma = 3, kDerBeta = 4, kNumDerived = 5 };

struct GrmhdSample {
    int emitting, has_chi;
    double ne, thetae, b, nu_scale, st, ct, cos2chi, sin2chi;
};

// theta(x1, x2) of the grid's FMKS map, with its first derivatives.
KP_HD void grid_theta(const GridConsts& g, double x1, double x2, double& th, double& dth1, double& dth2) {
    const FmksTheta t = fmks_theta(g.map, x1, x2);
    th = t.th;
    dth1 = t.dth1;
    dth2 = t.dth2;
}

// g_{mu nu} and g^{0 mu} of the native coordinates (native_fluid_metric).
KP_HD void grid_native_metric(const GridConsts& g, double r, double th, double dth1, double dth2,
                              double gcov[4][4], double gcon0[4]) {
    double s, c;
    sincos(th, &s, &c);
    const double s2 = s * s, a = g.map.spin, a2 = a * a;
    const double rho2 = r * r + a2 * c * c;
    const double f = 2.0 * r / rho2;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) gcov[i][j] = 0.0;
    const double g00 = -1.0 + f, g01 = f, g03 = -a * f * s2, g11 = 1.0 + f;
    const double g13 = -a * s2 * (1.0 + f), g22 = rho2, g33 = s2 * (rho2 + a2 * s2 * (1.0 + f));
    gcov[0][0] = g00;
    gcov[0][1] = gcov[1][0] = g01 * r;
    gcov[0][3] = gcov[3][0] = g03;
    gcov[1][1] = g11 * r * r + g22 * dth1 * dth1;
    gcov[1][2] = gcov[2][1] = g22 * dth1 * dth2;
    gcov[1][3] = gcov[3][1] = g13 * r;
    gcov[2][2] = g22 * dth2 * dth2;
    gcov[3][3] = g33;
    const double inv_r = 1.0 / max_val(r, kTiny);
    const double inv_dth2 = 1.0 / max_val(dth2, kTiny);
    gcon0[0] = -(1.0 + f);
    gcon0[1] = f * inv_r;
    gcon0[2] = -f * dth1 * inv_r * inv_dth2;
    gcon0[3] = 0.0;
}

// u^mu, b^mu and b.b from the primitives (U1..U3 relative to the normal
// observer, B1..B3) at a native point (fluid_state, :989-1026).
KP_HD double grid_four_vectors(const double gcov[4][4], const double gcon0[4], const double U[3], const double B[3],
                               double ucon[4], double bcon[4]) {
    double spatial = 0.0;
    for (int i = 1; i < 4; ++i)
        for (int j = 1; j < 4; ++j) spatial += gcov[i][j] * U[i - 1] * U[j - 1];
    const double vfac = sqrt(max_val(-1.0 / gcon0[0] * (1.0 + abs_val(spatial)), 0.0));
    ucon[0] = -vfac * gcon0[0];
    for (int i = 1; i < 4; ++i) ucon[i] = U[i - 1] - vfac * gcon0[i];
    double ucov[4];
    for (int mu = 0; mu < 4; ++mu) {
        double sum = 0.0;
        for (int nu = 0; nu < 4; ++nu) sum += gcov[mu][nu] * ucon[nu];
        ucov[mu] = sum;
    }
    double udotB = 0.0;
    for (int i = 1; i < 4; ++i) udotB += ucov[i] * B[i - 1];
    bcon[0] = udotB;
    for (int i = 1; i < 4; ++i) bcon[i] = (B[i - 1] + ucon[i] * udotB) / max_val(ucon[0], kTiny);
    double bsq = 0.0;
    for (int mu = 0; mu < 4; ++mu) {
        double bc = 0.0;
        for (int nu = 0; nu < 4; ++nu) bc += gcov[mu][nu] * bcon[nu];
        bsq += bcon[mu] * bc;
    }
    return max_val(abs_val(bsq), 1e-40);
}

// R-beta electron temperature unit (trat from beta, :1050-1063).
KP_HD double grid_thetae_unit(const GridConsts& g, double beta) {
    const double betasq = beta * beta / max_val(g.beta_crit * g.beta_crit, 1e-40);
    const double trat = (g.trat_large * betasq + g.trat_small) / (1.0 + betasq);
    const double mp_me = 1836.1526734400013, game = 4.0 / 3.0, gamp = 5.0 / 3.0;
    return mp_me * (game - 1.0) * (gamp - 1.0) / ((gamp - 1.0) + (game - 1.0) * trat);
}

KP_HD double grid_sigma_factor(const GridConsts& g, double sigma) {
    double above = g.sigma_cut;
    if (g.sigma_cut_high > 0.0) above = g.sigma_cut_high;
    if (sigma < g.sigma_cut) return 1.0;
    if (sigma >= above) return 0.0;
    const double dsig = max_val(above - g.sigma_cut, kTiny);
    return cos(kPi / 2.0 / dsig * (sigma - g.sigma_cut));
}

// Cell-corner stencil of a native point, or false outside the grid.
struct GridStencil {
    size_t cell[8];
    double w[8];
};

KP_HD bool grid_stencil(const GridConsts& g, double x1, double x2, double phi, GridStencil& st) {
    if (!(x1 >= g.startx1 && x1 < g.startx1 + double(g.n1) * g.dx1 && x2 >= g.startx2 &&
          x2 < g.startx2 + double(g.n2) * g.dx2))
        return false;
    const double two_pi = 6.283185307179586476925286766559005768;
    phi = phi - floor(phi / two_pi) * two_pi;
    const double ii = (x1 - g.startx1) / g.dx1 - 0.5;
    const double jj = (x2 - g.startx2) / g.dx2 - 0.5;
    const double kk = (phi - g.startx3) / g.dx3 - 0.5;
    int i0 = int(floor(ii)), j0 = int(floor(jj)), k0 = int(floor(kk));
    i0 = i0 < -1 ? -1 : (i0 >= g.n1 ? g.n1 - 1 : i0);
    j0 = j0 < -1 ? -1 : (j0 >= g.n2 ? g.n2 - 1 : j0);
    k0 = k0 < -1 ? -1 : (k0 >= g.n3 ? g.n3 - 1 : k0);
    const double di = clamp_val(ii - double(i0), 0.0, 1.0);
    const double dj = clamp_val(jj - double(j0), 0.0, 1.0);
    const double dk = clamp_val(kk - double(k0), 0.0, 1.0);
    auto cell = [&](int i, int j, int k) {
        // ghost cells: radius clamps, theta reflects across the pole with a
        // half turn in phi, phi wraps (map_ghost_index)
        if (i < 0) i = 0;
        if (i >= g.n1) i = g.n1 - 1;
        if (j < 0) {
            j = 0;
            k += g.n3 / 2;
        } else if (j >= g.n2) {
            j = g.n2 - 1;
            k += g.n3 / 2;
        }
        while (k < 0) k += g.n3;
        while (k >= g.n3) k -= g.n3;
        return (size_t(i) * size_t(g.n2) + size_t(j)) * size_t(g.n3) + size_t(k);
    };
    const double wi[2] = {1.0 - di, di}, wj[2] = {1.0 - dj, dj}, wk[2] = {1.0 - dk, dk};
    for (int n = 0; n < 8; ++n) {
        const int a = n & 1, b = (n >> 1) & 1, c2 = (n >> 2) & 1;
        st.cell[n] = cell(i0 + a, j0 + b, k0 + c2);
        st.w[n] = wi[a] * wj[b] * wk[c2];
    }
    return true;
}

// The eight primitives at a point: each corner is one 32-byte cell (two
// 16-byte loads); every field accumulates over the corners in stencil order.
KP_HD void grid_gather_prims(const GridStencil& st, const float* prims, double out[kPrimStride]) {
    for (int v = 0; v < kPrimStride; ++v) out[v] = 0.0;
    for (int n = 0; n < 8; ++n) {
        const float* c = prims + st.cell[n] * kPrimStride;
        float val[kPrimStride];
#ifdef __CUDA_ARCH__
        const float4 a = __ldg(reinterpret_cast<const float4*>(c));
        const float4 b = __ldg(reinterpret_cast<const float4*>(c) + 1);
        val[0] = a.x; val[1] = a.y; val[2] = a.z; val[3] = a.w;
        val[4] = b.x; val[5] = b.y; val[6] = b.z; val[7] = b.w;
#else
        for (int v = 0; v < kPrimStride; ++v) val[v] = c[v];
#endif
        for (int v = 0; v < kPrimStride; ++v) out[v] += st.w[n] * double(val[v]);
    }
}

// The five derived scalars at a point: each corner is one 48-byte cell
// (three 16-byte loads).
KP_HD void grid_gather_derived(const GridStencil& st, const double* derived, double out[kNumDerived]) {
    for (int v = 0; v < kNumDerived; ++v) out[v] = 0.0;
    for (int n = 0; n < 8; ++n) {
        const double* c = derived + st.cell[n] * kDerStride;
        double val[kDerStride];
#ifdef __CUDA_ARCH__
        const double2 a = __ldg(reinterpret_cast<const double2*>(c));
        const double2 b = __ldg(reinterpret_cast<const double2*>(c) + 1);
        const double2 d = __ldg(reinterpret_cast<const double2*>(c) + 2);
        val[0] = a.x; val[1] = a.y; val[2] = b.x; val[3] = b.y; val[4] = d.x; val[5] = d.y;
#else
        for (int v = 0; v < kDerStride; ++v) val[v] = c[v];
#endif
        for (int v = 0; v < kNumDerived; ++v) out[v] += st.w[n] * val[v];
    }
}

// Linear interpolation in time that keeps the endpoints and static values
// exact (interpolate_time_value, src/model/time_interpolation.hpp:27-32).
KP_HD double time_interp(double a, double b, double f) {
    if (f <= 0.0 || a == b) return a;
    if (f >= 1.0) return b;
    return (1.0 - f) * a + f * b;
}

// Plasma state at a sample point, the frequency-independent part of
// coefficients (:1091-1240 up to the thermal fit), from grid g, or with
// `up` the fluid interpolated in time between g and up at fraction f: every
// gathered primitive and derived scalar is interpolated after the trilinear
// gather, the four-vectors are formed from the interpolated primitives
// (fluid_state with time_upper, :945-962).  The grids share one geometry.
__device__ __forceinline__ GrmhdSample grmhd_sample_from(const ImageConsts& c, const Ray& s, const GridConsts& g,
                                                         const GridConsts* up, double f) {
    GrmhdSample out;
    out.emitting = 0;
    out.has_chi = 0;
    const double x1 = s.x.v[1], x2 = s.x.v[2], phi = s.x.v[3];
    const double r = exp(x1);
    double th, dth1, dth2;
    grid_theta(g, x1, x2, th, dth1, dth2);
    if (!(r >= g.r_in && r < g.r_out)) return out;
    GridStencil st;
    if (!grid_stencil(g, x1, x2, phi, st)) return out;
    double P[kPrimStride];
    grid_gather_prims(st, g.prims, P);
    if (up) {
        double Pu[kPrimStride];
        grid_gather_prims(st, up->prims, Pu);
        for (int v = 0; v < kPrimStride; ++v) P[v] = time_interp(P[v], Pu[v], f);
    }
    const double rho = P[kPrimRho];
    const double uu = P[kPrimU];
    if (!(rho > 0.0 && uu > 0.0)) return out;
    double U[3], B[3];
    for (int i = 0; i < 3; ++i) {
        U[i] = P[kPrimU1 + i];
        B[i] = P[kPrimB1 + i];
    }
    double gcov[4][4], gcon0[4];
    grid_native_metric(g, r, th, dth1, dth2, gcov, gcon0);
    double ucon[4], bcon[4];
    const double bsq = grid_four_vectors(gcov, gcon0, U, B, ucon, bcon);
    double ne, thetae, bcgs, sigma;
    if (g.has_derived) {
        double D[kNumDerived];
        grid_gather_derived(st, g.derived, D);
        if (up) {
            double Du[kNumDerived];
            grid_gather_derived(st, up->derived, Du);
            for (int v = 0; v < kNumDerived; ++v) D[v] = time_interp(D[v], Du[v], f);
        }
        ne = D[kDerNe];
        thetae = D[kDerThetae];
        bcgs = D[kDerB];
        sigma = D[kDerSigma];
    } else {
        sigma = bsq / max_val(rho, kTiny);
        const double beta = (g.gam - 1.0) * uu / (0.5 * bsq);
        ne = rho * g.rho_unit / 1.67353286206015e-24 * g.ne_factor;
        bcgs = sqrt(bsq) * g.b_unit;
        thetae = max_val(grid_thetae_unit(g, beta) * uu / max_val(rho, kTiny), 1e-3);
    }
    ne *= grid_sigma_factor(g, sigma);
    // frame quantities along the ray
    double ucov[4];
    for (int mu = 0; mu < 4; ++mu) {
        double sum = 0.0;
        for (int nu = 0; nu < 4; ++nu) sum += gcov[mu][nu] * ucon[nu];
        ucov[mu] = sum;
    }
    double uk = 0.0;
    for (int mu = 0; mu < 4; ++mu) uk += ucov[mu] * s.k.v[mu];
    const double nu_scale = max_val(abs_val(-uk), 1e-8);
    const double bnorm = max_val(sqrt(bsq), 1e-150);
    const double inv_bnorm = 1.0 / bnorm;
    double kdotb = 0.0, ub = 0.0, ue1 = 0.0, ue2 = 0.0, ke1 = 0.0, ke2 = 0.0, e1b = 0.0, e2b = 0.0;
    for (int mu = 0; mu < 4; ++mu) {
        double bcov_mu = 0.0, kcov_mu = 0.0;
        for (int n = 0; n < 4; ++n) {
            bcov_mu += gcov[mu][n] * bcon[n];
            kcov_mu += gcov[mu][n] * s.k.v[n];
        }
        kdotb += s.k.v[mu] * bcov_mu;
        ub += ucov[mu] * bcon[mu];
        ue1 += ucov[mu] * s.e1.v[mu];
        ue2 += ucov[mu] * s.e2.v[mu];
        ke1 += kcov_mu * s.e1.v[mu];
        ke2 += kcov_mu * s.e2.v[mu];
        e1b += bcov_mu * s.e1.v[mu];
        e2b += bcov_mu * s.e2.v[mu];
    }
    out.emitting = 1;
    out.ne = ne;
    out.thetae = thetae;
    out.b = bcgs;
    out.nu_scale = nu_scale;
    out.ct = clamp_val(kdotb / max_val(nu_scale * bnorm, 1e-30), -1.0, 1.0);
    out.st = max_val(sqrt(max_val(0.0, 1.0 - out.ct * out.ct)), 1e-4);
    const double ubunit = ub * inv_bnorm, kbunit = kdotb * inv_bnorm;
    double b1 = e1b * inv_bnorm, b2 = e2b * inv_bnorm;
    if (abs_val(uk) > kTiny) {
        const double minus_inv_uk = -1.0 / uk;
        const double eKb = minus_inv_uk * kbunit - ubunit;
        b1 += ue1 * ubunit - (minus_inv_uk * ke1 - ue1) * eKb;
        b2 += ue2 * ubunit - (minus_inv_uk * ke2 - ue2) * eKb;
    }
    const double bproj2 = b1 * b1 + b2 * b2;
    if (bproj2 > 1e-30) {
        out.has_chi = 1;
        out.cos2chi = (b2 * b2 - b1 * b1) / bproj2;
        out.sin2chi = -2.0 * b1 * b2 / bproj2;
    }
    return out;
}

static __device__ __noinline__ GrmhdSample grmhd_sample(const ImageConsts& c, const Ray& s) {
    return grmhd_sample_from(c, s, c.grid, nullptr, 0.0);
}

// Slow light: the snapshot pair whose times enclose t = t_obs + x^0 (binary
// search, SlowLightResidentWindows::sample_window, slow_light_driver.hpp:
// 1000-1010) and the clamped fraction (interpolation_fraction, :62-69);
// at the ends of the pair one snapshot alone (SlowLightTemporalModel::
// coefficients, :168-176).
KP_HD double series_time(const ImageConsts& c, const Ray& s) { return c.t_obs + s.x.v[0]; }

KP_HD bool series_holds(const ImageConsts& c, double t) {
    return t >= c.series_times[0] && t <= c.series_times[c.nseries - 1];
}

KP_HD int series_bracket(const ImageConsts& c, double x0, double& f) {
    const double t = c.t_obs + x0;
    int lo = 0, hi = c.nseries - 1;
    while (lo + 1 < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (t < c.series_times[mid]) hi = mid;
        else lo = mid;
    }
    const double t0 = c.series_times[lo], t1 = c.series_times[lo + 1];
    const double denom = t1 - t0;
    f = 0.0;
    if (abs_val(denom) > kTiny) f = (c.t_obs + x0 - t0) / denom;
    f = min_val(1.0, max_val(0.0, f));
    return lo;
}

static __device__ __noinline__ GrmhdSample grmhd_sample_series(const ImageConsts& c, const Ray& s) {
    double f;
    const int lo = series_bracket(c, s.x.v[0], f);
    if (f <= 0.0) return grmhd_sample_from(c, s, c.series[lo], nullptr, 0.0);
    if (f >= 1.0) return grmhd_sample_from(c, s, c.series[lo + 1], nullptr, 0.0);
    return grmhd_sample_from(c, s, c.series[lo], &c.series[lo + 1], f);
}

// Transfer coefficients at one frequency (the thermal fit and the rotation
// into the screen basis, :1175-1240).
__device__ __forceinline__ Coeffs<double> grmhd_coefficients(const ImageConsts& c, const GrmhdSample& p,
                                                              double freq) {
    Coeffs<double> o = {};
    if (!p.emitting) return o;
    ThermalIn ti = {max_val(freq * p.nu_scale, 1.0), p.ne, p.thetae, p.b, p.st, p.ct};
    const Coeffs<double> m = thermal_coefficients(ti, c);
    o.jI = m.jI;
    o.jV = m.jV;
    o.aI = m.aI;
    o.aV = m.aV;
    o.rV = m.rV;
    if (p.has_chi) {
        o.jQ = m.jQ * p.cos2chi;
        o.jU = m.jQ * p.sin2chi;
        o.aQ = m.aQ * p.cos2chi;
        o.aU = m.aQ * p.sin2chi;
        o.rQ = m.rQ * p.cos2chi;
        o.rU = m.rQ * p.sin2chi;
    }
    return o;
}

// Derived scalars of one cell (precompute_derived_scalars): n_e, Theta_e,
// B in gauss, sigma, beta from the cell-centre primitives.
KP_HD void grid_derived_cell(const GridConsts& g, int i, int j, int k, double out[kNumDerived]) {
    const size_t cell = (size_t(i) * size_t(g.n2) + size_t(j)) * size_t(g.n3) + size_t(k);
    const float* pc = g.prims + cell * kPrimStride;
    const double x1 = g.startx1 + (double(i) + 0.5) * g.dx1;
    const double x2 = g.startx2 + (double(j) + 0.5) * g.dx2;
    const double r = exp(x1);
    double th, dth1, dth2;
    grid_theta(g, x1, x2, th, dth1, dth2);
    double gcov[4][4], gcon0[4];
    grid_native_metric(g, r, th, dth1, dth2, gcov, gcon0);
    const double rho = pc[kPrimRho];
    const double uu = pc[kPrimU];
    double U[3], B[3];
    for (int n = 0; n < 3; ++n) {
        U[n] = pc[kPrimU1 + n];
        B[n] = pc[kPrimB1 + n];
    }
    double ucon[4], bcon[4];
    const double bsq = grid_four_vectors(gcov, gcon0, U, B, ucon, bcon);
    const double mp = 1.67262171e-24, me = 9.1093826e-28;
    const double beta = (g.gam - 1.0) * uu / (0.5 * bsq);
    const double sigma = bsq / max_val(rho, kTiny);
    const double betasq = beta * beta / max_val(g.beta_crit * g.beta_crit, 1e-40);
    const double trat = (g.trat_large * betasq + g.trat_small) / (1.0 + betasq);
    const double game = 4.0 / 3.0, gamp = 5.0 / 3.0;
    const double thetae_unit = (mp / me) * (game - 1.0) * (gamp - 1.0) / ((gamp - 1.0) + (game - 1.0) * trat);
    out[kDerNe] = rho * g.rho_unit / (mp + me) * g.ne_factor;
    out[kDerThetae] = max_val(thetae_unit * uu / max_val(rho, kTiny), 1e-3);
    out[kDerB] = sqrt(bsq) * g.b_unit;
    out[kDerSigma] = sigma;
    out[kDerBeta] = beta;
}

}  // namespace kp
