// kp_chart.cuh -- the change of chart between the FMKS coordinates of the
// GRMHD scene and Cartesian Kerr-Schild, for the mixed policy's far phase:
// beyond the radiating sphere a GRMHD ray carries no plasma, so the far
// kernel integrates it in CKS with the FP32 stage chains of the RIAF scene
// and converts at the phase boundary.  Records always hold FMKS states.
//
//   FMKS (x0, x1, x2, x3) -> spherical KS (t, r, theta, phi):
//       t = x0, r = exp(x1), theta = theta(x1, x2) (kerr_fmks.hpp:296-348), phi = x3
//   spherical KS -> Cartesian KS (x + i y = (r + i a) e^{i phi} sin theta):
//       x = sin(theta) (r cos phi - a sin phi), y = sin(theta) (r sin phi + a cos phi),
//       z = r cos(theta)
// Vectors go through the Jacobian of the two maps; the way back solves the
// 3x3 spatial block, finds x2 by bisection of theta(x1, x2) and unwraps phi
// against the ray's FMKS azimuth from before the far phase.
#pragma once

#include "kp_fmks.cuh"
#include "kp_geometry.cuh"

namespace kp {

// d(x, y, z) / d(x1, x2, x3) at an FMKS point.
struct ChartJacobian {
    double m[3][3];
};

KP_HD ChartJacobian fmks_cks_jacobian(double spin, double r, double th, double dth1, double dth2, double phi) {
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(phi, &sp, &cp);
    const double ra = r * cp - spin * sp;  // x / sin(theta)
    const double rb = r * sp + spin * cp;  // y / sin(theta)
    // d/dr, d/dtheta, d/dphi of (x, y, z)
    const double dr[3] = {st * cp, st * sp, ct};
    const double dt[3] = {ct * ra, ct * rb, -r * st};
    const double dp[3] = {-st * rb, st * ra, 0.0};
    ChartJacobian J;
    for (int i = 0; i < 3; ++i) {
        J.m[i][0] = r * dr[i] + dth1 * dt[i];  // d/dx1 = r d/dr + dth1 d/dtheta
        J.m[i][1] = dth2 * dt[i];              // d/dx2 = dth2 d/dtheta
        J.m[i][2] = dp[i];                     // d/dx3 = d/dphi
    }
    return J;
}

KP_HD D4 chart_push(const ChartJacobian& J, const D4& v) {
    D4 o;
    o.v[0] = v.v[0];
    for (int i = 0; i < 3; ++i) o.v[i + 1] = J.m[i][0] * v.v[1] + J.m[i][1] * v.v[2] + J.m[i][2] * v.v[3];
    return o;
}

// The inverse of chart_push: Cramer's rule on the spatial block.
KP_HD D4 chart_pull(const ChartJacobian& J, const D4& v) {
    const double(&a)[3][3] = J.m;
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    const double inv = 1.0 / det;
    const double b0 = v.v[1], b1 = v.v[2], b2 = v.v[3];
    D4 o;
    o.v[0] = v.v[0];
    o.v[1] = (b0 * c00 + b1 * (a[0][2] * a[2][1] - a[0][1] * a[2][2]) + b2 * (a[0][1] * a[1][2] - a[0][2] * a[1][1])) * inv;
    o.v[2] = (b0 * c01 + b1 * (a[0][0] * a[2][2] - a[0][2] * a[2][0]) + b2 * (a[0][2] * a[1][0] - a[0][0] * a[1][2])) * inv;
    o.v[3] = (b0 * c02 + b1 * (a[0][1] * a[2][0] - a[0][0] * a[2][1]) + b2 * (a[0][0] * a[1][1] - a[0][1] * a[1][0])) * inv;
    return o;
}

KP_HD Ray fmks_to_cks(const FmksParams& m, double spin, const Ray& s) {
    const FmksTheta t = fmks_theta(m, s.x.v[1], s.x.v[2]);
    const double phi = s.x.v[3];
    double st, ct, sp, cp;
    sincos(t.th, &st, &ct);
    sincos(phi, &sp, &cp);
    Ray o;
    o.x.v[0] = s.x.v[0];
    o.x.v[1] = st * (t.r * cp - spin * sp);
    o.x.v[2] = st * (t.r * sp + spin * cp);
    o.x.v[3] = t.r * ct;
    const ChartJacobian J = fmks_cks_jacobian(spin, t.r, t.th, t.dth1, t.dth2, phi);
    o.k = chart_push(J, s.k);
    o.e1 = chart_push(J, s.e1);
    o.e2 = chart_push(J, s.e2);
    return o;
}

// The radial coordinate of a CKS point as the FMKS record of it will hold
// it: exp(log r).  A far kernel that decides phases with this value agrees
// bit for bit with a near kernel reading exp(x1) from the record it writes.
KP_HD double cks_record_radius(double spin, const D4& X) { return exp(log(ks_radius(spin, X))); }

KP_HD Ray cks_to_fmks(const FmksParams& m, double spin, const Ray& s, double x3_ref) {
    const double x = s.x.v[1], y = s.x.v[2], z = s.x.v[3];
    const double r = ks_radius(spin, s.x);
    const double rho = sqrt(x * x + y * y);
    // sin(theta) = rho / sqrt(r^2 + a^2), cos(theta) = z / r: atan2 keeps
    // theta accurate near the poles
    const double th = atan2(rho / sqrt(r * r + spin * spin), z / r);
    // azimuth from x + i y = (r + i a) e^{i phi} sin(theta), unwrapped
    // against the FMKS azimuth the ray entered with
    const double phi0 = atan2(r * y - spin * x, r * x + spin * y);
    const double two_pi = 6.283185307179586476925286766559005768;
    const double dphi = remainder(phi0 - x3_ref, two_pi);
    const double x1 = log(r);
    Ray o;
    o.x.v[0] = s.x.v[0];
    o.x.v[1] = x1;
    o.x.v[2] = fmks_x2_of(m, x1, th);
    o.x.v[3] = x3_ref + dphi;
    const FmksTheta t = fmks_theta(m, o.x.v[1], o.x.v[2]);
    const ChartJacobian J = fmks_cks_jacobian(spin, t.r, t.th, t.dth1, t.dth2, o.x.v[3]);
    o.k = chart_pull(J, s.k);
    o.e1 = chart_pull(J, s.e1);
    o.e2 = chart_pull(J, s.e2);
    return o;
}

}  // namespace kp
