// kp_geometry_f32.cuh -- FP32 evaluation of the Kerr-Schild transport
// right-hand side for the mixed-precision policy (same algebra as ks_rhs in
// kp_geometry.cuh; inputs and outputs stay FP64 Rays).
#pragma once

#include "kp_geometry.cuh"

namespace kp {

KP_HD Ray ks_rhs_f32(double mass_d, double spin_d, const Ray& s) {
    const float mass = float(mass_d), a = float(spin_d);
    const float x = float(s.x.v[1]), y = float(s.x.v[2]), z = float(s.x.v[3]);
    const float a2 = a * a;
    const float radius2 = x * x + y * y + z * z;
    const float sqsum = radius2 - a2;
    const float discr = sqrtf(sqsum * sqsum + 4.0f * a2 * z * z);
    const float r2 = 0.5f * (sqsum + discr);
    const float r = sqrtf(fmaxf(r2, 1e-30f));
    const float denom = r2 * r2 + a2 * z * z;
    const float inv_denom = 1.0f / denom;
    const float amp = 2.0f * mass * r2 * r * inv_denom;
    const float amp_r = -2.0f * mass * r2 * (r2 * r2 - 3.0f * a2 * z * z) * (inv_denom * inv_denom);
    const float r2pa2 = r2 + a2;
    const float inv_r2pa2 = 1.0f / r2pa2;
    const float inv_r = 1.0f / r;
    const float inv_r2 = inv_r * inv_r;
    float l[4];
    l[0] = 1.0f;
    const float px = r * x + a * y;
    const float py = r * y - a * x;
    l[1] = px * inv_r2pa2;
    l[2] = py * inv_r2pa2;
    l[3] = z * inv_r;
    const float inv_r2pa2_2 = inv_r2pa2 * inv_r2pa2;
    const float inv_discr = 1.0f / discr;
    const float inv_2r = 0.5f * inv_r;
    const float dr1 = (x + sqsum * x * inv_discr) * inv_2r;
    const float dr2 = (y + sqsum * y * inv_discr) * inv_2r;
    const float dr3 = (z + (sqsum * z + 2.0f * a2 * z) * inv_discr) * inv_2r;
    float damp[4];
    damp[0] = 0.0f;
    damp[1] = amp_r * dr1;
    damp[2] = amp_r * dr2;
    damp[3] = 6.0f * mass * r2 * dr3 * inv_denom - amp * inv_denom * (4.0f * r * r2 * dr3 + 2.0f * a2 * z);
    float dl[4][4];
    dl[1][1] = ((r + x * dr1) * r2pa2 - 2.0f * r * px * dr1) * inv_r2pa2_2;
    dl[2][1] = ((-a + y * dr1) * r2pa2 - 2.0f * r * py * dr1) * inv_r2pa2_2;
    dl[3][1] = -z * inv_r2 * dr1;
    dl[1][2] = ((a + x * dr2) * r2pa2 - 2.0f * r * px * dr2) * inv_r2pa2_2;
    dl[2][2] = ((r + y * dr2) * r2pa2 - 2.0f * r * py * dr2) * inv_r2pa2_2;
    dl[3][2] = -z * inv_r2 * dr2;
    dl[1][3] = (x * dr3 * r2pa2 - 2.0f * r * px * dr3) * inv_r2pa2_2;
    dl[2][3] = (y * dr3 * r2pa2 - 2.0f * r * py * dr3) * inv_r2pa2_2;
    dl[3][3] = (r - z * dr3) * inv_r2;
    float kk[4];
    for (int i = 0; i < 4; ++i) kk[i] = float(s.k.v[i]);
    const float lq = kk[0] + l[1] * kk[1] + l[2] * kk[2] + l[3] * kk[3];
    float dlq[4];
    for (int al = 1; al < 4; ++al) dlq[al] = dl[1][al] * kk[1] + dl[2][al] * kk[2] + dl[3][al] * kk[3];
    Ray d;
    d.x = s.k;
    // contraction Gamma(k, p) for p = k, e1, e2
    for (int which = 0; which < 3; ++which) {
        float p[4];
        const D4& src = which == 0 ? s.k : (which == 1 ? s.e1 : s.e2);
        for (int i = 0; i < 4; ++i) p[i] = float(src.v[i]);
        const float lp = p[0] + l[1] * p[1] + l[2] * p[2] + l[3] * p[3];
        float dlp[4];
        for (int al = 1; al < 4; ++al) dlp[al] = dl[1][al] * p[1] + dl[2][al] * p[2] + dl[3][al] * p[3];
        float t[4];
        for (int nu = 0; nu < 4; ++nu) {
            float term = 0.0f;
            for (int al = 1; al < 4; ++al) {
                const float dlnu = nu == 0 ? 0.0f : dl[nu][al];
                // contract(q = k, p): p^a row(q) + q^a row(p)
                const float row_p = damp[al] * l[nu] * lp + amp * (dlnu * lp + l[nu] * dlp[al]);
                const float row_q = damp[al] * l[nu] * lq + amp * (dlnu * lq + l[nu] * dlq[al]);
                term += kk[al] * row_p + p[al] * row_q;
            }
            if (nu != 0) term -= damp[nu] * lq * lp + amp * (dlq[nu] * lp + lq * dlp[nu]);
            t[nu] = term;
        }
        const float lt = -t[0] + l[1] * t[1] + l[2] * t[2] + l[3] * t[3];
        D4& dst = which == 0 ? d.k : (which == 1 ? d.e1 : d.e2);
        dst.v[0] = -double(0.5f * (-t[0] + amp * lt));
        for (int mu = 1; mu < 4; ++mu) dst.v[mu] = -double(0.5f * (t[mu] - amp * l[mu] * lt));
    }
    return d;
}

}  // namespace kp
