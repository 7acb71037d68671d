// kp_geometry_f32.cuh -- the Kerr-Schild transport right-hand side of the
// mixed-precision policy, in a factored form templated on the arithmetic
// type: FP32 in the far field, FP64 inside the radiating sphere.  The core
// (ks_transport_factored) works on T values; ks_rhs_factored wraps it for
// FP64 Rays.
//
// Same algebra as ks_rhs in kp_geometry.cuh (the reference's specialised
// transport_rhs, src/geometry/kerr_schild_cartesian.hpp:194-363), regrouped:
//  * four reciprocals (1/r, 1/discr, 1/(r^2 + a^2), 1/denom) replace the
//    twenty divisions of the connection work;
//  * every transport contracts the connection with p = k, so the pieces of
//    Gamma(k, q) that depend on k alone (l.k, dl_{nu a} k^a, dl_{nu a} k^nu,
//    df.k) are formed once;
//  * the sum over a of Gamma's rows collapses to
//      t_nu = l_nu (lq Dk + lk Dq + f (S_kq + S_qk)) + f (lq M_nu(k) + lk M_nu(q))
//             - [nu > 0] (df_nu lk lq + f (dlk_nu lq + lk dlq_nu)),
//    with D = df.v, M_nu(v) = dl_{nu a} v^a, dl(v)_a = dl_{nu a} v^nu,
//    S_kq = k^a dl(q)_a;
// about 320 operations per evaluation instead of 1080.  The rounding differs
// from the reference's order, so this form serves the mixed policy only.
#pragma once

#include "kp_geometry.cuh"

namespace kp {

// sqrt(v) with its reciprocal, and 1/v: FP64 as written; FP32 (the far
// field, where the contraction's own cancellation already limits it to
// ~3e-5) from one hardware reciprocal square root or reciprocal each, a few
// ulp instead of the correctly rounded IEEE sequences.
template<class T>
KP_HD void kp_sqrt_pair(T v, T& sq, T& inv) {
    sq = sqrt(v);
    inv = T(1) / sq;
}
template<>
KP_HD void kp_sqrt_pair<float>(float v, float& sq, float& inv) {
#ifdef __CUDA_ARCH__
    inv = rsqrtf(v);
    sq = v * inv;
#else
    sq = sqrtf(v);
    inv = 1.0f / sq;
#endif
}
template<class T>
KP_HD T kp_recip(T v) {
    return T(1) / v;
}
template<>
KP_HD float kp_recip<float>(float v) {
#ifdef __CUDA_ARCH__
    return __fdividef(1.0f, v);
#else
    return 1.0f / v;
#endif
}

// The transports of q[0] = k, q[1] = e1, q[2] = e2 at spatial position
// (x, y, z): out[w] = dq[w]/dlambda = -Gamma(k, q[w]).
template<class T>
KP_HD void ks_transport_factored(T M, T a, T x, T y, T z, const T (&q)[3][4], T (&out)[3][4]) {
    const T a2 = a * a;
    const T sqsum = x * x + y * y + z * z - a2;
    T discr, inv_discr;
    kp_sqrt_pair<T>(sqsum * sqsum + T(4) * a2 * z * z, discr, inv_discr);
    const T r2 = T(0.5) * (sqsum + discr);
    T r, inv_r;
    kp_sqrt_pair<T>(r2 > T(1e-30) ? r2 : T(1e-30), r, inv_r);
    const T inv_denom = kp_recip<T>(r2 * r2 + a2 * z * z);
    const T inv_rp = kp_recip<T>(r2 + a2);
    const T amp = T(2) * M * r2 * r * inv_denom;
    const T amp_r = T(-2) * M * r2 * (r2 * r2 - T(3) * a2 * z * z) * (inv_denom * inv_denom);
    const T l1 = (r * x + a * y) * inv_rp;
    const T l2 = (r * y - a * x) * inv_rp;
    const T l3 = z * inv_r;
    const T inv_2r = T(0.5) * inv_r;
    const T g12 = (T(1) + sqsum * inv_discr) * inv_2r;
    const T dr1 = x * g12, dr2 = y * g12;
    const T dr3 = z * (T(1) + (sqsum + T(2) * a2) * inv_discr) * inv_2r;
    const T d1 = amp_r * dr1, d2 = amp_r * dr2;
    const T d3 = (T(6) * M * r2 * dr3 - amp * (T(4) * r * r2 * dr3 + T(2) * a2 * z)) * inv_denom;
    // dl[nu][a] = d l_nu / d x^a
    const T tr = T(2) * r;
    const T c1 = tr * l1, c2 = tr * l2, c3 = -l3 * inv_r;
    const T dl11 = (r + (x - c1) * dr1) * inv_rp;
    const T dl21 = (-a + (y - c2) * dr1) * inv_rp;
    const T dl31 = c3 * dr1;
    const T dl12 = (a + (x - c1) * dr2) * inv_rp;
    const T dl22 = (r + (y - c2) * dr2) * inv_rp;
    const T dl32 = c3 * dr2;
    const T dl13 = (x - c1) * dr3 * inv_rp;
    const T dl23 = (y - c2) * dr3 * inv_rp;
    const T dl33 = (r - z * dr3) * (inv_r * inv_r);

    const T k0 = q[0][0], k1 = q[0][1], k2 = q[0][2], k3 = q[0][3];
    const T lk = k0 + l1 * k1 + l2 * k2 + l3 * k3;
    const T Mk1 = dl11 * k1 + dl12 * k2 + dl13 * k3;
    const T Mk2 = dl21 * k1 + dl22 * k2 + dl23 * k3;
    const T Mk3 = dl31 * k1 + dl32 * k2 + dl33 * k3;
    const T dlk1 = dl11 * k1 + dl21 * k2 + dl31 * k3;
    const T dlk2 = dl12 * k1 + dl22 * k2 + dl32 * k3;
    const T dlk3 = dl13 * k1 + dl23 * k2 + dl33 * k3;
    const T Dk = d1 * k1 + d2 * k2 + d3 * k3;

#pragma unroll
    for (int which = 0; which < 3; ++which) {
        const T q0 = q[which][0], q1 = q[which][1], q2 = q[which][2], q3 = q[which][3];
        const T lq = q0 + l1 * q1 + l2 * q2 + l3 * q3;
        const T Mq1 = dl11 * q1 + dl12 * q2 + dl13 * q3;
        const T Mq2 = dl21 * q1 + dl22 * q2 + dl23 * q3;
        const T Mq3 = dl31 * q1 + dl32 * q2 + dl33 * q3;
        const T dlq1 = dl11 * q1 + dl21 * q2 + dl31 * q3;
        const T dlq2 = dl12 * q1 + dl22 * q2 + dl32 * q3;
        const T dlq3 = dl13 * q1 + dl23 * q2 + dl33 * q3;
        const T Dq = d1 * q1 + d2 * q2 + d3 * q3;
        const T Skq = k1 * dlq1 + k2 * dlq2 + k3 * dlq3;
        const T Sqk = q1 * dlk1 + q2 * dlk2 + q3 * dlk3;
        const T common = lq * Dk + lk * Dq + amp * (Skq + Sqk);
        const T lklq = lk * lq;
        const T t0 = common;
        const T t1 = l1 * common + amp * (lq * Mk1 + lk * Mq1) - (d1 * lklq + amp * (dlk1 * lq + lk * dlq1));
        const T t2 = l2 * common + amp * (lq * Mk2 + lk * Mq2) - (d2 * lklq + amp * (dlk2 * lq + lk * dlq2));
        const T t3 = l3 * common + amp * (lq * Mk3 + lk * Mq3) - (d3 * lklq + amp * (dlk3 * lq + lk * dlq3));
        const T lt = -t0 + l1 * t1 + l2 * t2 + l3 * t3;
        const T al = amp * lt;
        out[which][0] = -(T(0.5) * (-t0 + al));
        out[which][1] = -(T(0.5) * (t1 - l1 * al));
        out[which][2] = -(T(0.5) * (t2 - l2 * al));
        out[which][3] = -(T(0.5) * (t3 - l3 * al));
    }
}

template<class T>
KP_HD Ray ks_rhs_factored(double mass_d, double spin_d, const Ray& s) {
    T q[3][4], o[3][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        q[0][i] = T(s.k.v[i]);
        q[1][i] = T(s.e1.v[i]);
        q[2][i] = T(s.e2.v[i]);
    }
    ks_transport_factored<T>(T(mass_d), T(spin_d), T(s.x.v[1]), T(s.x.v[2]), T(s.x.v[3]), q, o);
    Ray d;
    d.x = s.k;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        d.k.v[i] = double(o[0][i]);
        d.e1.v[i] = double(o[1][i]);
        d.e2.v[i] = double(o[2][i]);
    }
    return d;
}

}  // namespace kp
