// kp_geometry.cuh -- Kerr spacetime in Cartesian Kerr-Schild coordinates and
// the transport right-hand side, FP64.
//
// The metric is g = eta + f l (x) l (src/geometry/kerr_schild_cartesian.hpp:19-51).
// The connection is never formed: Gamma(p, q) is contracted directly from
// (f, df, l, dl) as the reference's specialised transport_rhs does
// (kerr_schild_cartesian.hpp:194-363).  The expressions keep the reference's
// IEEE operation order (compiled with --fmad=false in the FP64 kernels) so
// integer outputs (termination, step counts) are bit-identical to its CPU run.
#pragma once

#include "kp_common.cuh"

namespace kp {

KP_HD D4 d4(double a, double b, double c, double d) {
    D4 o;
    o.v[0] = a;
    o.v[1] = b;
    o.v[2] = c;
    o.v[3] = d;
    return o;
}

KP_HD D4 d4_scale(const D4& a, double s) {
    return d4(a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s);
}

KP_HD D4 d4_sub_scaled(const D4& a, const D4& b, double s) {
    return d4(a.v[0] - b.v[0] * s, a.v[1] - b.v[1] * s, a.v[2] - b.v[2] * s, a.v[3] - b.v[3] * s);
}


// Radius only: the `r` of KerrSchildInMetric::build_work (:27-40).
KP_HD double ks_radius(double spin, const D4& X) {
    const double x = X.v[1], y = X.v[2], z = X.v[3];
    const double a2 = spin * spin;
    const double radius2 = x * x + y * y + z * z;
    const double sqsum = radius2 - a2;
    const double discr = sqrt(sqsum * sqsum + 4.0 * a2 * z * z);
    const double r2 = 0.5 * (sqsum + discr);
    return sqrt(max_val(r2, kTiny));
}

// f and l of the Kerr-Schild form (build_work, :27-51).
struct KSMetricPoint {
    double amp;
    double l[4];
};

KP_HD KSMetricPoint ks_point(double mass, double spin, const D4& X) {
    const double x = X.v[1], y = X.v[2], z = X.v[3];
    const double a = spin;
    const double a2 = spin * spin;
    const double radius2 = x * x + y * y + z * z;
    const double sqsum = radius2 - a2;
    const double discr = sqrt(sqsum * sqsum + 4.0 * a2 * z * z);
    const double r2 = 0.5 * (sqsum + discr);
    const double r = sqrt(max_val(r2, kTiny));
    const double denom = r2 * r2 + a2 * z * z;
    KSMetricPoint p;
    p.amp = 2.0 * mass * r2 * r / denom;
    const double r2pa2 = r2 + a2;
    p.l[0] = 1.0;
    p.l[1] = (r * x + a * y) / r2pa2;
    p.l[2] = (r * y - a * x) / r2pa2;
    p.l[3] = z / r;
    return p;
}

// g(u, v) (KerrSchildInMetric::dot, :92-108).
KP_HD double ks_dot_at(const KSMetricPoint& w, const D4& u, const D4& v) {
    double eta_dot = 0.0 + (-u.v[0]) * v.v[0];
    eta_dot += u.v[1] * v.v[1];
    eta_dot += u.v[2] * v.v[2];
    eta_dot += u.v[3] * v.v[3];
    double lu = 0.0 + u.v[0];
    double lv = 0.0 + v.v[0];
    lu += w.l[1] * u.v[1];
    lv += w.l[1] * v.v[1];
    lu += w.l[2] * u.v[2];
    lv += w.l[2] * v.v[2];
    lu += w.l[3] * u.v[3];
    lv += w.l[3] * v.v[3];
    return eta_dot + w.amp * lu * lv;
}

KP_HD double ks_dot(double mass, double spin, const D4& X, const D4& u, const D4& v) {
    return ks_dot_at(ks_point(mass, spin, X), u, v);
}

// g_{mu nu} (gcov_matrix, :72-79).
KP_HD void ks_gcov_matrix(double mass, double spin, const D4& X, double g[4][4]) {
    const KSMetricPoint w = ks_point(mass, spin, X);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) {
            const double eta = mu != nu ? 0.0 : (mu == 0 ? -1.0 : 1.0);
            g[mu][nu] = eta + w.amp * w.l[mu] * w.l[nu];
        }
}

// g^{mu nu} (gcon, :65-70): eta - f lcon lcon with lcon_0 = -1.
KP_HD double ks_gcon_entry(const KSMetricPoint& w, int mu, int nu) {
    const double lmu = (mu == 0 ? -w.l[0] : w.l[mu]);
    const double lnu = (nu == 0 ? -w.l[0] : w.l[nu]);
    const double eta = mu != nu ? 0.0 : (mu == 0 ? -1.0 : 1.0);
    return eta - w.amp * lmu * lnu;
}

// Connection work: f, df, l, dl (build_ks_connection_work, :198-252).
// dl[mu][alpha] is stored for mu, alpha in 1..3 only (row/column 0 vanish).
struct KSConn {
    double amp;
    double damp[4];
    double l[4];
    double dl[4][4];
};

KP_HD KSConn ks_conn(double mass, double spin, const D4& X) {
    const double x = X.v[1], y = X.v[2], z = X.v[3];
    const double a = spin;
    const double a2 = spin * spin;
    const double radius2 = x * x + y * y + z * z;
    const double sqsum = radius2 - a2;
    const double discr = sqrt(sqsum * sqsum + 4.0 * a2 * z * z);
    const double r2 = 0.5 * (sqsum + discr);
    const double r = sqrt(max_val(r2, kTiny));
    const double denom = r2 * r2 + a2 * z * z;
    const double amp = 2.0 * mass * r2 * r / denom;
    const double amp_r = -2.0 * mass * r2 * (r2 * r2 - 3.0 * a2 * z * z) / (denom * denom);
    const double r2pa2 = r2 + a2;
    KSConn c;
    c.amp = amp;
    c.l[0] = 1.0;
    c.l[1] = (r * x + a * y) / r2pa2;
    c.l[2] = (r * y - a * x) / r2pa2;
    c.l[3] = z / r;
    const double r2pa2_2 = r2pa2 * r2pa2;
    const double inv_2r = 0.5 / r;
    const double dr1 = (x + sqsum * x / discr) * inv_2r;
    const double dr2 = (y + sqsum * y / discr) * inv_2r;
    const double dr3 = (z + (sqsum * z + 2.0 * a2 * z) / discr) * inv_2r;
    c.damp[0] = 0.0;
    c.damp[1] = amp_r * dr1;
    c.damp[2] = amp_r * dr2;
    c.damp[3] = 6.0 * mass * r2 * dr3 / denom - amp / denom * (4.0 * r * r2 * dr3 + 2.0 * a2 * z);
    const double px = r * x + a * y;
    const double py = r * y - a * x;
    c.dl[1][1] = ((r + x * dr1) * r2pa2 - 2.0 * r * px * dr1) / r2pa2_2;
    c.dl[2][1] = ((-a + y * dr1) * r2pa2 - 2.0 * r * py * dr1) / r2pa2_2;
    c.dl[3][1] = -z / r2 * dr1;
    c.dl[1][2] = ((a + x * dr2) * r2pa2 - 2.0 * r * px * dr2) / r2pa2_2;
    c.dl[2][2] = ((r + y * dr2) * r2pa2 - 2.0 * r * py * dr2) / r2pa2_2;
    c.dl[3][2] = -z / r2 * dr2;
    c.dl[1][3] = (x * dr3 * r2pa2 - 2.0 * r * px * dr3) / r2pa2_2;
    c.dl[2][3] = (y * dr3 * r2pa2 - 2.0 * r * py * dr3) / r2pa2_2;
    c.dl[3][3] = (r - z * dr3) / r2;
    return c;
}

// Gamma^mu_{ab} p^a q^b without forming Gamma (ks_connection_contract, :302-327).
// l.p, l.q, dl_alpha.p, dl_alpha.q are evaluated once per call; every term
// keeps the reference's summation order.
KP_HD D4 ks_contract(const KSConn& c, const D4& p, const D4& q) {
    const double lp = ((0.0 + p.v[0]) + c.l[1] * p.v[1] + c.l[2] * p.v[2]) + c.l[3] * p.v[3];
    const double lq = ((0.0 + q.v[0]) + c.l[1] * q.v[1] + c.l[2] * q.v[2]) + c.l[3] * q.v[3];
    double dlp[4], dlq[4];
#pragma unroll
    for (int a = 1; a < 4; ++a) {
        dlp[a] = ((0.0 + c.dl[1][a] * p.v[1]) + c.dl[2][a] * p.v[2]) + c.dl[3][a] * p.v[3];
        dlq[a] = ((0.0 + c.dl[1][a] * q.v[1]) + c.dl[2][a] * q.v[2]) + c.dl[3][a] * q.v[3];
    }
    double t[4];
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
        // dl[0][alpha] = 0: the row-0 contraction has no dl term.
        double term = 0.0;
#pragma unroll
        for (int a = 1; a < 4; ++a) {
            const double dlnu = nu == 0 ? 0.0 : c.dl[nu][a];
            const double row_q = c.damp[a] * c.l[nu] * lq + c.amp * (dlnu * lq + c.l[nu] * dlq[a]);
            const double row_p = c.damp[a] * c.l[nu] * lp + c.amp * (dlnu * lp + c.l[nu] * dlp[a]);
            term += p.v[a] * row_q + q.v[a] * row_p;
        }
        if (nu != 0) {
            term -= c.damp[nu] * lp * lq + c.amp * (dlp[nu] * lq + lp * dlq[nu]);
        } else {
            term -= 0.0;
        }
        t[nu] = term;
    }
    // lcon = (-1, l1, l2, l3)
    double lt = 0.0 + (-c.l[0]) * t[0];
    lt += c.l[1] * t[1];
    lt += c.l[2] * t[2];
    lt += c.l[3] * t[3];
    D4 out;
    out.v[0] = 0.5 * (-t[0] - c.amp * (-c.l[0]) * lt);
#pragma unroll
    for (int mu = 1; mu < 4; ++mu) out.v[mu] = 0.5 * (t[mu] - c.amp * c.l[mu] * lt);
    return out;
}

// dx = k, dk = -Gamma(k,k), de_i = -Gamma(k, e_i) (transport_rhs, :347-363).
KP_HD Ray ks_rhs(double mass, double spin, const Ray& s) {
    Ray d;
    d.x = s.k;
    const KSConn c = ks_conn(mass, spin, s.x);
    const D4 ck = ks_contract(c, s.k, s.k);
    const D4 ce1 = ks_contract(c, s.k, s.e1);
    const D4 ce2 = ks_contract(c, s.k, s.e2);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        d.k.v[mu] = -ck.v[mu];
        d.e1.v[mu] = -ce1.v[mu];
        d.e2.v[mu] = -ce2.v[mu];
    }
    return d;
}

}  // namespace kp
