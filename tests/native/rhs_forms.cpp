// Host check of the mixed policy's factored transport RHS
// (kpolaris_b200/csrc/kp_geometry_f32.cuh) against the reference-order FP64
// RHS (kp_geometry.cuh) on seeded states around a Kerr black hole.  Prints
// the largest normwise relative deviation of the FP64 form (all radii) and of
// the FP32 form beyond r = 100 M (where the mixed policy uses it).
#include <cmath>
#include <cstdio>
#include <random>
#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__
#include "kp_geometry_f32.cuh"

int main() {
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    double worst64 = 0.0, far32 = 0.0;
    for (int i = 0; i < 20000; ++i) {
        const double spin = 0.99 * std::fabs(u(rng));
        const double rad = 1.5 + std::pow(10.0, 3.0 * std::fabs(u(rng)));
        double dir[3] = {u(rng), u(rng), u(rng)};
        const double n = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]) + 1e-12;
        kp::Ray s;
        s.x.v[0] = 0.0;
        for (int k = 0; k < 3; ++k) s.x.v[k + 1] = rad * dir[k] / n;
        for (int k = 0; k < 4; ++k) {
            s.k.v[k] = u(rng);
            s.e1.v[k] = u(rng);
            s.e2.v[k] = u(rng);
        }
        s.k.v[0] = 1.0 + std::fabs(u(rng));
        const kp::Ray ref = kp::ks_rhs(1.0, spin, s);
        const kp::Ray f64 = kp::ks_rhs_factored<double>(1.0, spin, s);
        const kp::Ray f32 = kp::ks_rhs_factored<float>(1.0, spin, s);
        const kp::D4* R[3] = {&ref.k, &ref.e1, &ref.e2};
        const kp::D4* A[3] = {&f64.k, &f64.e1, &f64.e2};
        const kp::D4* B[3] = {&f32.k, &f32.e1, &f32.e2};
        for (int w = 0; w < 3; ++w) {
            double scale = 0.0, d64 = 0.0, d32 = 0.0;
            for (int k = 0; k < 4; ++k) {
                scale = std::fmax(scale, std::fabs(R[w]->v[k]));
                d64 = std::fmax(d64, std::fabs(A[w]->v[k] - R[w]->v[k]));
                d32 = std::fmax(d32, std::fabs(B[w]->v[k] - R[w]->v[k]));
            }
            if (scale > 0.0) {
                worst64 = std::fmax(worst64, d64 / scale);
                if (rad > 100.0) far32 = std::fmax(far32, d32 / scale);
            }
        }
    }
    std::printf("%.3e %.3e\n", worst64, far32);
    return 0;
}
