/*
 * kp_oracle.h -- CPU restatement of the reference's per-pixel GRRT path,
 * used ONLY as test infrastructure (parity checker, CPU baseline).  The
 * product library never includes or links it.
 *
 * Parity pinning: every function follows the cited reference file:line with
 * the same floating-point operation order and is compiled with
 * -ffp-contract=off, so on identical inputs it reproduces the reference's
 * own templates (built as oracle/_ref/libkpref.so) bit for bit; the tests
 * check this and also check the reference's known-answer values
 * (tests/test_core.cpp:247-288, :2188-2240 of the reference).
 */
#ifndef KP_ORACLE_H
#define KP_ORACLE_H

#include "kpolaris_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Pixels [pixel_begin, pixel_end) of a RIAF image; OpenMP `threads` (0 = all).
 * integrator: kp_integrator.  Writes only the selected pixels of *out. */
int kpo_image_riaf_range(const kp_pass_a_params* params, const kp_riaf_model* model,
                         int radiation_substeps, const double* freqs, int nfreq,
                         int integrator, int threads, int pixel_begin, int pixel_end,
                         kp_image_out* out);

int kpo_thermal_coefficients(int fit, double nu, double ne, double thetae, double b_cgs,
                             double theta, double sin_theta, double cos_theta,
                             double max_pol_frac, double min_sin_theta, double* out11);
int kpo_stokes_step(double* stokes4, const double* coeffs11, double dlambda);
int kpo_riaf_coefficients_cks(double mass, double spin, const kp_riaf_model* model,
                              const double* state16, double* out11);
int kpo_camera_ray_cks(const kp_pass_a_params* params, int pixel, double* state16);
int kpo_transport_rhs_cks(double mass, double spin, const double* state16, double* d16);
int kpo_adaptive_step_cks(int integrator, double mass, double spin, const double* state16, double requested_h,
                          double tolerance, double min_step, double max_step, int max_attempts,
                          double* out32, double* scalars3);
const char* kpo_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
