/* kt_oracle.h -- TEST INFRASTRUCTURE: the CPU oracle of the geodesic path.
 *
 * A plain-C restatement of the reference renderer's per-pixel path (camera,
 * KNdS metric in BL and KS charts, Hamiltonian RHS, RK4 step doubling,
 * DOPRI5, Hermite event location, disk redshift, Jacobi ray bundles,
 * thin-disk shading), written to reproduce the reference's floating-point
 * operation order exactly.  Compiled with -ffp-contract=off and the
 * renderer's own libm (ktmath.h) it is bit-identical to the reference built
 * the same way (oracle/_ref/libktref_strict.so); tests/test_oracle.py checks
 * that on every path.  Only the tests, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it, as the checker; the product never does. */
#ifndef KT_ORACLE_H
#define KT_ORACLE_H

#include <stdint.h>
#include "../include/kerrtrace.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-frame host derivations (trace_geodesics main.cpp:2033-2082). */
int orc_frame_derive(const kt_frame_desc* d, kt_frame_derived* out);

double orc_r_horizon(double M, double a, double Q, double L);
double orc_r_isco(double M, double a, double Q, double L);

/* Trace pixels pix[i] = py*width+px; float64 SoA out (GeoPixel slots).
 * steps/attempts may be NULL.  nthreads <= 0: OpenMP default. */
void orc_trace_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix,
                      uint8_t* outcome, double* r, double* redshift, double* magnif,
                      double* phi_disk, double* theta_esc, double* phi_esc,
                      uint32_t* steps, uint32_t* attempts, int nthreads);

/* colorize_buffer on float64 SoA (rounded to float32 first, as GeoPixel
 * does), blackbody palette, RGB8 background or NULL. */
void orc_colorize(const kt_frame_desc* d, int64_t n, const uint8_t* outcome, const double* r,
                  const double* redshift, const double* magnif, const double* theta_esc,
                  const double* phi_esc, double exposure, double gamma, double temp_scale,
                  const uint8_t* bg, int bg_w, int bg_h, uint8_t* rgb);

/* colorize_buffer with every ColorParams field (blackbody or interstellar
 * palette, main.cpp:1719-1866); disk edges r_isco and disk_out. */
void orc_colorize_cp(const kt_frame_desc* d, int64_t n, const uint8_t* outcome, const double* r,
                     const double* redshift, const double* magnif, const double* phi_disk,
                     const double* theta_esc, const double* phi_esc, const kt_color_params* cp,
                     const uint8_t* bg, int bg_w, int bg_h, uint8_t* rgb);

/* --camera-spp: jitter offsets (2*spp doubles) and the linear-light average
 * of spp RGB8 passes (spp*n*3 bytes, pass after pass). */
void orc_spp_offsets(int spp, double* xy);
void orc_spp_combine(int64_t n, int spp, const uint8_t* passes, double gamma, uint8_t* rgb);
void orc_elliptic_reasons(const kt_frame_desc* d, int64_t n, const uint32_t* pix, uint8_t* reason);

/* Known-answer helpers (tests/core_tests.cpp of the reference). */
void orc_metric_bl(double M, double a, double Q, double L, double r, double th, double* cov16,
                   double* con16);
double orc_hamiltonian(double M, double a, double Q, double L, const double* s7);
void orc_angle_ray(double M, double a, double Q, double L, double r_obs, double th_deg,
                   double ph_deg, double fov_deg, int W, int H, double alpha, double beta,
                   double* s7);
int orc_adaptive_step(double M, double a, double Q, double L, double* s7, double* h, int dopri5,
                      double* fsal4, double tol);
double orc_keplerian_omega(double M, double a, double Q, double L, double r);
void orc_bl_to_ks(double r, double th, double ph, double a, double* xyz);
double orc_r_ks(double X, double Y, double Z, double a);

#ifdef __cplusplus
}
#endif
#endif
