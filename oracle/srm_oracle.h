/*
 * srm_oracle.h -- CPU restatement of SCARF3D's spectral-representation method
 * (SRM), used ONLY as test infrastructure: by tests/, by the smoke check and by
 * bench.py's CPU-baseline leg. The product library never links or calls it.
 *
 * Parity status: UNPINNED. The reference (Fortran 2003 + MPI + TRNG4) cannot be
 * compiled in this environment (no Fortran compiler, no MPI, no TRNG4) and ships
 * no golden vectors or known-answer tests. This restatement follows the reference
 * source line by line (citations below) and is checked against analytic known
 * answers (spectral integrals, rotation identities) and the reference's own
 * invariants (structured == unstructured on the same points, decomposition
 * invariance, rescale gives std == sigma, mute zeroes the radius).
 *
 * The uniform random source is a YARN2-type generator restated from TRNG's
 * published description (order-2 multiple recursive generator modulo 2^31-1
 * with an exponentiation output transform); it is unverified against a TRNG
 * build. Everything downstream of the uniform draws is a faithful restatement.
 */
#ifndef SRM_ORACLE_H
#define SRM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Inputs of one SRM call (scarflib.f90:67-87 scarf_obj, restricted to SRM). */
typedef struct {
  int ndim_hint;      /* unused by the algorithm: ndim follows cl[2] > 0          */
  int acf;            /* 0 = von Karman, 1 = Gaussian                              */
  int nharm;          /* number of harmonics (reference: constant 10000)          */
  int seed;
  int rescale;        /* 1 = rescale discrete std to sigma                        */
  float hurst, sigma, ds, dh;
  float cl[3], nc[3], fc[3];
  float alpha, beta, gamma;
} orc_params;

/* Derived scalars (scarflib_srm.f90:617-720). */
typedef struct {
  int ndim;
  float kmin, kmax, kc, nu, cnst, scaling, scaling0;
  float m[9];         /* rotation matrix, row-major: m[3*r + c] = matrix(r+1,c+1) */
  float bar[3];       /* translation after rotation about the half span           */
  float info0, info1; /* "domain too small", "grid-step too large"                */
  float intg_band, intg_full;
  int ier_band, ier_full;
} orc_setup;

/* --- uniform source ------------------------------------------------------ */
typedef struct { int64_t r0, r1; } orc_rng;
void orc_rng_seed(orc_rng *g, int seed);
uint32_t orc_rng_next(orc_rng *g);            /* raw output in [0, 2^31-2]  */
float orc_u01(uint32_t y);                   /* [0,1] float: double draw rounded to float */
void orc_srng(orc_rng *g, float r[2]);       /* prng.cpp:152-165 analogue  */

/* --- spectra and quadrature ---------------------------------------------- */
float orc_fn_vk(float x, float nu);
float orc_fn_gs(float x);
double orc_srm_fn(double x, int ndim, int acf, float nu);
void orc_dqng(int ndim, int acf, float nu, double a, double b, double epsabs,
              double epsrel, double *result, double *abserr, int *neval, int *ier);
void orc_dqagi(int ndim, int acf, float nu, double bound, int inf, double epsabs,
               double epsrel, int limit, double *result, double *abserr,
               int *neval, int *ier, int *last);

/* --- setup and sampler --------------------------------------------------- */
int orc_setup_compute(const orc_params *p, orc_setup *s);
/* Writes up to nharm rows {v1,v2,v3,a,b}; returns the number of rows kept
 * (harmonics with u > kc are dropped, scarflib_srm.f90:751). *pairs receives
 * the number of srng() calls consumed. */
int orc_sample(const orc_params *p, const orc_setup *s, float *tab, int64_t *pairs);

/* --- sums (selected points, linear index i + nx*(j + ny*k), 0-based) ----- */
void orc_sum_structured_f32(const orc_setup *s, const int fs[3], const int n[3],
                            float ds, const float *tab, int nh,
                            const int64_t *idx, int64_t nidx, float *out);
void orc_sum_structured_f64(const orc_setup *s, const int fs[3], const int n[3],
                            float ds, const float *tab, int nh,
                            const int64_t *idx, int64_t nidx, double *out);
void orc_sum_points_f32(const orc_setup *s, const float *x, const float *y,
                        const float *z, const float *tab, int nh,
                        const int64_t *idx, int64_t nidx, float *out);
void orc_sum_points_f64(const orc_setup *s, const float *x, const float *y,
                        const float *z, const float *tab, int nh,
                        const int64_t *idx, int64_t nidx, double *out);
/* Multi-threaded FP32 restatement over all points of a structured block
 * (each worker evaluates every harmonic for its points, like an MPI rank). */
void orc_sum_structured_f32_mt(const orc_setup *s, const int fs[3], const int n[3],
                               float ds, const float *tab, int nh,
                               float *field, int nthreads);
void orc_sum_points_f32_mt(const orc_setup *s, const float *x, const float *y,
                           const float *z, int64_t npts, const float *tab, int nh,
                           float *field, int nthreads);

/* --- statistics, rescale, taper ----------------------------------------- */
float orc_mean(const float *f, int64_t n);
float orc_variance(const float *f, int64_t n);
void orc_parallel_variance(const float *var, const float *avg, const int *nset,
                           int nsets, float *var_out, float *avg_out);
void orc_rescale(float *f, int64_t n, float sigma, float std, float mean);
void orc_taper_structured(float dh, const int fs[3], const int fe[3], float *field,
                          const float poi[3], float mute, float taper);
void orc_taper_points(const float *x, const float *y, const float *z, int64_t n,
                      float *field, const float poi[3], float mute, float taper);

/* Whole structured execute on the CPU (scarflib_srm.f90:505-929):
 * field (n0*n1*n2, column-major) and info[6]. nthreads > 1 parallelises the
 * sum over points. Returns 0 on success. */
int orc_execute_structured(const orc_params *p, const int fs[3], const int fe[3],
                           const float *poi, int npoi, float mute, float taper,
                           float *field, float info[6], int nthreads);

/* FIM restatement (fim_oracle.c): internal grid, spectrum with Hermitian
 * planes (half grid, interleaved complex), nearest-node mapping. */
void orc_fim_grid(int ndim, const float nc[3], const float fc[3], float dh, const float cl[3], int pad, int npts[3],
                  float off_axis[3], float info01[2]);
void orc_fim_spectrum(const int npts[3], int ndim, float ds, float dh, int acf, const float cl[3], float sigma,
                      float hurst, int seed, float *spec);
void orc_fim_map_structured(const int npts[3], const float *delta, float dh, const float off_axis[3], const int fs[3],
                            const int fe[3], float ds, float *field);
void orc_fim_map_points(const int npts[3], const float *delta, float dh, const float off_axis[3], const float *x,
                        const float *y, const float *z, int64_t n, int ndim, float *field);

#ifdef __cplusplus
}
#endif
#endif
