/* CPU restatement of the reference's FIM (Fourier integral method) path.
 *
 * TEST INFRASTRUCTURE ONLY (like srm_oracle.c, built into the same
 * liboracle_srm.so): tests/ use it as the checker of the CUDA FIM path, never
 * the product. Parity status: UNPINNED -- the reference (Fortran + MPI +
 * FFTW + TRNG4) cannot be built here and ships no golden vectors; the uniform
 * stream is the documented one of srm_oracle.c.
 *
 * Single precision in the reference's written operation order (no FMA
 * contraction, glibc single-precision libm), one process (the reference's
 * decomposition collapses to ls = 1, le = npts). Steps restated:
 *   internal grid          scarflib_fim.f90:787-828 (npts, offset, off_axis, info flags)
 *   spectrum               scarflib_fim.f90:2390-2547 (compute_spectrum)
 *   uniforms               prng.cpp:67-124 (one draw per internal grid point,
 *                          in x-fastest order, block-split by jumps)
 *   Hermitian symmetry     scarflib_fim.f90:2660-3007 (planes i = 1 and
 *                          i = npts(1)/2 + 1)
 *   mapping                scarflib_fim.f90:1303-1699, 3086-3162 (nearest
 *                          internal node, with the halo rules of exchange_halo
 *                          :3013-3080: zero below x and y, periodic in z)
 * The inverse transform itself (c2c along z and y, c2r along x, unnormalised)
 * is taken by the Python side with numpy's FFT in double precision.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "srm_oracle.h"

#define ORC_PI_F 3.141592653589793f

static int orc_nint(float x) { return (int)lroundf(x); } /* Fortran NINT: half away from zero */

/* Internal (FFT) grid of scarf3d_structured_fim / _unstructured_fim without
 * the DIP rotation (scarflib_fim.f90:787-815, 817-818). */
void orc_fim_grid(int ndim, const float nc[3], const float fc[3], float dh, const float cl[3], int pad, int npts[3],
                  float off_axis[3], float info01[2]) {
  for (int i = 0; i < 3; i++) {
    float span = ((fc[i] + dh * 0.5f) - nc[i]) + dh * 0.5f;
    npts[i] = orc_nint(span / dh) + 1;
    int offset = orc_nint(cl[i] / dh);
    if (pad != 1) offset = 0;
    npts[i] = npts[i] + 2 * offset;
    if (npts[i] % 2 != 0) npts[i] = npts[i] + 1;
    off_axis[i] = nc[i] - ((float)offset + 0.5f) * dh;
    if (ndim == 2 && i == 2) {
      off_axis[i] = -off_axis[i];
      npts[i] = 1;
    }
  }
  info01[0] = 0.0f;
  info01[1] = 0.0f;
  for (int i = 0; i < ndim; i++) {
    if (npts[i] <= orc_nint(2.0f * ORC_PI_F * cl[i] / dh)) info01[0] = 1.0f;
    if (dh > cl[i] / 2.0f) info01[1] = 1.0f;
  }
}

/* Wavenumber of 0-based index t on an axis of n points: t dk for t <= n/2,
 * (n - t) dk above (the reference's [0..n/2, n/2-1..1] * dk). */
static float orc_fim_k(int t, int n, float dk) {
  int m = (t <= n / 2) ? t : n - t;
  return (float)m * dk;
}

/* Amplitude constant and PSD of compute_spectrum (:2470-2485). */
static float orc_fim_const(int ndim, int acf, float sigma, float hurst, const float cl[3], float nu) {
  float prod = cl[0] * cl[1];
  if (ndim == 3) prod = prod * cl[2];
  float half_n = (float)ndim / 2.0f;
  if (acf == 0) {
    float c = (float)(1 << ndim) * powf(ORC_PI_F, half_n);
    c = c * tgammaf(nu);
    c = c * (sigma * sigma);
    c = c * prod;
    return c / tgammaf(hurst);
  }
  float c = powf(ORC_PI_F, half_n) * (sigma * sigma);
  return c * prod;
}

/* Spectrum over the half grid i = 0 .. n1/2 (the part the c2r transform
 * along x reads), layout spec[(k * n2 + j) * n1h + i] as interleaved
 * (re, im) floats, n1h = n1 / 2 + 1; then the Hermitian symmetry of planes
 * i = 0 and i = n1/2. */
void orc_fim_spectrum(const int npts[3], int ndim, float ds, float dh, int acf, const float cl[3], float sigma,
                      float hurst, int seed, float *spec) {
  const int n1 = npts[0], n2 = npts[1], n3 = npts[2];
  const int n1h = n1 / 2 + 1;
  float dk[3];
  for (int i = 0; i < 3; i++) dk[i] = 2.0f * ORC_PI_F / ((float)npts[i] * dh);
  const float kc = ORC_PI_F / ds;
  const int filter = ds != dh;
  const float nu = hurst + (float)ndim / 2.0f;
  const float cnst = orc_fim_const(ndim, acf, sigma, hurst, cl, nu);
  orc_rng g;
  orc_rng_seed(&g, seed);
  for (int k = 0; k < n3; k++) {
    const float kz = orc_fim_k(k, n3, dk[2]);
    for (int j = 0; j < n2; j++) {
      const float ky = orc_fim_k(j, n2, dk[1]);
      for (int i = 0; i < n1; i++) {
        const float u = orc_u01(orc_rng_next(&g)); /* one draw per internal point */
        if (i >= n1h) continue;
        const float kx = orc_fim_k(i, n1, dk[0]);
        float kr = sqrtf((kx * kx + ky * ky) + kz * kz);
        float butter = 1.0f;
        if (filter && kr > kc) butter = 0.0f;
        const float ax = kx * cl[0], ay = ky * cl[1], az = kz * cl[2];
        kr = sqrtf((ax * ax + ay * ay) + az * az);
        const float fv = (acf == 0) ? orc_fn_vk(kr, nu) : orc_fn_gs(kr);
        float amp = sqrtf(cnst * fv);
        amp = amp * butter;
        const float h = (u * 2.0f) * ORC_PI_F;
        float *c = spec + 2 * (((int64_t)k * n2 + j) * n1h + i);
        c[0] = cosf(h) * amp;
        c[1] = sinf(h) * amp;
      }
    }
  }
  /* enforce_symmetry (:2660-3007) on planes i = 0 and i = n1/2 (1-based 1
   * and nyquist(1)). Special points first, then conjugate mirrors of the
   * second half of each plane (sources are never written). */
  const int q2 = n2 / 2, q3 = n3 / 2; /* 0-based nyquist(2), nyquist(3) */
  const int planes[2] = {0, n1 / 2};
  for (int pi_ = 0; pi_ < 2; pi_++) {
    const int i = planes[pi_];
#define ORC_AT(jj, kk) (spec + 2 * (((int64_t)(kk) * n2 + (jj)) * n1h + i))
    if (i == 0) {
      ORC_AT(0, 0)[0] = 0.0f;
      ORC_AT(0, 0)[1] = 0.0f;
    } else {
      ORC_AT(0, 0)[1] = 0.0f;
    }
    ORC_AT(q2, q3)[1] = 0.0f;
    ORC_AT(0, q3)[1] = 0.0f;
    ORC_AT(q2, 0)[1] = 0.0f;
    /* k > nyquist(3): every j takes the conjugate of its mirror (n2 - j,
     * n3 - k); k = 0 and k = nyquist(3) with j > nyquist(2) likewise, except
     * the row k = 0 of a 3-D grid: exchange_conjg's second alltoallw gives
     * one process both of its subarray types (j = 1 column and k = 1 row) in
     * the same sendtypes(p) slot, so only the column travels and the row
     * keeps its own values, conjugated (:2880-2967, 2991-2995). */
    for (int k = 0; k < n3; k++) {
      for (int j = 0; j < n2; j++) {
        int w = 0;
        if (k > q3) w = 1;
        if ((k == 0 || k == q3) && j > q2) w = 1;
        if (!w) continue;
        int jm = (n2 - j) % n2, km = (n3 - k) % n3;
        if (k == 0 && n3 > 1) jm = j; /* the row that is not exchanged */
        const float *src = ORC_AT(jm, km);
        float *dst = ORC_AT(j, k);
        const float re = src[0], im = src[1];
        dst[0] = re;
        dst[1] = -im;
      }
    }
#undef ORC_AT
    if (n1 / 2 == 0) break;
  }
}

/* Nearest internal node of each external structured point (grid_mapping_struct
 * with order_points_struct and interpolate, no rotation): field[p] takes the
 * internal value delta at the node, or keeps 0 when the point falls outside.
 * delta: n1 x n2 x n3 internal field (x fastest). */
void orc_fim_map_structured(const int npts[3], const float *delta, float dh, const float off_axis[3], const int fs[3],
                            const int fe[3], float ds, float *field) {
  const int n1 = npts[0], n2 = npts[1], n3 = npts[2];
  const int e1 = fe[0] - fs[0] + 1, e2 = fe[1] - fs[1] + 1, e3 = fe[2] - fs[2] + 1;
  for (int k0 = 1; k0 <= e3; k0++) {
    const float z = (float)(fs[2] - 1 + k0 - 1) * ds - off_axis[2];
    for (int j0 = 1; j0 <= e2; j0++) {
      const float y = (float)(fs[1] - 1 + j0 - 1) * ds - off_axis[1];
      for (int i0 = 1; i0 <= e1; i0++) {
        const float x = (float)(fs[0] - 1 + i0 - 1) * ds - off_axis[0];
        const int64_t p = (i0 - 1) + (int64_t)e1 * ((j0 - 1) + (int64_t)e2 * (k0 - 1));
        /* identity rotation, bar = 0: ((1 x + 0 y) + 0 z) + 0 = x */
        const float fi = (x / dh + 3.0f) - 1.0f;
        const float fj = (y / dh + 3.0f) - 1.0f;
        const float fk = (z / dh + 3.0f) - 1.0f;
        field[p] = 0.0f;
        if (!(fi >= 1.0f && fi < (float)(n1 + 1) && fj >= 1.0f && fj < (float)(n2 + 1) && fk >= 1.0f &&
              fk < (float)(n3 + 1)))
          continue;
        /* 1-based index into delta(0:n1, 0:n2, 0:n3): internal node NINT - 1,
         * halo 0 = zero along x and y, the last plane along z (periodic). */
        const int a = orc_nint(fi) - 1, b = orc_nint(fj) - 1;
        int c = orc_nint(fk) - 1;
        if (a == 0 || b == 0) continue;
        if (c == 0) c = n3;
        field[p] = delta[(a - 1) + (int64_t)n1 * ((b - 1) + (int64_t)n2 * (c - 1))];
      }
    }
  }
}

/* The same for a point set (grid_mapping_unstruct / order_points_unstruct). */
void orc_fim_map_points(const int npts[3], const float *delta, float dh, const float off_axis[3], const float *x,
                        const float *y, const float *z, int64_t n, int ndim, float *field) {
  const int n1 = npts[0], n2 = npts[1], n3 = npts[2];
  for (int64_t p = 0; p < n; p++) {
    const float xc = x[p] - off_axis[0];
    const float yc = y[p] - off_axis[1];
    const float zc = z[p] - off_axis[2]; /* 2-D meshes pass z = 0 (the library's own zeros) */
    const float fi = (xc / dh + 3.0f) - 1.0f;
    const float fj = (yc / dh + 3.0f) - 1.0f;
    const float fk = (zc / dh + 3.0f) - 1.0f;
    field[p] = 0.0f;
    if (!(fi >= 1.0f && fi < (float)(n1 + 1) && fj >= 1.0f && fj < (float)(n2 + 1) && fk >= 1.0f &&
          fk < (float)(n3 + 1)))
      continue;
    const int a = orc_nint(fi) - 1, b = orc_nint(fj) - 1;
    int c = orc_nint(fk) - 1;
    if (a == 0 || b == 0) continue;
    if (c == 0) c = n3;
    field[p] = delta[(a - 1) + (int64_t)n1 * ((b - 1) + (int64_t)n2 * (c - 1))];
  }
}
