/*
 * scarf3d.h -- reference-compatible C/C++ interface of the B200 SCARF3D library.
 *
 * Same names, argument meaning and struct layout as SCARF3D's own header
 * (src/scarf3d.h:52-85 and the C++ wrapper :91-159), so that C and C++ callers
 * of the reference link against libscarf3d_b200.so unchanged. Single precision
 * only (the reference's default build; `real` = float). scarf_opt.method == 1
 * selects the SRM, 0 (the default) the FIM (scarflib_fim.f90:141-1104, on
 * cuFFT, with the reference's default build options: no rotated axes).
 *
 * Entry points and the reference interface each one replaces:
 *   scarf_opt_init           <- src/c_binding.c:62-80
 *   scarf_cart_initialize    <- src/c_binding.c:83-108 -> f_binding.f90:57-113
 *                               -> scarflib.f90:97-189
 *   scarf_nocart_initialize  <- src/c_binding.c:110-136 -> f_binding.f90:119-175
 *                               -> scarflib.f90:195-296
 *   scarf_execute            <- src/c_binding.c:138-143 -> f_binding.f90:181-217
 *                               -> scarflib.f90:302-426 -> scarflib_srm.f90:105-929
 *                               or scarflib_fim.f90:141-1104
 *   scarf_finalize           <- src/c_binding.c:145-150 -> scarflib.f90:432-455
 *   scarf_io_one             <- src/c_binding.c:154-158 -> scarflib_common.f90:245-418
 *   scarf_io_slice           <- src/c_binding.c:160-164 -> scarflib_common.f90:527-646
 */
#ifndef SCARF3D_H_
#define SCARF3D_H_

typedef float real;

#ifdef __cplusplus
extern "C" {
#endif

enum algorithm { fim, srm };

/* Optional arguments; a field counts as given when method == 1, hurst > 0,
 * dh > 0, ds > 0, poi != NULL, npoi > 0, mute > 0, taper > 0, rescale == 1,
 * pad == 1, nc && fc, alpha/beta/gamma != 0 (src/c_binding.c:89-103). */
struct scarf_opt {
  int method;
  real hurst;
  real dh;
  real ds;
  real *poi;
  int npoi;
  real mute;
  real taper;
  int rescale;
  int pad;
  real *nc;
  real *fc;
  real alpha;
  real beta;
  real gamma;
};

void scarf_opt_init(struct scarf_opt *var);

void scarf_cart_initialize(const int nd, const int fs[], const int fe[], const real ds, const int acf,
                           const real cl[], const real sigma, struct scarf_opt *var);

void scarf_nocart_initialize(const int nd, const int npts, const real *x, const real *y, const real *z,
                             const real dh, const int acf, const real cl[], const real sigma,
                             struct scarf_opt *var);

void scarf_execute(const int seed, real *field, real stats[]);

void scarf_finalize(void);

void scarf_io_one(const int nd, const int *npts, const real *field, const char fname[], const int *nwriters);

void scarf_io_slice(const int *npts, const char axis[], const int plane, const real *field, const char fname[]);

#ifdef __cplusplus
}

namespace Scarf3D {

inline scarf_opt options{0, 0, 0, 0, nullptr, 0, 0, 0, 0, 0, nullptr, nullptr, 0, 0, 0};

template <algorithm method>
class Initialize {
 public:
  Initialize(const int nd, const int fs[], const int fe[], const real ds, const int acf, const real cl[],
             const real sigma) {
    if (method == srm) options.method = 1;
    scarf_cart_initialize(nd, fs, fe, ds, acf, cl, sigma, &options);
  }
  Initialize(const int nd, const int npts, const real *x, const real *y, const real *z, const real dh,
             const int acf, const real cl[], const real sigma) {
    if (method == srm) options.method = 1;
    scarf_nocart_initialize(nd, npts, x, y, z, dh, acf, cl, sigma, &options);
  }
  Initialize(const int nd, const int npts, const real *x, const real *y, const real dh, const int acf,
             const real cl[], const real sigma) {
    if (method == srm) options.method = 1;
    scarf_nocart_initialize(nd, npts, x, y, nullptr, dh, acf, cl, sigma, &options);
  }
  ~Initialize() {
    scarf_finalize();
    options = {0, 0, 0, 0, nullptr, 0, 0, 0, 0, 0, nullptr, nullptr, 0, 0, 0};
  }
  void execute(const int seed, real *field, real stats[]) { scarf_execute(seed, field, stats); }
  void io(const int nd, const int npts[], const real *field, const char fname[], const int *nwriters = nullptr) {
    scarf_io_one(nd, npts, field, fname, nwriters);
  }
  void io(const int npts[], const char axis[], const int plane, const real *field, const char fname[]) {
    scarf_io_slice(npts, axis, plane, field, fname);
  }
};

}  // namespace Scarf3D
#endif

#endif /* SCARF3D_H_ */
