// libscarf3d_b200_fbind.so -- the reference's Fortran BIND(C) layer
// (src/f_binding.f90) over libscarf3d_b200.so.
//
// The reference's C wrapper (src/c_binding.c) implements scarf_* by calling
// these six routines, which its Fortran module exports: arguments by
// reference, optional ones as NULL pointers, fields passed as the address of
// the caller's pointer (c_binding.c:138-164). A program that links the
// reference's own c_binding.c, or calls these names directly, links this shim
// (and libscarf3d_b200.so next to it) in place of libscarflib. The names are
// kept out of the main library on purpose: `execute` and `finalize` are
// common symbols that would clash in unrelated programs.
//
// An optional argument counts as given when its pointer is non-NULL, as in
// the Fortran routines; the values are then handed to the C API, whose
// "given" rule (c_binding.c:89-103: method == 1, hurst > 0, ...) the
// reference's wrapper has already applied before passing a pointer.
#include "scarf3d.h"

extern "C" {

// f_binding.f90:57-113
void struct_initialize(const int* nd, const int* fs, const int* fe, const real* ds, const int* acf, const real* cl,
                       const real* sigma, const int* method, const real* hurst, const real* dh, real** poi,
                       const int* np, const real* mute, const real* taper, const int* rescale, const int* pad,
                       const real* nc, const real* fc, const real* alpha, const real* beta, const real* gamma) {
  scarf_opt o;
  scarf_opt_init(&o);
  if (method) o.method = *method;
  if (hurst) o.hurst = *hurst;
  if (dh) o.dh = *dh;
  if (poi) o.poi = *poi;
  if (np) o.npoi = *np;
  if (mute) o.mute = *mute;
  if (taper) o.taper = *taper;
  if (rescale) o.rescale = *rescale;
  if (pad) o.pad = *pad;
  if (nc && fc) {
    o.nc = const_cast<real*>(nc);
    o.fc = const_cast<real*>(fc);
  }
  if (alpha) o.alpha = *alpha;
  if (beta) o.beta = *beta;
  if (gamma) o.gamma = *gamma;
  scarf_cart_initialize(*nd, fs, fe, *ds, *acf, cl, *sigma, &o);
}

// f_binding.f90:119-175 (argument order as the Fortran routine declares it)
void unstruct_initialize(const int* nd, const int* npts, const real* dh, const int* acf, const real* cl,
                         const real* sigma, const real* x, const real* y, const real* z, const int* method,
                         const real* hurst, const real* ds, real** poi, const int* np, const real* mute,
                         const real* taper, const int* rescale, const int* pad, const real* nc, const real* fc,
                         const real* alpha, const real* beta, const real* gamma) {
  scarf_opt o;
  scarf_opt_init(&o);
  if (method) o.method = *method;
  if (hurst) o.hurst = *hurst;
  if (ds) o.ds = *ds;
  if (poi) o.poi = *poi;
  if (np) o.npoi = *np;
  if (mute) o.mute = *mute;
  if (taper) o.taper = *taper;
  if (rescale) o.rescale = *rescale;
  if (pad) o.pad = *pad;
  if (nc && fc) {
    o.nc = const_cast<real*>(nc);
    o.fc = const_cast<real*>(fc);
  }
  if (alpha) o.alpha = *alpha;
  if (beta) o.beta = *beta;
  if (gamma) o.gamma = *gamma;
  scarf_nocart_initialize(*nd, *npts, x, y, z, *dh, *acf, cl, *sigma, &o);
}

// f_binding.f90:181-217: `field` is the address of the caller's pointer.
void execute(const int* seed, real** field, real* stats) { scarf_execute(*seed, *field, stats); }

// f_binding.f90:223-240
void finalize() { scarf_finalize(); }

// f_binding.f90:246-292
void io_one(const int* nd, const int* npts, real** field, const char* fout, const int* nwriters) {
  scarf_io_one(*nd, npts, *field, fout, nwriters);
}

// f_binding.f90:298-
void io_slice(const int* n, const char* axis, const int* plane, real** field, const char* fout) {
  scarf_io_slice(n, axis, *plane, *field, fout);
}

}  // extern "C"
