// Host-side pieces of the SRM path: parameters, derived setup, uniform
// source, quadrature and the harmonic sampler. Pure C++ (no CUDA types).
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>

#include "scarf3d_b200.h"

namespace scarf {

// YARN2-type uniform source: order-2 multiple recursive generator modulo the
// Mersenne prime 2^31-1 (multipliers 1498809829, 1160990996) whose output is
// the power g^r mod (2^31-1), g = 123567893 -- the parameters TRNG publishes
// for trng::yarn2, which prng.cpp:60 instantiates. A draw is
// trng::uniform01_dist<> with its default (double) result type, stored into
// a float as srng does (prng.cpp:152-165): y * (1/m) in double, rounded to
// float, so 0 <= draw <= 1 (0 for y = 0, 1.0f for the largest y).
class Yarn2 {
 public:
  static constexpr uint64_t kMod = 2147483647ull;
  static constexpr uint64_t kA1 = 1498809829ull;
  static constexpr uint64_t kA2 = 1160990996ull;
  static constexpr uint64_t kGen = 123567893ull;

  void seed(int s);
  uint32_t next_raw();
  float next_u01() { return to_u01(next_raw()); }
  // Advance the state by n raw draws in O(log n).
  void jump(uint64_t n);

  static float to_u01(uint32_t y) { return static_cast<float>(static_cast<double>(y) * kInvMod); }
  static constexpr double kInvMod = 0x1.00000002p-31;  // 1 / (2^31 - 1), rounded to double
  static uint32_t output(uint64_t r);  // g^r mod m (0 for r == 0)
  static uint64_t mulmod(uint64_t a, uint64_t b);

  uint64_t r0 = 0, r1 = 1;  // r0 = newest state word
};

// Output-transform tables of the device generator (yarn2.cuh): g^k,
// g^(k 2^11), g^(k 2^22) mod m for k < 2048, 2048, 512.
std::vector<uint32_t> device_pow_tables();

// Spectral integrand of the SRM (scarflib_srm.f90:975-995 with
// psdf.f90:50-90): x * psd(float(x)) [* x in 3D], FP32 spectrum, FP64 rest.
double srm_fn(double x, int ndim, int acf, float nu);

// QUADPACK restatements (quadpack.f90): DQNG (:8137) over [a,b] and DQAGI
// (:1177, via DQAGIE :712) over [bound, +inf). Return the QUADPACK ier.
int quad_dqng(int ndim, int acf, float nu, double a, double b, double epsabs, double epsrel, double* result,
              double* abserr);
int quad_dqagi(int ndim, int acf, float nu, double bound, double epsabs, double epsrel, int limit,
               double* result, double* abserr);

// Derived scalars (scarflib_srm.f90:617-720).
int srm_setup(const scarf_srm_params& p, scarf_srm_setup* s);

// Harmonic sampler (scarflib_srm.f90:731-778). Fills table rows
// {v1,v2,v3,a,b} for kept harmonics; returns the count kept. Uses the
// caller-supplied uniform source when one is installed, else Yarn2; with
// Yarn2 the rejection tests run on `threads` host threads over jumped
// sub-streams and the result is identical to the serial walk.
struct UniformSource {
  void (*set_seed)(int) = nullptr;
  void (*srng)(float*) = nullptr;
};
int srm_sample(const scarf_srm_params& p, const scarf_srm_setup& s, const UniformSource* src, int threads,
               float* table, long long* pairs_used);

// Success probability of one rejection trial: spectral mass in [kmin, kmax]
// times the majorant constant over the interval width. srm_sample returns -1
// without drawing when it is below kMinAcceptance (the domain is too small
// for the correlation lengths, e.g. a Gaussian spectrum whose bulk lies below
// kmin).
constexpr double kMinAcceptance = 1e-6;
double acceptance_rate(const scarf_srm_setup& s);

// Same table as srm_sample with the built-in generator, with the rejection
// tests run on the current GPU: the device evaluates every pair of the
// stream and the host walks the accepted ones (and decides the few pairs
// whose test lies within float rounding of the threshold), so the result is
// bit-identical to the serial host loop. Returns the harmonics kept, -1 if
// rejection sampling is infeasible, -2 on a CUDA error. *uncertain counts the
// pairs decided on the host.
int srm_sample_device(const scarf_srm_params& p, const scarf_srm_setup& s, float* table, long long* pairs_used,
                      void* stream, long long* uncertain);
// srm_sample_device for many fields at once: the first pass of every field
// runs in one count launch and one write launch, then the host walks the
// fields one by one (further passes per field only if needed). Tables are
// bit-identical to srm_sample_device's. Returns 0; -1 - f if field f is
// infeasible; -2 - nfields on a CUDA error.
int srm_sample_device_batch(int nfields, const scarf_srm_params* p, const scarf_srm_setup* s, float* const* tables,
                            int* kept, long long* pairs_used, void* stream, long long* uncertain);
// Certain-reject thresholds of the device scan, one per bin of the first
// draw's raw output (bin = y1 >> kRejectShift, kRejectBins entries; both
// constants in srm_kernels.h beside SamplerArgs): a pair whose second raw draw
// y2 is at least thr[bin] fails the decision r2 < d(u) (1 + margin) for every
// u that the bin's r1 values give, so the scan drops it without evaluating
// the spectrum. thr[bin] bounds the spectrum's exact maximum over the bin's u
// interval (it is unimodal: x^(ndim-1) psd(x) peaks at x^2 = (ndim-1) /
// (2 nu - ndim + 1) for von Karman, 2 (ndim-1) for Gaussian) with 1e-4
// relative and 1e-30 absolute room for the device's FP32 evaluation;
// 0xFFFFFFFF = never.
void sampler_reject_thresholds(const scarf_srm_setup& s, int acf, float margin, uint32_t* thr);
// Relative band around the decision r2 < d in which the device leaves a pair
// to the host: device and host spectra differ by a few ulps at most.
constexpr float kSamplerMargin = 2e-5f;

// Upper bound on the pairs tested per device pass (0 = sized from the
// acceptance rate); smaller passes are chained until every harmonic is drawn.
void set_device_sampler_pass_cap(long long pairs);

int host_threads();

// Device allocations of the library's own buffers (tables, staging fields,
// scratch), counted over all devices against the cap that
// scarf_set_device_memory_cap sets (0: none). device_alloc returns a
// cudaError_t value: cudaErrorMemoryAllocation when the request would pass
// the cap, without calling the driver.
int device_alloc(void** p, size_t bytes);
void device_free(void* p, size_t bytes);
void set_device_memory_cap(size_t bytes);
size_t device_memory_in_use();
// Whether a device_alloc on the calling thread ran out of memory (or into
// the cap) since the last call; clears the flag.
bool take_device_alloc_failure();
// Frees the device sampler's scratch buffers (they grow again on demand).
void release_sampler_device_memory();

// Runs fn(0) .. fn(ntasks - 1) on at most `width` host threads (the caller's
// included) from a persistent worker pool; returns when all have returned.
void parallel_tasks(int ntasks, int width, const std::function<void(int)>& fn);

}  // namespace scarf
