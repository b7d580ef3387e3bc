// The YARN2 uniform source on the device: the order-2 multiple recursive
// generator modulo m = 2^31 - 1 (multipliers 1498809829, 1160990996; the
// parameters TRNG publishes for trng::yarn2, which prng.cpp:60 instantiates),
// its output transform g^t mod m (g = 123567893) and the float draw. Shared by
// the harmonic sampler (srm_sampler.cu) and the FIM spectrum (fim.cu); each
// translation unit keeps its own copy of the output transform's tables.
//
// The output transform g^t mod m is evaluated from three tables of exact
// residues, g^(t & 2047) * g^(((t >> 11) & 2047) * 2^11) * g^((t >> 22) * 2^22),
// which the kernels hold in shared memory (Gen::sp).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace scarf {
namespace yarn2 {

constexpr uint64_t kMod = 2147483647ull;
constexpr uint64_t kA1 = 1498809829ull;
constexpr uint64_t kA2 = 1160990996ull;

constexpr int kPow0 = 2048, kPow1 = 2048, kPow2 = 512;  // t < 2^31
constexpr int kPowWords = kPow0 + kPow1 + kPow2;

__device__ __forceinline__ uint64_t mulmod(uint64_t a, uint64_t b) {
  uint64_t p = a * b;  // < 2^62
  p = (p & kMod) + (p >> 31);
  p = (p & kMod) + (p >> 31);
  return p >= kMod ? p - kMod : p;
}
// x mod m for x < 2m + 2 (unsigned wrap-around makes x - m huge when x < m).
__device__ __forceinline__ uint32_t sub_m(uint32_t x) { return min(x, x - static_cast<uint32_t>(kMod)); }
// a * b mod m for a, b < 2^31, in 32-bit operations: the 62-bit product
// hi:lo folds once into (p >> 31) + (p & m) < 2^32 - 1, then at most two
// subtractions of m.
__device__ __forceinline__ uint32_t mulmod32(uint32_t a, uint32_t b) {
  const uint32_t lo = a * b, hi = __umulhi(a, b);
  const uint32_t f = __funnelshift_l(lo, hi, 1) + (lo & static_cast<uint32_t>(kMod));
  return sub_m(sub_m(f));
}
// g^u mod m from the three table residues t0 t1 t2 (each < m): the first
// product folds once at bit 31 and stays unreduced (< 2^32); the second,
// < 2^63, folds into a 33-bit sum, folds again (< 2^31 + 4) and takes one
// subtraction of m. Two instructions fewer than two full mulmod32.
__device__ __forceinline__ uint32_t mulmod3(uint32_t t0, uint32_t t1, uint32_t t2) {
  uint32_t lo = t0 * t1, hi = __umulhi(t0, t1);
  const uint32_t f = __funnelshift_l(lo, hi, 1) + (lo & static_cast<uint32_t>(kMod));  // < 2^32
  lo = f * t2;
  hi = __umulhi(f, t2);
  const uint64_t s = static_cast<uint64_t>(__funnelshift_l(lo, hi, 1)) + (lo & static_cast<uint32_t>(kMod));
  return sub_m(static_cast<uint32_t>(s & kMod) + static_cast<uint32_t>(s >> 31));
}
__device__ __forceinline__ uint64_t addmod(uint64_t a, uint64_t b) {
  const uint64_t s = a + b;
  return s >= kMod ? s - kMod : s;
}

struct Gen {
  uint64_t r0, r1;
  const uint32_t* sp;  // shared-memory power tables
  __device__ __forceinline__ uint32_t next() {
    // a1 r0 + a2 r1 < 2^63 as one 64-bit sum of two wide 32-bit products,
    // folded at bit 31 twice (< 2^32 + 2^31, then < 2^31 + 2), then at most
    // one subtraction of m.
    const uint64_t t = static_cast<uint64_t>(static_cast<uint32_t>(kA1)) * static_cast<uint32_t>(r0) +
                       static_cast<uint64_t>(static_cast<uint32_t>(kA2)) * static_cast<uint32_t>(r1);
    const uint64_t f = (t & kMod) + (t >> 31);
    const uint32_t u = sub_m(static_cast<uint32_t>(f & kMod) + static_cast<uint32_t>(f >> 31));
    r1 = r0;
    r0 = u;
    // The state 0 outputs 0; the power is formed regardless (no branch).
    const uint32_t y = mulmod3(sp[u & 2047u], sp[kPow0 + ((u >> 11) & 2047u)], sp[kPow0 + kPow1 + (u >> 22)]);
    return u == 0 ? 0u : y;
  }
  __device__ __forceinline__ void jump(uint64_t n) {
    uint64_t m00 = kA1, m01 = kA2, m10 = 1, m11 = 0;
    uint64_t p00 = 1, p01 = 0, p10 = 0, p11 = 1;
    while (n) {
      if (n & 1) {
        const uint64_t q00 = addmod(mulmod(p00, m00), mulmod(p01, m10));
        const uint64_t q01 = addmod(mulmod(p00, m01), mulmod(p01, m11));
        const uint64_t q10 = addmod(mulmod(p10, m00), mulmod(p11, m10));
        const uint64_t q11 = addmod(mulmod(p10, m01), mulmod(p11, m11));
        p00 = q00, p01 = q01, p10 = q10, p11 = q11;
      }
      const uint64_t s00 = addmod(mulmod(m00, m00), mulmod(m01, m10));
      const uint64_t s01 = addmod(mulmod(m00, m01), mulmod(m01, m11));
      const uint64_t s10 = addmod(mulmod(m10, m00), mulmod(m11, m10));
      const uint64_t s11 = addmod(mulmod(m10, m01), mulmod(m11, m11));
      m00 = s00, m01 = s01, m10 = s10, m11 = s11;
      n >>= 1;
    }
    const uint64_t n0 = addmod(mulmod(p00, r0), mulmod(p01, r1));
    const uint64_t n1 = addmod(mulmod(p10, r0), mulmod(p11, r1));
    r0 = n0;
    r1 = n1;
  }
};

// The host's Yarn2::to_u01: y * (1/m) in double, rounded to float.
__device__ __forceinline__ float to_u01(uint32_t y) {
  return __double2float_rn(__dmul_rn(static_cast<double>(y), 0x1.00000002p-31));
}

}  // namespace yarn2
}  // namespace scarf
