// FP32 direct-sum SRM kernels (the "plain" form): for every point,
//   field = scaling * sum_h [ a_h sin(arg_h) + b_h cos(arg_h) ],
//   arg_h = v1*P1 + v2*P2 + v3*P3,  P = M x + bar,
// evaluated in the reference's operation order without FMA contraction
// (scarflib_srm.f90:794-809 structured, :397-406 points, :843-851 scaling).
// The rotated coordinates P are loop invariant in the reference, so they are
// computed once per point; the harmonic table streams through shared memory
// in tiles moved by 1-D bulk (TMA) copies, double-buffered on mbarriers,
// and every thread reads four table rows at a time with five 16-byte loads.
#include <cuda_runtime.h>

#include "common.cuh"
#include "srm_kernels.h"

namespace scarf {
namespace {

constexpr int kTile = 256;           // harmonics per shared-memory tile
constexpr int kRow = 5;              // floats per table row {v1,v2,v3,a,b}
// Points per thread: 8 (two float4 stores) with the SFU sin/cos; 4 with
// CUDA's sincosf, whose slow path needs the registers (8 would spill).
template <bool kFast>
constexpr int points_per_thread() { return kFast ? 8 : 4; }
constexpr int kThreads = 128;
constexpr uint32_t kTileBytes = kTile * kRow * 4;  // 5120, multiple of 16

struct DirectArgs {
  float m[9];
  float bar[3];
  float scaling;
  int nh;
  const float* table;  // device, nh x 5
  float* field;
  long long npts;
  int* status;
  // structured
  int n0, n1;
  float ds;
  int off0, off1, off2;  // fs - 2 (so x = (i1 + off) * ds with 1-based i1)
  // points
  const float* x;
  const float* y;
  const float* z;
  // optional: one statistics record per block (count, mean, M2 of its stored values)
  Moments* stats;
};

__device__ __forceinline__ void rotate(const DirectArgs& A, float x, float y, float z, float& p1, float& p2,
                                       float& p3) {
  // ((m1 x + m2 y) + m3 z) + bar, each operation rounded (no contraction).
  p1 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(A.m[0], x), __fmul_rn(A.m[1], y)), __fmul_rn(A.m[2], z)), A.bar[0]);
  p2 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(A.m[3], x), __fmul_rn(A.m[4], y)), __fmul_rn(A.m[5], z)), A.bar[1]);
  p3 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(A.m[6], x), __fmul_rn(A.m[7], y)), __fmul_rn(A.m[8], z)), A.bar[2]);
}

// sin and cos of an FP32 phase, two ways.
// Accurate (kFast = false): CUDA's sincosf, correctly rounded to ~1 ulp with
// full range reduction. Fast (default): the phase reduced to [-pi, pi] by
// Cody-Waite's method (Cody & Waite, "Software Manual for the Elementary
// Functions", 1980) with 2 pi split into two floats C1 + C2 (the residual,
// 6.9e-15, times |j| < 2^22 stays below 3e-8), each product applied by one
// FMA, then the SFU's __sinf/__cosf, whose absolute error on [-pi, pi] is
// about 2^-21.4. C1 has 24 significant bits, so arg - j C1 is exact (a
// multiple of 2^-21 below 2^2 in magnitude, or Sterbenz's case for |j| = 1);
// only the C2 step rounds. For the
// phases here (|arg| < 1e4 rad) the reduced argument is within ~2.5e-7 of
// exact, so each term is within ~6e-7 absolute, and fields agree with the
// FP32 restatement (glibc sinf/cosf) to ~4e-7 of their standard deviation.
// (Phases up to 2^22 * 2 pi = 2.6e7 rad; the FP32 phase itself carries an
// error of several radians long before that.)
constexpr float kInv2Pi = 0x1.45f306p-3f;
constexpr float kTwoPi1 = 0x1.921fb6p+2f;
constexpr float kTwoPi2 = -0x1.777a5cp-23f;

// Nearest integer of arg / (2 pi) for |arg / (2 pi)| < 2^22 on the FMA pipe:
// one FMA adds 1.5 * 2^23 to the exact product (rounding it to an integer,
// nearest even) and a subtraction removes it. rintf itself would issue on
// the SFU's pipe, which __sinf and __cosf already saturate here. Near a
// half-integer either neighbour may be chosen; both leave |r| <= pi + 3e-7.
constexpr float kRoundMagic = 0x1.8p23f;

template <bool kFast>
__device__ __forceinline__ void phase_sincos(float arg, float* sn, float* cs) {
  if constexpr (kFast) {
    const float j = __fsub_rn(__fmaf_rn(arg, kInv2Pi, kRoundMagic), kRoundMagic);
    float r = fmaf(-j, kTwoPi1, arg);
    r = fmaf(-j, kTwoPi2, r);
    *sn = __sinf(r);
    *cs = __cosf(r);
  } else {
    sincosf(arg, sn, cs);
  }
}

template <bool kStructured, bool kFast>
__global__ void __launch_bounds__(kThreads) srm_direct_kernel(const DirectArgs A) {
  constexpr int kPts = points_per_thread<kFast>();
  __shared__ __align__(128) float s_tab[2][kTile * kRow];
  __shared__ __align__(8) uint64_t s_full[2];

  const int tid = threadIdx.x;
  const long long p0 = (static_cast<long long>(blockIdx.x) * kThreads + tid) * kPts;

  // Rotated coordinates of this thread's points (loop invariant).
  float P1[kPts], P2[kPts], P3[kPts], acc[kPts];
#pragma unroll
  for (int q = 0; q < kPts; ++q) {
    const long long p = p0 + q < A.npts ? p0 + q : A.npts - 1;
    float x, y, z;
    if constexpr (kStructured) {
      const long long plane = static_cast<long long>(A.n0) * A.n1;
      const int k = static_cast<int>(p / plane);
      const long long rem = p - static_cast<long long>(k) * plane;
      const int j = static_cast<int>(rem / A.n0);
      const int i = static_cast<int>(rem - static_cast<long long>(j) * A.n0);
      // x = (i + fs(1) - 2) * ds with the 1-based index i+1.
      x = __fmul_rn(static_cast<float>(i + 1 + A.off0), A.ds);
      y = __fmul_rn(static_cast<float>(j + 1 + A.off1), A.ds);
      z = __fmul_rn(static_cast<float>(k + 1 + A.off2), A.ds);
    } else {
      x = __ldg(A.x + p);
      y = __ldg(A.y + p);
      z = __ldg(A.z + p);
    }
    rotate(A, x, y, z, P1[q], P2[q], P3[q]);
    acc[q] = 0.0f;
  }

  const int nfull = A.nh / kTile;            // tiles moved by bulk copy
  const int tail = A.nh - nfull * kTile;     // rows of the last tile
  const int ntiles = nfull + (tail ? 1 : 0);
  const bool aligned = (reinterpret_cast<uintptr_t>(A.table) & 15u) == 0;

  if (tid == 0) {
    mbar_init(&s_full[0], 1);
    mbar_init(&s_full[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int issued = 0;  // bulk copies issued so far (meaningful in thread 0)
  if (tid == 0 && aligned) {
    for (int t = 0; t < 2 && t < nfull; ++t) {
      mbar_arrive_expect_tx(&s_full[t], kTileBytes);
      bulk_g2s(s_tab[t], A.table + static_cast<size_t>(t) * kTile * kRow, kTileBytes, &s_full[t]);
      ++issued;
    }
  }

  bool ok = true;
  int t = 0;
  for (; t < ntiles; ++t) {
    const int buf = t & 1;
    int rows = kTile;
    if (t < nfull && aligned) {
      if (!mbar_wait_bounded(&s_full[buf], (t >> 1) & 1, A.status)) ok = false;
    } else {
      // Unaligned table or the partial last tile: cooperative plain loads.
      rows = (t < nfull) ? kTile : tail;
      const float* src = A.table + static_cast<size_t>(t) * kTile * kRow;
      for (int e = tid; e < rows * kRow; e += kThreads) s_tab[buf][e] = __ldg(src + e);
      __syncthreads();
    }
    if (!__syncthreads_and(ok)) break;  // all threads agree before consuming
    const float* tb = s_tab[buf];
    auto harmonic = [&](float v1, float v2, float v3, float a, float b) {
#pragma unroll
      for (int q = 0; q < kPts; ++q) {
        const float arg = __fadd_rn(__fadd_rn(__fmul_rn(v1, P1[q]), __fmul_rn(v2, P2[q])), __fmul_rn(v3, P3[q]));
        float sn, cs;
        phase_sincos<kFast>(arg, &sn, &cs);
        acc[q] = __fadd_rn(__fadd_rn(acc[q], __fmul_rn(a, sn)), __fmul_rn(b, cs));
      }
    };
    // Four rows (20 floats, 80 bytes from a 16-byte aligned tile) per step.
    int h = 0;
    for (; h + 4 <= rows; h += 4) {
      const float4* g4 = reinterpret_cast<const float4*>(tb + h * kRow);
      const float4 q0 = g4[0], q1 = g4[1], q2 = g4[2], q3 = g4[3], q4 = g4[4];
      harmonic(q0.x, q0.y, q0.z, q0.w, q1.x);
      harmonic(q1.y, q1.z, q1.w, q2.x, q2.y);
      harmonic(q2.z, q2.w, q3.x, q3.y, q3.z);
      harmonic(q3.w, q4.x, q4.y, q4.z, q4.w);
    }
    for (; h < rows; ++h) harmonic(tb[h * kRow + 0], tb[h * kRow + 1], tb[h * kRow + 2], tb[h * kRow + 3], tb[h * kRow + 4]);
    __syncthreads();  // buffer `buf` fully consumed
    if (tid == 0 && aligned && t + 2 < nfull) {
      mbar_arrive_expect_tx(&s_full[buf], kTileBytes);
      bulk_g2s(s_tab[buf], A.table + static_cast<size_t>(t + 2) * kTile * kRow, kTileBytes, &s_full[buf]);
      ++issued;
    }
  }
  if (!ok) {
    // Drain the copies still in flight into this block's shared memory
    // (tiles t .. issued-1) before the block exits; each wait is bounded.
    if (tid == 0) {
      for (int u = t; u < issued; ++u) mbar_wait_drain(&s_full[u & 1], (u >> 1) & 1);
    }
    return;
  }

  // Normalise (field * scaling) and store.
  float out[kPts];
#pragma unroll
  for (int q = 0; q < kPts; ++q) out[q] = __fmul_rn(acc[q], A.scaling);
  float* dst = A.field + p0;
  if (p0 + kPts <= A.npts && (reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
#pragma unroll
    for (int q = 0; q < kPts; q += 4)
      *reinterpret_cast<float4*>(dst + q) = make_float4(out[q], out[q + 1], out[q + 2], out[q + 3]);
  } else {
#pragma unroll
    for (int q = 0; q < kPts; ++q)
      if (p0 + q < A.npts) dst[q] = out[q];
  }
  if (A.stats) {
    // Statistics of the stored values (FP64): thread, warp (fixed tree), then
    // the block's warps in order; one record per block.
    __shared__ Moments s_warp[kThreads / 32];
    double s1 = 0.0, s2 = 0.0, cnt = 0.0;
    const double shift = p0 < A.npts ? static_cast<double>(out[0]) : 0.0;
#pragma unroll
    for (int q = 0; q < kPts; ++q) {
      if (p0 + q < A.npts) {
        const double d = static_cast<double>(out[q]) - shift;
        s1 += d;
        s2 = fma(d, d, s2);
        cnt += 1.0;
      }
    }
    Moments m = warp_moments(moments_from_shifted(cnt, shift, s1, s2));
    if ((tid & 31) == 0) s_warp[tid >> 5] = m;
    __syncthreads();
    if (tid == 0) {
      Moments b = s_warp[0];
      for (int w = 1; w < kThreads / 32; ++w) b = moments_merge(b, s_warp[w]);
      A.stats[blockIdx.x] = b;
    }
  }
}

}  // namespace

int g_direct_fast = 1;

void direct_set_sincos(int fast) { g_direct_fast = fast ? 1 : 0; }
int direct_get_sincos() { return g_direct_fast; }

int direct_points_per_thread() { return g_direct_fast ? points_per_thread<true>() : points_per_thread<false>(); }

long long direct_stat_records(long long npts) {
  const long long per_block = static_cast<long long>(kThreads) * direct_points_per_thread();
  return (npts + per_block - 1) / per_block;
}

cudaError_t launch_direct_structured(const scarf_srm_setup& s, const int fs[3], const int n[3], float ds,
                                     const float* d_table, int nh, float* d_field, int* d_status,
                                     cudaStream_t stream, StatRecord* d_stats) {
  DirectArgs A{};
  for (int i = 0; i < 9; ++i) A.m[i] = s.m[i];
  for (int i = 0; i < 3; ++i) A.bar[i] = s.bar[i];
  A.scaling = s.scaling;
  A.nh = nh;
  A.table = d_table;
  A.field = d_field;
  A.npts = static_cast<long long>(n[0]) * n[1] * n[2];
  A.status = d_status;
  A.n0 = n[0];
  A.n1 = n[1];
  A.ds = ds;
  A.off0 = fs[0] - 2;
  A.off1 = fs[1] - 2;
  A.off2 = fs[2] - 2;
  A.stats = d_stats;
  const long long per_block = static_cast<long long>(kThreads) * direct_points_per_thread();
  const long long blocks = (A.npts + per_block - 1) / per_block;
  if (blocks <= 0) return cudaSuccess;
  if (g_direct_fast)
    srm_direct_kernel<true, true><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(A);
  else
    srm_direct_kernel<true, false><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_direct_points(const scarf_srm_setup& s, const float* d_x, const float* d_y, const float* d_z,
                                 long long npts, const float* d_table, int nh, float* d_field, int* d_status,
                                 cudaStream_t stream, StatRecord* d_stats) {
  DirectArgs A{};
  for (int i = 0; i < 9; ++i) A.m[i] = s.m[i];
  for (int i = 0; i < 3; ++i) A.bar[i] = s.bar[i];
  A.scaling = s.scaling;
  A.nh = nh;
  A.table = d_table;
  A.field = d_field;
  A.npts = npts;
  A.status = d_status;
  A.x = d_x;
  A.y = d_y;
  A.z = d_z;
  A.stats = d_stats;
  const long long per_block = static_cast<long long>(kThreads) * direct_points_per_thread();
  const long long blocks = (npts + per_block - 1) / per_block;
  if (blocks <= 0) return cudaSuccess;
  if (g_direct_fast)
    srm_direct_kernel<false, true><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(A);
  else
    srm_direct_kernel<false, false><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace scarf
