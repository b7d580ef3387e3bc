// Field statistics, rescaling and tapering on the device.
//
// The reference computes, on the host and in FP64 (scarflib_common.f90):
//   mean     = running mean of the FP32 field, returned as FP32   (:780-817)
//   variance = (s2 - s1^2/n)/(n-1) with x - mu, mu the FP32 mean,
//              returned as FP32                                   (:694-737)
// scarf_execute takes them from per-tile (count, mean, M2) records that the
// summation kernels write as they store the field, merged here in record
// order (Chan's pairwise formula, FP64); scarf_field_stats and fields
// without harmonics take two FP64 passes over the field in a fixed tree
// order (per-block partials, then one block). Results are rounded to FP32
// exactly where the reference rounds them. Rescale and taper run as one pass.
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "srm_kernels.h"

namespace scarf {
namespace {

constexpr int kStatThreads = 512;
constexpr int kStatBlocks = 1184;  // 148 SMs x 8, fixed so the order is fixed

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  v = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

// Pass 1 (mu == nullptr): partial sums of x. Pass 2: partial sums of
// d = x - mu and d^2, mu read from the device (double of the FP32 mean).
__global__ void __launch_bounds__(kStatThreads) stats_partials(const float* __restrict__ f, long long n,
                                                               const double* __restrict__ mu, double* part) {
  __shared__ double red[kStatThreads / 32];
  const bool second = mu != nullptr;
  const double m = second ? *mu : 0.0;
  double s1 = 0.0, s2 = 0.0;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  // Vectorised body when the base is 16-byte aligned.
  if ((reinterpret_cast<uintptr_t>(f) & 15u) == 0) {
    const long long n4 = n / 4;
    const float4* f4 = reinterpret_cast<const float4*>(f);
    for (long long q = i; q < n4; q += stride) {
      const float4 v = __ldg(f4 + q);
      const double d0 = (double)v.x - m, d1 = (double)v.y - m, d2 = (double)v.z - m, d3 = (double)v.w - m;
      s1 += (d0 + d1) + (d2 + d3);
      if (second) s2 += (d0 * d0 + d1 * d1) + (d2 * d2 + d3 * d3);
    }
    for (long long q = 4 * n4 + i; q < n; q += stride) {
      const double d = (double)__ldg(f + q) - m;
      s1 += d;
      if (second) s2 += d * d;
    }
  } else {
    for (long long q = i; q < n; q += stride) {
      const double d = (double)__ldg(f + q) - m;
      s1 += d;
      if (second) s2 += d * d;
    }
  }
  s1 = block_sum(s1, red);
  if (second) s2 = block_sum(s2, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
}

// Single block: reduce the partials, then either publish the FP32 mean (as
// a double in mu_out) or the FP32 mean/variance pair in out.
__global__ void __launch_bounds__(1024) stats_finish(const double* part, int nparts, long long n, double* mu_io,
                                                      float* out, int second) {
  __shared__ double red[32];
  double s1 = 0.0, s2 = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    s1 += part[2 * b];
    s2 += part[2 * b + 1];
  }
  s1 = block_sum(s1, red);
  s2 = block_sum(s2, red);
  if (threadIdx.x == 0) {
    const double dn = static_cast<double>(n);
    if (!second) {
      const float mean32 = static_cast<float>(s1 / dn);
      mu_io[0] = static_cast<double>(mean32);
      out[0] = mean32;
    } else {
      const double c1 = (s1 * s1) / dn;
      const double v = (s2 - c1) / static_cast<double>(n - 1);
      out[1] = static_cast<float>(v);
    }
  }
}

// One block merges the statistics records written by a summation kernel:
// thread t takes a contiguous run of records in order, then the threads'
// results are merged by a fixed tree in shared memory. FP64 throughout;
// mean and variance rounded to FP32 once, where the reference rounds them.
// The record merge gives the variance as M2 / (n - 1), which is the
// reference's compensated two-pass sum (s2 - s1^2 / n) / (n - 1) about the
// FP32 mean in exact arithmetic.
constexpr int kMergeThreads = 1024;

__global__ void __launch_bounds__(kMergeThreads) stats_records_merge(const Moments* __restrict__ rec, long long count,
                                                                      float* out) {
  __shared__ Moments red[kMergeThreads];
  const long long per = (count + kMergeThreads - 1) / kMergeThreads;
  const long long r0 = static_cast<long long>(threadIdx.x) * per;
  const long long r1 = r0 + per < count ? r0 + per : count;
  Moments m{0.0, 0.0, 0.0};
  for (long long r = r0; r < r1; ++r) m = moments_merge(m, rec[r]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = kMergeThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = moments_merge(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const Moments t = red[0];
    out[0] = static_cast<float>(t.mean);
    out[1] = static_cast<float>(t.m2 / (t.n - 1.0));
  }
}

__device__ __forceinline__ float taper_value(float f, float d, float mute, float taper, float dsum) {
  const float pi = 3.14159265358979323846f;
  if (d <= mute) return 0.0f;
  if (d > mute && d <= dsum) {
    const float t = __fdiv_rn(__fsub_rn(d, mute), taper);
    return __fmul_rn(f, __fsub_rn(0.5f, __fmul_rn(0.5f, cosf(__fmul_rn(t, pi)))));
  }
  return f;
}

// Rescale, then the taper of every point of interest in order, per point:
// the same operations, in the same order, as a rescale pass followed by one
// taper pass per point of interest.
__global__ void finalize_kernel(float* f, long long n, const FinalizeArgs a) {
  const float dsum = __fadd_rn(a.mute, a.taper);
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long plane = static_cast<long long>(a.n0) * a.n1;
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += stride) {
    float v = f[p];
    if (a.rescale) v = __fsub_rn(__fmul_rn(v, a.scaling), a.mean);
    if (a.npoi > 0) {
      float x, y, z;
      if (a.d_x) {
        x = a.d_x[p];
        y = a.d_y[p];
        z = a.d_z[p];
      } else {
        const int k = static_cast<int>(p / plane);
        const long long rem = p - k * plane;
        const int j = static_cast<int>(rem / a.n0);
        const int i = static_cast<int>(rem - static_cast<long long>(j) * a.n0);
        x = __fmul_rn(static_cast<float>(i + a.o0), a.dh);
        y = __fmul_rn(static_cast<float>(j + a.o1), a.dh);
        z = __fmul_rn(static_cast<float>(k + a.o2), a.dh);
      }
      for (int q = 0; q < a.npoi; ++q) {
        const float* pt = a.d_poi + 3 * q;
        float d;
        if (a.d_x) {
          const float ex = __fsub_rn(x, pt[0]), ey = __fsub_rn(y, pt[1]), ez = __fsub_rn(z, pt[2]);
          d = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez)));
        } else {
          float dx = __fsub_rn(x, pt[0]), dy = __fsub_rn(y, pt[1]), dz = __fsub_rn(z, pt[2]);
          dx = __fmul_rn(dx, dx);
          dy = __fmul_rn(dy, dy);
          dz = __fmul_rn(dz, dz);
          d = __fsqrt_rn(__fadd_rn(__fadd_rn(dx, dy), dz));
        }
        v = taper_value(v, d, a.mute, a.taper, dsum);
      }
    }
    f[p] = v;
  }
}

int elementwise_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<int>(b < 1 ? 1 : b);
}

}  // namespace

size_t stats_partials_bytes(long long) { return sizeof(double) * (2 * kStatBlocks + 2); }

cudaError_t launch_field_stats(const float* d_field, long long n, double* d_partials, float* d_out,
                               cudaStream_t stream) {
  double* mu = d_partials + 2 * kStatBlocks;
  stats_partials<<<kStatBlocks, kStatThreads, 0, stream>>>(d_field, n, nullptr, d_partials);
  stats_finish<<<1, 1024, 0, stream>>>(d_partials, kStatBlocks, n, mu, d_out, 0);
  stats_partials<<<kStatBlocks, kStatThreads, 0, stream>>>(d_field, n, mu, d_partials);
  stats_finish<<<1, 1024, 0, stream>>>(d_partials, kStatBlocks, n, mu, d_out, 1);
  return cudaGetLastError();
}

cudaError_t launch_stats_records(const StatRecord* d_rec, long long count, float* d_out, cudaStream_t stream) {
  stats_records_merge<<<1, kMergeThreads, 0, stream>>>(d_rec, count, d_out);
  return cudaGetLastError();
}

cudaError_t launch_finalize_field(float* d_field, long long n, const FinalizeArgs& a, cudaStream_t stream) {
  finalize_kernel<<<elementwise_blocks(n), 256, 0, stream>>>(d_field, n, a);
  return cudaGetLastError();
}

}  // namespace scarf
