// Field statistics, rescaling and tapering on the device.
//
// The reference computes, on the host and in FP64 (scarflib_common.f90):
//   mean     = running mean of the FP32 field, returned as FP32   (:780-817)
//   variance = (s2 - s1^2/n)/(n-1) with x - mu, mu the FP32 mean,
//              returned as FP32                                   (:694-737)
// Here both passes are FP64 sums over the field in a fixed, deterministic
// tree order (per-block partials, then one block); results are rounded to
// FP32 exactly where the reference rounds them.
#include <cuda_runtime.h>

#include <cstdint>

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

__global__ void rescale_kernel(float* f, long long n, float scaling, float mean) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    f[i] = __fsub_rn(__fmul_rn(f[i], scaling), mean);
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

__global__ void taper_structured_kernel(float* f, int n0, int n1, long long npts, int o0, int o1, int o2, float dh,
                                        float p0, float p1, float p2, float mute, float taper) {
  const float dsum = __fadd_rn(mute, taper);
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long plane = static_cast<long long>(n0) * n1;
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < npts; p += stride) {
    const int k = static_cast<int>(p / plane);
    const long long rem = p - k * plane;
    const int j = static_cast<int>(rem / n0);
    const int i = static_cast<int>(rem - static_cast<long long>(j) * n0);
    // ((i - 1) * dh - poi)^2 with the global 1-based index i.
    float dx = __fsub_rn(__fmul_rn(static_cast<float>(i + o0), dh), p0);
    float dy = __fsub_rn(__fmul_rn(static_cast<float>(j + o1), dh), p1);
    float dz = __fsub_rn(__fmul_rn(static_cast<float>(k + o2), dh), p2);
    dx = __fmul_rn(dx, dx);
    dy = __fmul_rn(dy, dy);
    dz = __fmul_rn(dz, dz);
    const float d = __fsqrt_rn(__fadd_rn(__fadd_rn(dx, dy), dz));
    f[p] = taper_value(f[p], d, mute, taper, dsum);
  }
}

__global__ void taper_points_kernel(float* f, const float* x, const float* y, const float* z, long long n, float p0,
                                    float p1, float p2, float mute, float taper) {
  const float dsum = __fadd_rn(mute, taper);
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float ex = __fsub_rn(x[i], p0), ey = __fsub_rn(y[i], p1), ez = __fsub_rn(z[i], p2);
    const float d = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez)));
    f[i] = taper_value(f[i], d, mute, taper, dsum);
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

cudaError_t launch_rescale(float* d_field, long long n, float sigma, float std_, float mean, cudaStream_t stream) {
  const float scaling = sigma / std_;  // scarflib_srm.f90:899, FP32 on the host
  rescale_kernel<<<elementwise_blocks(n), 256, 0, stream>>>(d_field, n, scaling, mean);
  return cudaGetLastError();
}

cudaError_t launch_taper_structured(float* d_field, const int fs[3], const int n[3], float dh, const float poi[3],
                                    float mute, float taper, cudaStream_t stream) {
  const long long npts = static_cast<long long>(n[0]) * n[1] * n[2];
  taper_structured_kernel<<<elementwise_blocks(npts), 256, 0, stream>>>(
      d_field, n[0], n[1], npts, fs[0] - 1, fs[1] - 1, fs[2] - 1, dh, poi[0], poi[1], poi[2], mute, taper);
  return cudaGetLastError();
}

cudaError_t launch_taper_points(float* d_field, const float* d_x, const float* d_y, const float* d_z, long long n,
                                const float poi[3], float mute, float taper, cudaStream_t stream) {
  taper_points_kernel<<<elementwise_blocks(n), 256, 0, stream>>>(d_field, d_x, d_y, d_z, n, poi[0], poi[1], poi[2],
                                                                  mute, taper);
  return cudaGetLastError();
}

}  // namespace scarf
