// FIM (Fourier integral method) on one GPU: the reference's other algorithm
// (scarflib_fim.f90:141-1104), with the decomposition over MPI processes
// collapsed to one device.
//
//   1. spectrum     (compute_spectrum, :2390-2547): on the internal grid of
//      n1 x n2 x n3 points, a random phase per point drawn from the uniform
//      stream in x-fastest order (prng.cpp:67-124: one draw per point, block
//      split by jumps) and the amplitude sqrt(const * psd(k)); only the half
//      i <= n1/2 that the c2r transform along x reads is formed. One warp per
//      run of rows along x: lane l takes the points i = l + 32 t, its
//      generator jumped to its first draw through a table of matrix powers
//      and advanced by A^32 between draws (coalesced stores).
//   2. Hermitian planes i = 0 and i = n1/2 (enforce_symmetry, :2660-3007),
//      including the row k = 0 of 3-D grids that the reference conjugates in
//      place instead of mirroring (its exchange sends only one of two
//      subarrays; see fim_symmetry_kernel).
//   3. inverse transform (:1705-2315): c2c along z and y (FFTW_BACKWARD, no
//      normalisation), then c2r along x, by cuFFT; the imaginary parts of the
//      x bins 0 and n1/2, which a c2r transform does not use, are cleared
//      before it so that every c2r implementation reads the same input.
//   4. scaling by 1 / sqrt(n1 n2 n3 dh^n) (:1019), with per-block statistics
//      records of the scaled values (the mean/variance of the internal grid,
//      :1027-1036), merged in record order.
//   5. rescale and taper on the internal grid (:1038-1070) in one pass.
//   6. each external point takes the value of its nearest internal node
//      (grid_mapping / order_points / interpolate, :1110-1699, 3086-3162),
//      with exchange_halo's halo (:3013-3080): zero below the grid along x
//      and y, periodic along z.
// The rotation of the reference's DIP build option is not applied: the
// default build ignores the rotation angles on this path.
#include <cuda_runtime.h>
#include <cufft.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "srm_host.h"
#include "srm_kernels.h"
#include "yarn2.cuh"

namespace scarf {
namespace {

using namespace yarn2;

constexpr float kPiF = 3.14159265358979323846f;  // scarflib_common.f90:94, nearest float
constexpr int kJumpBits = 48;                     // draw indices below 2^48
constexpr int kRowsPerWarp = 8;

__device__ uint32_t g_fim_pow[kPowWords];
// c_jump[b] = A^(2^b), c_lane[l] = A^(l + 1), c_step = A^32; each row-major
// {a, b, c, d} for [[a, b], [c, d]] acting on the state (r0, r1).
__constant__ uint64_t c_jump[kJumpBits][4];
__constant__ uint64_t c_lane[32][4];
__constant__ uint64_t c_step[4];

struct State {
  uint64_t r0, r1;
};

__device__ __forceinline__ State apply(const uint64_t* M, State s) {
  return State{addmod(mulmod(M[0], s.r0), mulmod(M[1], s.r1)), addmod(mulmod(M[2], s.r0), mulmod(M[3], s.r1))};
}

struct SpecArgs {
  int n1, n2, n3, n1h;
  float dk1, dk2, dk3, kc, nu, cnst, cl1, cl2, cl3;
  int filter, acf;
  uint64_t s0, s1;        // state after seeding
  uint64_t row_step[4];   // A^n1: one row of draws
  float2* spec;           // [n3][n2][n1h]
};

// Wavenumber of 0-based index t on an axis of n points (the reference's
// [0 .. n/2, n/2 - 1 .. 1] * dk).
__device__ __forceinline__ float axis_k(int t, int n, float dk) {
  return __fmul_rn(static_cast<float>(t <= n / 2 ? t : n - t), dk);
}

__global__ void __launch_bounds__(256) fim_spectrum_kernel(const SpecArgs A) {
  __shared__ uint32_t sp[kPowWords];
  for (int i = threadIdx.x; i < kPowWords; i += blockDim.x) sp[i] = g_fim_pow[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long warp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long rows = static_cast<long long>(A.n2) * A.n3;
  const long long r0 = warp * kRowsPerWarp;
  if (r0 >= rows) return;
  // State at the first draw of this lane in row r0: A^(r0 n1) then A^(l + 1).
  State st{A.s0, A.s1};
  const unsigned long long skip = static_cast<unsigned long long>(r0) * A.n1;
  for (int b = 0; b < kJumpBits; ++b)
    if ((skip >> b) & 1ull) st = apply(c_jump[b], st);
  st = apply(c_lane[lane], st);
  const float pi2 = 2.0f;
  for (long long r = r0; r < r0 + kRowsPerWarp && r < rows; ++r) {
    const int k = static_cast<int>(r / A.n2);
    const int j = static_cast<int>(r - static_cast<long long>(k) * A.n2);
    const float ky = axis_k(j, A.n2, A.dk2), kz = axis_k(k, A.n3, A.dk3);
    const float kyy = __fmul_rn(ky, ky), kzz = __fmul_rn(kz, kz);
    const float ay = __fmul_rn(ky, A.cl2), az = __fmul_rn(kz, A.cl3);
    const float ayy = __fmul_rn(ay, ay), azz = __fmul_rn(az, az);
    State s = st;
    float2* out = A.spec + r * A.n1h;
    for (int i = lane; i < A.n1h; i += 32) {
      const uint32_t x = static_cast<uint32_t>(s.r0);
      const uint32_t y = x == 0 ? 0u
                                : mulmod3(sp[x & 2047u], sp[kPow0 + ((x >> 11) & 2047u)], sp[kPow0 + kPow1 + (x >> 22)]);
      const float u = to_u01(y);
      const float kx = __fmul_rn(static_cast<float>(i), A.dk1);  // i <= n1/2 on the half grid
      const float kr = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(kx, kx), kyy), kzz));
      const float butter = (A.filter && kr > A.kc) ? 0.0f : 1.0f;
      const float ax = __fmul_rn(kx, A.cl1);
      const float kr2 = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ax, ax), ayy), azz));
      float fv;
      if (A.acf == 0)
        fv = __fdiv_rn(1.0f, powf(__fadd_rn(1.0f, __fmul_rn(kr2, kr2)), A.nu));
      else
        fv = expf(__fmul_rn(-0.25f, __fmul_rn(kr2, kr2)));
      const float amp = __fmul_rn(__fsqrt_rn(__fmul_rn(A.cnst, fv)), butter);
      const float h = __fmul_rn(__fmul_rn(u, pi2), kPiF);
      float sn, cs;
      sincosf(h, &sn, &cs);
      out[i] = make_float2(__fmul_rn(cs, amp), __fmul_rn(sn, amp));
      s = apply(c_step, s);
    }
    st = apply(A.row_step, st);
  }
}

// Hermitian planes i = 0 and i = n1/2 of the half spectrum. Per plane:
// (0,0) becomes 0 (plane 0) or real (plane n1/2); (q2,q3), (0,q3), (q2,0)
// become real; then every point with k > q3, or k in {0, q3} and j > q2,
// takes the conjugate of its mirror (n2 - j, n3 - k) -- except the row k = 0
// of a 3-D grid, which exchange_conjg leaves unmirrored (one process gets
// both of its subarray types in one sendtypes slot and sends only the j = 1
// column, :2880-2967), so its points are only conjugated. Mirrors never fall
// on written or special points, so one pass in place is exact.
__global__ void fim_symmetry_kernel(float2* spec, int n1, int n2, int n3) {
  const int n1h = n1 / 2 + 1, q2 = n2 / 2, q3 = n3 / 2;
  const long long per_plane = static_cast<long long>(n2) * n3;
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= 2 * per_plane) return;
  const int plane = static_cast<int>(t / per_plane);
  const int i = plane == 0 ? 0 : n1 / 2;
  if (plane == 1 && n1 / 2 == 0) return;
  const long long r = t - plane * per_plane;
  const int k = static_cast<int>(r / n2), j = static_cast<int>(r - static_cast<long long>(k) * n2);
  float2* at = spec + (static_cast<long long>(k) * n2 + j) * n1h + i;
  if (j == 0 && k == 0) {
    if (i == 0)
      *at = make_float2(0.0f, 0.0f);
    else
      at->y = 0.0f;
    return;
  }
  if ((j == q2 && k == q3) || (j == 0 && k == q3) || (j == q2 && k == 0)) {
    at->y = 0.0f;
    return;
  }
  const bool w = (k > q3) || ((k == 0 || k == q3) && j > q2);
  if (!w) return;
  int jm = (n2 - j) % n2;
  const int km = (n3 - k) % n3;
  if (k == 0 && n3 > 1) jm = j;
  const float2 src = spec[(static_cast<long long>(km) * n2 + jm) * n1h + i];
  *at = make_float2(src.x, -src.y);
}

// The x bins 0 and n1/2 after the z/y transforms: imaginary parts cleared.
__global__ void fim_clear_imag_kernel(float2* spec, int n1h, long long rows, int last) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= 2 * rows) return;
  const long long r = t >> 1;
  const int i = (t & 1) ? last : 0;
  spec[r * n1h + i].y = 0.0f;
}

// Scaling of the transform's real output, with one statistics record per
// block (count, mean, M2 of the scaled values, FP64). A block covers
// kScaleThreads * kScaleRun values as kScaleRun / 4 coalesced float4 sweeps;
// each thread sums its values about its first one before the warp and block
// merges (a fixed order, so the records are deterministic).
constexpr int kScaleRun = 16;
constexpr int kScaleThreads = 256;

__global__ void __launch_bounds__(kScaleThreads) fim_scale_kernel(float* f, long long n, float scaling, Moments* rec) {
  __shared__ Moments s_warp[kScaleThreads / 32];
  const long long base = static_cast<long long>(blockIdx.x) * kScaleThreads * kScaleRun;
  double cnt = 0.0, s1 = 0.0, s2 = 0.0, shift = 0.0;
  bool have = false;
  auto take = [&](float v) {
    if (!have) {
      shift = v;
      have = true;
    }
    const double d = static_cast<double>(v) - shift;
    s1 += d;
    s2 = fma(d, d, s2);
    cnt += 1.0;
  };
#pragma unroll
  for (int q = 0; q < kScaleRun / 4; ++q) {
    const long long p = base + (static_cast<long long>(q) * kScaleThreads + threadIdx.x) * 4;
    if (p + 4 <= n) {
      float4 v = *reinterpret_cast<const float4*>(f + p);
      v.x = __fmul_rn(v.x, scaling);
      v.y = __fmul_rn(v.y, scaling);
      v.z = __fmul_rn(v.z, scaling);
      v.w = __fmul_rn(v.w, scaling);
      *reinterpret_cast<float4*>(f + p) = v;
      take(v.x);
      take(v.y);
      take(v.z);
      take(v.w);
    } else {
      for (long long e = p; e < n && e < p + 4; ++e) {
        const float v = __fmul_rn(f[e], scaling);
        f[e] = v;
        take(v);
      }
    }
  }
  Moments mo = warp_moments(moments_from_shifted(cnt, shift, s1, s2));
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = mo;
  __syncthreads();
  if (threadIdx.x == 0) {
    Moments b = s_warp[0];
    for (int w = 1; w < kScaleThreads / 32; ++w) b = moments_merge(b, s_warp[w]);
    rec[blockIdx.x] = b;
  }
}

struct MapArgs {
  int n1, n2, n3;       // internal grid
  float dh;
  float o1, o2, o3;     // off_axis
  const float* delta;   // internal field, x fastest
  // structured external grid (x null): fs - 1 and extents, step ds
  int f1, f2, f3, e1, e2;
  float ds;
  const float *x, *y, *z;
  float* field;
  long long n;
};

// Nearest internal node of one external point: NINT of (P / dh + 3) - 1 in
// the reference's 1-based index space of delta(0:n1, 0:n2, 0:n3), 0 = halo.
__device__ __forceinline__ float map_value(const MapArgs& A, float px, float py, float pz) {
  const float fi = __fsub_rn(__fadd_rn(__fdiv_rn(px, A.dh), 3.0f), 1.0f);
  const float fj = __fsub_rn(__fadd_rn(__fdiv_rn(py, A.dh), 3.0f), 1.0f);
  const float fk = __fsub_rn(__fadd_rn(__fdiv_rn(pz, A.dh), 3.0f), 1.0f);
  if (!(fi >= 1.0f && fi < static_cast<float>(A.n1 + 1) && fj >= 1.0f && fj < static_cast<float>(A.n2 + 1) &&
        fk >= 1.0f && fk < static_cast<float>(A.n3 + 1)))
    return 0.0f;
  const int a = static_cast<int>(roundf(fi)) - 1, b = static_cast<int>(roundf(fj)) - 1;
  int c = static_cast<int>(roundf(fk)) - 1;
  if (a == 0 || b == 0) return 0.0f;  // halo below x and y: zero (no neighbour)
  if (c == 0) c = A.n3;               // halo below z: the last plane (periodic)
  return A.delta[(a - 1) + static_cast<long long>(A.n1) * ((b - 1) + static_cast<long long>(A.n2) * (c - 1))];
}

// Point sets: one thread per point.
__global__ void fim_map_points_kernel(const MapArgs A) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.n; p += stride)
    A.field[p] = map_value(A, __fsub_rn(A.x[p], A.o1), __fsub_rn(A.y[p], A.o2), __fsub_rn(A.z[p], A.o3));
}

// Structured grids: blocks along x, rows (j, k) over blockIdx.y; each row's
// y and z coordinates are computed once, x per thread.
__global__ void fim_map_grid_kernel(const MapArgs A, int rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.e1) return;
  const float px = __fsub_rn(__fmul_rn(static_cast<float>(A.f1 + i), A.ds), A.o1);
  for (int row = blockIdx.y; row < rows; row += gridDim.y) {
    const int k = row / A.e2, j = row - k * A.e2;
    const float py = __fsub_rn(__fmul_rn(static_cast<float>(A.f2 + j), A.ds), A.o2);
    const float pz = __fsub_rn(__fmul_rn(static_cast<float>(A.f3 + k), A.ds), A.o3);
    A.field[static_cast<long long>(row) * A.e1 + i] = map_value(A, px, py, pz);
  }
}

// ------------------------------------------------------------------ host --
// Fortran NINT: nearest integer, halves away from zero.
int nint(float x) { return static_cast<int>(std::lround(x)); }

struct Mat {
  uint64_t v[4];
};
Mat mat_mul(const Mat& x, const Mat& y) {
  auto mm = Yarn2::mulmod;
  auto add = [](uint64_t a, uint64_t b) {
    const uint64_t s = a + b;
    return s >= Yarn2::kMod ? s - Yarn2::kMod : s;
  };
  return Mat{{add(mm(x.v[0], y.v[0]), mm(x.v[1], y.v[2])), add(mm(x.v[0], y.v[1]), mm(x.v[1], y.v[3])),
              add(mm(x.v[2], y.v[0]), mm(x.v[3], y.v[2])), add(mm(x.v[2], y.v[1]), mm(x.v[3], y.v[3]))}};
}
Mat mat_pow(Mat a, unsigned long long n) {
  Mat r{{1, 0, 0, 1}};
  while (n) {
    if (n & 1) r = mat_mul(r, a);
    a = mat_mul(a, a);
    n >>= 1;
  }
  return r;
}
const Mat kStepMat{{Yarn2::kA1, Yarn2::kA2, 1, 0}};

// cuFFT, loaded on first use so that the library itself does not depend on it.
struct Cufft {
  bool tried = false, ok = false;
  cufftResult (*plan_many)(cufftHandle*, int, int*, int*, int, int, int*, int, int, cufftType, int) = nullptr;
  cufftResult (*set_stream)(cufftHandle, cudaStream_t) = nullptr;
  cufftResult (*exec_c2c)(cufftHandle, cufftComplex*, cufftComplex*, int) = nullptr;
  cufftResult (*exec_c2r)(cufftHandle, cufftComplex*, cufftReal*) = nullptr;
  cufftResult (*destroy)(cufftHandle) = nullptr;
};
Cufft g_cufft;

bool load_cufft() {
  if (g_cufft.tried) return g_cufft.ok;
  g_cufft.tried = true;
  void* h = dlopen("libcufft.so.11", RTLD_NOW | RTLD_LOCAL);
  if (!h) h = dlopen("libcufft.so", RTLD_NOW | RTLD_LOCAL);
  if (!h) return false;
  g_cufft.plan_many = reinterpret_cast<decltype(g_cufft.plan_many)>(dlsym(h, "cufftPlanMany"));
  g_cufft.set_stream = reinterpret_cast<decltype(g_cufft.set_stream)>(dlsym(h, "cufftSetStream"));
  g_cufft.exec_c2c = reinterpret_cast<decltype(g_cufft.exec_c2c)>(dlsym(h, "cufftExecC2C"));
  g_cufft.exec_c2r = reinterpret_cast<decltype(g_cufft.exec_c2r)>(dlsym(h, "cufftExecC2R"));
  g_cufft.destroy = reinterpret_cast<decltype(g_cufft.destroy)>(dlsym(h, "cufftDestroy"));
  g_cufft.ok = g_cufft.plan_many && g_cufft.set_stream && g_cufft.exec_c2c && g_cufft.exec_c2r && g_cufft.destroy;
  return g_cufft.ok;
}

std::mutex g_fim_mu;
int g_fim_tables_dev = -1;
unsigned long long g_fim_tables_ctx = 0;

// The two cuFFT plans of the last internal grid transformed on each device,
// kept across calls: building a plan (kernel selection and the allocation of
// its work area) takes far longer than the transforms. Plans belong to the
// device context they were made in; after a reset (a new context id) the old
// handles are dropped, not destroyed. Guarded by g_fim_mu.
struct FimPlans {
  unsigned long long ctx = 0;
  int n1 = 0, n2 = 0, n3 = 0, three = -1;
  cufftHandle yz = 0, x = 0;
};
constexpr int kPlanDevices = 64;
FimPlans g_fim_plans[kPlanDevices];

void destroy_plans(FimPlans& p) {
  if (p.yz) g_cufft.destroy(p.yz);
  if (p.x) g_cufft.destroy(p.x);
  p = FimPlans();
}

}  // namespace

// Frees the cached cuFFT plans (and their work areas) of the current device.
void release_fim_plans() {
  std::lock_guard<std::mutex> lk(g_fim_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= kPlanDevices) {
    (void)cudaGetLastError();
    return;
  }
  FimPlans& P = g_fim_plans[dev];
  if (P.yz && P.ctx == current_context_id() && g_cufft.ok) destroy_plans(P);
  P = FimPlans();
}

namespace {

// The generator tables in this module's device and constant memory, uploaded
// once per device context (a reset context has a new id; when the id cannot
// be read they are uploaded on every call).
cudaError_t ensure_fim_tables() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long ctx = current_context_id();
  if (dev == g_fim_tables_dev && ctx != 0 && ctx == g_fim_tables_ctx) return cudaSuccess;
  static const std::vector<uint32_t> pw = device_pow_tables();
  e = cudaMemcpyToSymbol(g_fim_pow, pw.data(), sizeof(uint32_t) * pw.size());
  if (e != cudaSuccess) return e;
  uint64_t jump[kJumpBits][4], lane[32][4], step[4];
  Mat p = kStepMat;
  for (int b = 0; b < kJumpBits; ++b) {
    std::memcpy(jump[b], p.v, sizeof(p.v));
    p = mat_mul(p, p);
  }
  Mat q = kStepMat;
  for (int l = 0; l < 32; ++l) {
    std::memcpy(lane[l], q.v, sizeof(q.v));
    q = mat_mul(q, kStepMat);
  }
  std::memcpy(step, mat_pow(kStepMat, 32).v, sizeof(step));
  if ((e = cudaMemcpyToSymbol(c_jump, jump, sizeof(jump))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_lane, lane, sizeof(lane))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_step, step, sizeof(step))) != cudaSuccess) return e;
  g_fim_tables_dev = dev;
  g_fim_tables_ctx = current_context_id();
  return cudaSuccess;
}

int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return static_cast<int>(std::max(1LL, std::min(b, 148LL * 32)));
}

}  // namespace

void fim_grid(const FimInputs& in, FimGrid* g) {
  const float dh = in.dh;
  for (int i = 0; i < 3; ++i) {
    const float span = ((in.fc[i] + dh * 0.5f) - in.nc[i]) + dh * 0.5f;
    int n = nint(span / dh) + 1;
    int offset = nint(in.cl[i] / dh);
    if (in.pad != 1) offset = 0;
    n = n + 2 * offset;
    if (n % 2 != 0) n = n + 1;
    float off = in.nc[i] - (static_cast<float>(offset) + 0.5f) * dh;
    if (in.ndim == 2 && i == 2) {
      off = -off;
      n = 1;
    }
    g->npts[i] = n;
    g->off_axis[i] = off;
  }
  g->info0 = g->info1 = 0.0f;
  for (int i = 0; i < in.ndim; ++i) {
    if (g->npts[i] <= nint(2.0f * kPiF * in.cl[i] / dh)) g->info0 = 1.0f;
    if (dh > in.cl[i] / 2.0f) g->info1 = 1.0f;
  }
}

namespace {
size_t align256(size_t v) { return (v + 255) / 256 * 256; }
struct FimLayout {
  size_t off_spec, off_real, off_rec, off_poi, off_out, bytes;
  long long n1h, rows, real, nrec;
};
FimLayout fim_layout(const FimGrid& g, int npoi) {
  FimLayout L{};
  L.n1h = g.npts[0] / 2 + 1;
  L.rows = static_cast<long long>(g.npts[1]) * g.npts[2];
  L.real = static_cast<long long>(g.npts[0]) * L.rows;
  L.nrec = (L.real + kScaleThreads * kScaleRun - 1) / (kScaleThreads * kScaleRun);
  size_t off = 0;
  L.off_spec = off;
  off = align256(off + sizeof(float2) * static_cast<size_t>(L.n1h * L.rows));
  L.off_real = off;
  off = align256(off + sizeof(float) * static_cast<size_t>(L.real));
  L.off_rec = off;
  off = align256(off + sizeof(StatRecord) * static_cast<size_t>(L.nrec));
  L.off_poi = off;
  off = align256(off + sizeof(float) * 3 * static_cast<size_t>(std::max(npoi, 1)));
  L.off_out = off;  // mean, variance
  off = align256(off + 2 * sizeof(float));
  L.bytes = off;
  return L;
}
}  // namespace

size_t fim_workspace_bytes(const FimGrid& g, int npoi) { return fim_layout(g, npoi).bytes; }

cudaError_t fim_run(const FimInputs& in, const FimGrid& g, void* d_work, float* d_field, float stats[8],
                    cudaStream_t st, const char** what) {
  std::lock_guard<std::mutex> lk(g_fim_mu);
  auto failed = [&](const char* w, cudaError_t e) {
    *what = w;
    return e;
  };
  if (!load_cufft()) return failed("cuFFT (libcufft.so.11) could not be loaded", cudaErrorSharedObjectInitFailed);
  cudaError_t e = ensure_fim_tables();
  if (e != cudaSuccess) return failed("FIM generator tables", e);
  const int n1 = g.npts[0], n2 = g.npts[1], n3 = g.npts[2];
  const FimLayout L = fim_layout(g, in.npoi);
  uint8_t* w = static_cast<uint8_t*>(d_work);
  float2* spec = reinterpret_cast<float2*>(w + L.off_spec);
  float* real = reinterpret_cast<float*>(w + L.off_real);
  StatRecord* rec = reinterpret_cast<StatRecord*>(w + L.off_rec);
  float* d_poi = reinterpret_cast<float*>(w + L.off_poi);
  float* d_out = reinterpret_cast<float*>(w + L.off_out);

  cudaEvent_t ev[5] = {};
  for (auto& x : ev)
    if ((e = cudaEventCreate(&x)) != cudaSuccess) return failed("cudaEventCreate", e);
  struct EventsGuard {
    cudaEvent_t* ev;
    ~EventsGuard() {
      for (int i = 0; i < 5; ++i)
        if (ev[i]) cudaEventDestroy(ev[i]);
    }
  } eg{ev};

  // 1. spectrum on the half grid (compute_spectrum).
  SpecArgs A{};
  A.n1 = n1, A.n2 = n2, A.n3 = n3, A.n1h = static_cast<int>(L.n1h);
  float dk[3];
  for (int i = 0; i < 3; ++i) dk[i] = 2.0f * kPiF / (static_cast<float>(g.npts[i]) * in.dh);
  A.dk1 = dk[0], A.dk2 = dk[1], A.dk3 = dk[2];
  A.kc = kPiF / in.ds;
  A.filter = in.ds != in.dh;
  const float half_n = static_cast<float>(in.ndim) / 2.0f;
  A.nu = in.hurst + half_n;
  float prod = in.cl[0] * in.cl[1];
  if (in.ndim == 3) prod = prod * in.cl[2];
  if (in.acf == 0) {
    float c = static_cast<float>(1 << in.ndim) * std::pow(kPiF, half_n);
    c = c * std::tgamma(A.nu);
    c = c * (in.sigma * in.sigma);
    c = c * prod;
    A.cnst = c / std::tgamma(in.hurst);
  } else {
    A.cnst = (std::pow(kPiF, half_n) * (in.sigma * in.sigma)) * prod;
  }
  A.cl1 = in.cl[0], A.cl2 = in.cl[1], A.cl3 = in.cl[2];
  A.acf = in.acf;
  Yarn2 y;
  y.seed(in.seed);
  A.s0 = y.r0, A.s1 = y.r1;
  std::memcpy(A.row_step, mat_pow(kStepMat, static_cast<unsigned long long>(n1)).v, sizeof(A.row_step));
  A.spec = spec;
  cudaEventRecord(ev[0], st);
  const long long warps = (L.rows + kRowsPerWarp - 1) / kRowsPerWarp;
  fim_spectrum_kernel<<<static_cast<unsigned>((warps * 32 + 255) / 256), 256, 0, st>>>(A);
  if ((e = cudaGetLastError()) != cudaSuccess) return failed("fim_spectrum_kernel", e);
  cudaEventRecord(ev[1], st);
  // 2. Hermitian planes (enforce_symmetry).
  fim_symmetry_kernel<<<static_cast<unsigned>((2 * L.rows + 255) / 256), 256, 0, st>>>(spec, n1, n2, n3);
  if ((e = cudaGetLastError()) != cudaSuccess) return failed("fim_symmetry_kernel", e);
  cudaEventRecord(ev[2], st);
  // 3. inverse transform: c2c along z and y (x bins as the batch), the
  // unused imaginary parts of x bins 0 and n1/2 cleared, c2r along x.
  const int n1h = static_cast<int>(L.n1h);
  const bool three = in.ndim == 3 && n3 > 1;
  // The plans: this device's cached pair when the grid matches, else new
  // ones (cached for the next call; on devices beyond the cache, freed on
  // return).
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return failed("cudaGetDevice", e);
  const unsigned long long ctx = current_context_id();
  const bool cacheable = dev < kPlanDevices && ctx != 0;
  FimPlans local;
  FimPlans& P = cacheable ? g_fim_plans[dev] : local;
  struct LocalGuard {
    FimPlans* p;
    ~LocalGuard() { destroy_plans(*p); }
  } lg{&local};
  if (cacheable && P.ctx != ctx) P = FimPlans();  // handles of a reset context are dropped
  if (P.yz && !(P.n1 == n1 && P.n2 == n2 && P.n3 == n3 && P.three == (three ? 1 : 0))) destroy_plans(P);
  if (!P.yz) {
    FimPlans fresh;
    struct FreshGuard {
      FimPlans* p;
      bool keep = false;
      ~FreshGuard() {
        if (!keep) destroy_plans(*p);
      }
    } fg{&fresh};
    int dims3[2] = {n3, n2}, dims2[1] = {n2};
    int* dims = three ? dims3 : dims2;
    const int rank = three ? 2 : 1;
    if (g_cufft.plan_many(&fresh.yz, rank, dims, dims, n1h, 1, dims, n1h, 1, CUFFT_C2C, n1h) != CUFFT_SUCCESS)
      return failed("cufftPlanMany (z, y)", cudaErrorUnknown);
    int dx[1] = {n1}, ex[1] = {n1h}, ox[1] = {n1};
    if (g_cufft.plan_many(&fresh.x, 1, dx, ex, 1, n1h, ox, 1, n1, CUFFT_C2R, static_cast<int>(L.rows)) !=
        CUFFT_SUCCESS)
      return failed("cufftPlanMany (x)", cudaErrorUnknown);
    fresh.ctx = ctx;
    fresh.n1 = n1, fresh.n2 = n2, fresh.n3 = n3, fresh.three = three ? 1 : 0;
    P = fresh;
    fg.keep = true;
  }
  const cufftHandle p_yz = P.yz, p_x = P.x;
  {
    if (g_cufft.set_stream(p_yz, st) != CUFFT_SUCCESS || g_cufft.set_stream(p_x, st) != CUFFT_SUCCESS)
      return failed("cufftSetStream", cudaErrorUnknown);
    cufftComplex* c = reinterpret_cast<cufftComplex*>(spec);
    if (g_cufft.exec_c2c(p_yz, c, c, CUFFT_INVERSE) != CUFFT_SUCCESS) return failed("cufftExecC2C", cudaErrorUnknown);
    fim_clear_imag_kernel<<<static_cast<unsigned>((2 * L.rows + 255) / 256), 256, 0, st>>>(spec, n1h, L.rows, n1 / 2);
    if ((e = cudaGetLastError()) != cudaSuccess) return failed("fim_clear_imag_kernel", e);
    if (g_cufft.exec_c2r(p_x, c, real) != CUFFT_SUCCESS) return failed("cufftExecC2R", cudaErrorUnknown);
  }
  cudaEventRecord(ev[3], st);
  // 4. scaling 1 / sqrt(n1 n2 n3 dh^n) and statistics of the internal grid.
  const float dhn = in.ndim == 2 ? in.dh * in.dh : (in.dh * in.dh) * in.dh;
  const float scaling = 1.0f / std::sqrt(((static_cast<float>(n1) * static_cast<float>(n2)) * static_cast<float>(n3)) *
                                         dhn);
  fim_scale_kernel<<<static_cast<unsigned>(L.nrec), kScaleThreads, 0, st>>>(real, L.real, scaling, rec);
  if ((e = cudaGetLastError()) != cudaSuccess) return failed("fim_scale_kernel", e);
  if ((e = launch_stats_records(rec, L.nrec, d_out, st)) != cudaSuccess) return failed("statistics", e);
  float mv[2];
  if ((e = cudaMemcpyAsync(mv, d_out, sizeof(mv), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return failed("statistics copy", e);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return failed("FIM transform", e);
  stats[0] = g.info0;
  stats[1] = g.info1;
  stats[2] = std::sqrt(mv[1]);
  stats[3] = mv[0];
  // 5. rescale and taper on the internal grid.
  std::vector<float> pt;
  if (in.rescale == 1 || in.npoi > 0) {
    FinalizeArgs fa{};
    if (in.rescale == 1) {
      fa.rescale = 1;
      fa.scaling = in.sigma / stats[2];
      fa.mean = stats[3];
      stats[2] = in.sigma;
      stats[3] = 0.0f;
    }
    if (in.npoi > 0) {
      pt.assign(3 * static_cast<size_t>(in.npoi), 0.0f);
      for (int q = 0; q < in.npoi; ++q)
        for (int c = 0; c < in.ndim; ++c) pt[3 * q + c] = in.poi[in.poi_stride * q + c] - g.off_axis[c];
      if ((e = cudaMemcpyAsync(d_poi, pt.data(), sizeof(float) * pt.size(), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess)
        return failed("POI copy", e);
      fa.d_poi = d_poi;
      fa.npoi = in.npoi;
      fa.mute = in.mute;
      fa.taper = in.taper;
      fa.n0 = n1;
      fa.n1 = n2;
      fa.dh = in.dh;
    }
    if ((e = launch_finalize_field(real, L.real, fa, st)) != cudaSuccess) return failed("rescale/taper", e);
  }
  // 6. external points from their nearest internal nodes.
  MapArgs M{};
  M.n1 = n1, M.n2 = n2, M.n3 = n3;
  M.dh = in.dh;
  M.o1 = g.off_axis[0], M.o2 = g.off_axis[1], M.o3 = g.off_axis[2];
  M.delta = real;
  M.field = d_field;
  if (in.structured) {
    M.f1 = in.fs[0] - 1, M.f2 = in.fs[1] - 1, M.f3 = in.fs[2] - 1;
    M.e1 = in.fe[0] - in.fs[0] + 1, M.e2 = in.fe[1] - in.fs[1] + 1;
    M.ds = in.ds;
    M.n = static_cast<long long>(M.e1) * M.e2 * (in.fe[2] - in.fs[2] + 1);
  } else {
    M.x = in.d_x, M.y = in.d_y, M.z = in.d_z;
    M.n = in.npts;
  }
  if (in.structured) {
    const int rows = M.e2 * (in.fe[2] - in.fs[2] + 1);
    const dim3 grid((M.e1 + 127) / 128, static_cast<unsigned>(std::min(rows, 65535)));
    fim_map_grid_kernel<<<grid, 128, 0, st>>>(M, rows);
  } else {
    fim_map_points_kernel<<<blocks_for(M.n, 256), 256, 0, st>>>(M);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return failed("fim_map kernels", e);
  cudaEventRecord(ev[4], st);
  if ((e = cudaEventSynchronize(ev[4])) != cudaSuccess) return failed("FIM mapping", e);
  float ms[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
  // info(5:8) of the reference's TIMING build: spectrum, symmetry, transform
  // (here with scaling, statistics, rescale and taper), mapping.
  stats[4] = ms[0] * 1e-3f;
  stats[5] = ms[1] * 1e-3f;
  stats[6] = ms[2] * 1e-3f;
  stats[7] = ms[3] * 1e-3f;
  return cudaSuccess;
}

}  // namespace scarf
