// Factorised tensor-core SRM for structured grids, single field or a batch of
// fields in one persistent launch.
//
// The phase of harmonic h at grid point (x, y, z) is linear in the
// coordinates (scarflib_srm.f90:802-804): arg = kx x + ky y + kz z + c with
// k' = M^T v and c = v . bar. Hence
//   a sin(arg) + b cos(arg) = Re[(b - i a) e^{i c} e^{i kx x} e^{i ky y} e^{i kz z}]
// and the field over an (i,j) x k block is a real contraction
//   F[(i,j), k] = sum_h  Re(P_h(i,j)) cos(kz z_k) - Im(P_h(i,j)) sin(kz z_k),
//   P_h(i,j) = R_h(i) S_h(j),  R_h(i) = (b - i a) e^{i (kx x_i + c)},  S_h(j) = e^{i ky y_j}.
// Per-axis factors are computed in FP64 (phases reach ~1e4 rad) and rounded to
// FP32. The A operand [128 rows x 2 nh] is generated in shared memory from the
// R and S factor tiles (complex multiply, 16-bit hi/lo split: BF16 by
// default, FP16 on request); the B operand [cos; sin](kz z) is pre-split into
// hi/lo images of the same type in global memory and staged by 1-D bulk
// copies. Three tcgen05 kind::f16 products (hi*hi, hi*lo, lo*hi) accumulate
// in FP32 in tensor memory.
//
// Work distribution: one persistent CTA per SM pulls work items (one 128-row
// x <=256-column output tile of one field) from a device work queue (an
// atomic counter over an item list sorted longest first); the producer warp
// fetches each item and broadcasts it to the other warp roles through a small
// shared-memory ring.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "srm_kernels.h"

namespace scarf {
namespace {

constexpr int kStageHarm = 16;                  // harmonics per pipeline stage (K = 32)
constexpr int kRows = 128;                      // M of one tile (one CTA)
constexpr int kRowBytes = 64;                   // 32 fp16 along K = one 64-B swizzle row
constexpr int kATileBytes = kRows * kRowBytes;  // 8 KB per hi or lo
#ifndef SCARF_TC_GEN_WARPS
#define SCARF_TC_GEN_WARPS 8
#endif
constexpr int kGenWarps = SCARF_TC_GEN_WARPS;   // A generators: 8 or 16
constexpr int kGenWarp0 = 8;                    // warps 8.. generate A (8 % 4 == 0: lane quadrants line up)
constexpr int kEpiWarp0 = 4;                    // warps 4..7 drain the accumulators
constexpr int kThreads = 32 * (kGenWarp0 + kGenWarps);
constexpr int kGenHarm = kStageHarm * 4 / kGenWarps;  // harmonics per generator thread and stage
static_assert(kGenWarps == 8 || kGenWarps == 16, "generator warps: 8 or 16");
constexpr int kItemRing = 4;                    // work items in flight between roles
constexpr int kItemConsumers = 1 + 4 + kGenWarps;  // MMA warp, epilogue warps, generator warps
constexpr uint32_t kSwizzle64 = 4;              // tcgen05 descriptor: 64-B swizzle

__host__ __device__ constexpr uint32_t swz64(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 512u + (row & 7u) * 64u + ((chunk ^ ((row & 7u) >> 1)) << 4);
}

// Split of two FP32 values into hi and lo 16-bit operands (hi = round(v),
// lo = round(v - hi)), packed as two 2-byte elements: FP16 (the default) or
// BF16 (the operand-precision setting; same layouts, same MMA kind).
template <bool kBf16>
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
  if constexpr (kBf16) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 f = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - f.x, b - f.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  } else {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 f = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - f.x, b - f.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
  }
}

// Operand pair type of the A image: FP16 or BF16 hi/lo halves.
template <bool kBf16>
struct OperandPair {
  using T2 = __half2;
  static __device__ __forceinline__ T2 pack(float a, float b) { return __floats2half2_rn(a, b); }
  static __device__ __forceinline__ float2 unpack(T2 v) { return __half22float2(v); }
};
template <>
struct OperandPair<true> {
  using T2 = __nv_bfloat162;
  static __device__ __forceinline__ T2 pack(float a, float b) { return __floats2bfloat162_rn(a, b); }
  static __device__ __forceinline__ float2 unpack(T2 v) { return __bfloat1622float2(v); }
};

// The A operand of kGenHarm harmonics for one row: the complex products
// R_h(i) S_h(j) (the conjugate's imaginary part, as the MMA sums re cos -
// im sin), split into hi/lo pairs. rt / stt: this row's R and S entries of
// the first harmonic, strided by the tiles' widths. The operand type is a
// compile-time choice: a run-time branch here costs the FP16 kernel ~4 %.
template <bool kBf16>
__device__ __forceinline__ void gen_products(const float2* rt, const float2* stt, int ti, int tj,
                                             typename OperandPair<kBf16>::T2* hv,
                                             typename OperandPair<kBf16>::T2* lv) {
  using Op = OperandPair<kBf16>;
#pragma unroll
  for (int u = 0; u < kGenHarm; ++u) {
    const float2 x = rt[u * ti];
    const float2 y = stt[u * tj];
    const float re = x.x * y.x - x.y * y.y;
    const float nim = -(x.x * y.y + x.y * y.x);
    hv[u] = Op::pack(re, nim);
    const float2 hf = Op::unpack(hv[u]);
    lv[u] = Op::pack(re - hf.x, nim - hf.y);
  }
}

// Geometry and table images of one field in the factorised form.
struct TcField {
  int n1, n2, n3;
  int bi, bj, ntile_n, stages, chunk_stages;
  int bix, bjx;         // item grid: bi x bj, or CTA pairs along j (bi x ceil(bj/2)) or i (ceil(bi/2) x bj)
  int bn;               // column tiles
  long long sr, ss, sc; // field strides (elements) of the i, j and k axes
  int pair_i;           // CTA pairs split along i (2D fields: one row block along j)
  int band;             // item order: row blocks along i per band (>= bix: natural order)
  int terms;            // split products per K step: 3 (hi.hi, hi.lo, lo.hi) or 2 (hi.hi, lo.hi)
  int bf16;             // operands split into BF16 instead of FP16
  uint32_t idesc;
  float scaling;
  const float2* rimg;   // [bi][stages][16][ti]
  const float2* simg;   // [bj][stages][16][tj]
  const uint8_t* cimg;  // [bn][stages][part][hi,lo][ntile_n / parts * 64 B]
  float* field;
  // Completion signal of a batch field (null when unused): every epilogue
  // warp of every item adds one to done_cnt after its last chunk; the
  // arrival that reaches done_expect sets the host-mapped done_flag.
  int* done_cnt;
  volatile int* done_flag;
  int done_expect;
  // Statistics records of the stored field (null when unused): one per
  // epilogue warp and item, at (local item * CTAs per item + CTA) * 4 + warp.
  Moments* stats;
  // Split of the harmonics (K) over `split` segments, each its own work item
  // (1: none). Segment s sums stages [s stages / split, (s + 1) stages /
  // split) and stores its unscaled partial sums at partial + s * seg_stride
  // (the field's layout); an ordered reduction then scales their sum.
  int split;
  float* partial;
  long long seg_stride;
};

struct TcKernelArgs {
  TcField f0;             // the field when `fields` is null
  int bf16;               // generators split A into BF16 (uniform over a launch)
  const TcField* fields;  // per-field descriptors of a batch
  const int2* items;      // {field, local item}, longest first; null: field 0 in natural order
  int num_items;
  int* queue;             // work-queue counter, zero at launch
  int* status;
  int ti, tj, ti_shift;   // row-tile shape (uniform over a launch)
  int nstage_buf;
  uint32_t stage_bytes, off_b, off_a, off_r, off_s, bars_off;
  // CTA-pair layout only: a separate ring of nrs factor-tile (R, S) slots.
  int nrs;
  uint32_t rs_base, rs_bytes;
  // Slab completion signal (single-field launches; null otherwise): a slab
  // is one column tile x a run of slab_jbs row blocks along j, contiguous
  // pieces of the field that the host copies out while the kernel runs.
  int* slab_cnt;            // device counters, zero at launch
  volatile int* slab_flag;  // host-mapped flags, set once a slab is stored
  int slab_jbs, slab_spn;   // row blocks per slab, slabs per column tile
};

// Per-field inputs of the table builders.
struct TableJob {
  const float* table;  // nh x {v1,v2,v3,a,b}
  int nh, stages;
  double m[9], bar[3];
  double ds;
  int off[3];            // coordinate of 0-based index t on axis a: (t + off[a]) * ds
  int ax_r, ax_s, ax_c;  // physical axis of the row-fast, row-slow and column factors
  int n1, n2, n3, ti, tj, bi, bj, ntile_n, bn;  // bj: S-image blocks (even for CTA pairs)
  int parts;             // column image split: 1, or 2 halves (one per CTA of a pair)
  int bf16;              // C image split into BF16 instead of FP16
  float2* rimg;
  float2* simg;
  uint8_t* cimg;
};

__device__ __forceinline__ void harmonic_k(const TableJob& T, int h, double k[3], double& c, double& a,
                                           double& b) {
  const float* r = T.table + 5 * static_cast<size_t>(h);
  const double v1 = r[0], v2 = r[1], v3 = r[2];
  // k'_col = sum_r v_r M[r][col]; c = sum_r v_r bar_r.
  for (int col = 0; col < 3; ++col) k[col] = v1 * T.m[col] + v2 * T.m[3 + col] + v3 * T.m[6 + col];
  c = v1 * T.bar[0] + v2 * T.bar[1] + v3 * T.bar[2];
  a = r[3];
  b = r[4];
}

// R image (the harmonic's complex amplitude and constant phase folded in) and
// S image; one thread per entry. blockIdx.y selects the field of a batch.
__global__ void tc_build_rs(const TableJob j0, const TableJob* jobs) {
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const long long nr = static_cast<long long>(T.bi) * T.stages * kStageHarm * T.ti;
  const long long ns = static_cast<long long>(T.bj) * T.stages * kStageHarm * T.tj;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nr + ns;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const bool is_r = e < nr;
    const long long q = is_r ? e : e - nr;
    const int tw = is_r ? T.ti : T.tj;
    const int t = static_cast<int>(q % tw);
    const long long q2 = q / tw;
    const int hp = static_cast<int>(q2 % kStageHarm);
    const long long q3 = q2 / kStageHarm;
    const int k = static_cast<int>(q3 % T.stages);
    const int blk = static_cast<int>(q3 / T.stages);
    const int h = k * kStageHarm + hp;
    const int idx = blk * tw + t;
    const int nlim = is_r ? T.n1 : T.n2;
    float2 out = make_float2(0.0f, 0.0f);
    if (h < T.nh && idx < nlim) {
      double kv[3], c, a, b;
      harmonic_k(T, h, kv, c, a, b);
      const int ax = is_r ? T.ax_r : T.ax_s;
      const double coord = static_cast<double>(idx + T.off[ax]) * T.ds;
      double sn, cs;
      if (is_r) {
        sincos(kv[ax] * coord + c, &sn, &cs);
        // (b - i a)(cos + i sin)
        out = make_float2(static_cast<float>(b * cs + a * sn), static_cast<float>(b * sn - a * cs));
      } else {
        sincos(kv[ax] * coord, &sn, &cs);
        out = make_float2(static_cast<float>(cs), static_cast<float>(sn));
      }
    }
    (is_r ? T.rimg : T.simg)[q] = out;
  }
}

// Column image: per (column block, stage) a 64-B-swizzled K-major tile of
// ntile_n rows x 32 fp16 ([cos, sin] of 16 harmonics), hi then lo.
template <bool kBf16>
__global__ void tc_build_c(const TableJob j0, const TableJob* jobs) {
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const long long nchunks = static_cast<long long>(T.bn) * T.stages * T.ntile_n * 4;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nchunks;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int chunk = static_cast<int>(e & 3);
    const long long q = e >> 2;
    const int row = static_cast<int>(q % T.ntile_n);
    const long long q2 = q / T.ntile_n;
    const int k = static_cast<int>(q2 % T.stages);
    const int nb = static_cast<int>(q2 / T.stages);
    const int col = nb * T.ntile_n + row;
    const int part_rows = T.ntile_n / T.parts;
    const int part = row / part_rows, prow = row - part * part_rows;
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int h = k * kStageHarm + chunk * 4 + u;
      float cs32 = 0.0f, sn32 = 0.0f;
      if (h < T.nh && col < T.n3) {
        double kv[3], c, a, b;
        harmonic_k(T, h, kv, c, a, b);
        const double coord = static_cast<double>(col + T.off[T.ax_c]) * T.ds;
        double sn, cs;
        sincos(kv[T.ax_c] * coord, &sn, &cs);
        cs32 = static_cast<float>(cs);
        sn32 = static_cast<float>(sn);
      }
      split_pair<kBf16>(cs32, sn32, hi[u], lo[u]);
    }
    uint8_t* base = T.cimg + ((static_cast<size_t>(nb) * T.stages + k) * T.parts + part) *
                                 (2u * part_rows * kRowBytes);
    const uint32_t off = swz64(static_cast<uint32_t>(prow), static_cast<uint32_t>(chunk));
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(base + static_cast<size_t>(part_rows) * kRowBytes + off) =
        *reinterpret_cast<const uint4*>(lo);
  }
}

// ---- factored table builders -------------------------------------------
// The same images with far fewer FP64 transcendentals: along an axis the
// phase of index t = 16 a + b splits as
//   k ((16 a + off) ds) + c  +  k (b ds),
// so e^{i phase} = U[a] V[b] with U, V built once per harmonic in shared
// memory (one sincos per 16 entries, plus 16), and every entry is one FP64
// complex product before its rounding to FP32. Used when the factor tables
// fit kFactorSmem of shared memory; otherwise the builders above run.
constexpr int kFactorSmem = 48 * 1024;

__device__ __forceinline__ double2 cmul(double2 x, double2 y) {
  return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}

__device__ __forceinline__ double2 expi(double th) {
  double s, c;
  sincos(th, &s, &c);
  return make_double2(c, s);
}

// R and S images: one block per harmonic at a time (grid-strided),
// blockIdx.y the field of a batch.
__global__ void tc_build_rs_factored(const TableJob j0, const TableJob* jobs) {
  extern __shared__ double2 fsh[];
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const int nr = T.bi * T.ti, ns = T.bj * T.tj;  // image widths (padded)
  const int nur = (nr + 15) / 16, nus = (ns + 15) / 16;
  double2* ur = fsh;
  double2* vr = ur + nur;
  double2* us = vr + 16;
  double2* vs = us + nus;
  const int nfac = nur + nus + 32;
  const double offr = T.off[T.ax_r], offs = T.off[T.ax_s];
  for (int h = blockIdx.x; h < T.stages * kStageHarm; h += gridDim.x) {
    const bool valid = h < T.nh;
    double kv[3] = {0.0, 0.0, 0.0}, c = 0.0, a = 0.0, b = 0.0;
    if (valid) harmonic_k(T, h, kv, c, a, b);
    const double kr = kv[T.ax_r], ks = kv[T.ax_s];
    __syncthreads();  // the previous harmonic's entries are written
    for (int e = threadIdx.x; e < nfac; e += blockDim.x) {
      if (e < nur) {
        ur[e] = expi(kr * ((16.0 * e + offr) * T.ds) + c);
      } else if (e < nur + 16) {
        vr[e - nur] = expi(kr * ((e - nur) * T.ds));
      } else if (e < nur + 16 + nus) {
        us[e - nur - 16] = expi(ks * ((16.0 * (e - nur - 16) + offs) * T.ds));
      } else {
        vs[e - nur - 16 - nus] = expi(ks * ((e - nur - 16 - nus) * T.ds));
      }
    }
    __syncthreads();
    const int k = h / kStageHarm, hp = h - k * kStageHarm;
    for (int e = threadIdx.x; e < nr + ns; e += blockDim.x) {
      const bool is_r = e < nr;
      const int idx = is_r ? e : e - nr;
      const int tw = is_r ? T.ti : T.tj;
      const int blk = idx / tw, t = idx - blk * tw;
      float2 out = make_float2(0.0f, 0.0f);
      if (valid && idx < (is_r ? T.n1 : T.n2)) {
        if (is_r) {
          const double2 z = cmul(ur[idx >> 4], vr[idx & 15]);
          // (b - i a)(cos + i sin)
          out = make_float2(static_cast<float>(b * z.x + a * z.y), static_cast<float>(b * z.y - a * z.x));
        } else {
          const double2 z = cmul(us[idx >> 4], vs[idx & 15]);
          out = make_float2(static_cast<float>(z.x), static_cast<float>(z.y));
        }
      }
      const size_t q = ((static_cast<size_t>(blk) * T.stages + k) * kStageHarm + hp) * tw + t;
      (is_r ? T.rimg : T.simg)[q] = out;
    }
  }
}

// Column image: one block per 4-harmonic chunk of a stage at a time
// (grid-strided), blockIdx.y the field of a batch.
template <bool kBf16>
__global__ void tc_build_c_factored(const TableJob j0, const TableJob* jobs) {
  extern __shared__ double2 fsh[];
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const int ncol = T.bn * T.ntile_n;
  const int nu = (ncol + 15) / 16;
  double2* u4 = fsh;          // [4][nu]
  double2* v4 = u4 + 4 * nu;  // [4][16]
  const double offc = T.off[T.ax_c];
  const int part_rows = T.ntile_n / T.parts;
  for (int j = blockIdx.x; j < T.stages * 4; j += gridDim.x) {
    const int k = j >> 2, chunk = j & 3;
    bool valid[4];
    double kc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int h = k * kStageHarm + chunk * 4 + u;
      valid[u] = h < T.nh;
      double kv[3] = {0.0, 0.0, 0.0}, c, a, b;
      if (valid[u]) harmonic_k(T, h, kv, c, a, b);
      kc[u] = kv[T.ax_c];
    }
    __syncthreads();  // the previous chunk's entries are written
    for (int e = threadIdx.x; e < 4 * (nu + 16); e += blockDim.x) {
      const int u = e / (nu + 16), r = e - u * (nu + 16);
      if (r < nu) u4[u * nu + r] = expi(kc[u] * ((16.0 * r + offc) * T.ds));
      else v4[u * 16 + (r - nu)] = expi(kc[u] * ((r - nu) * T.ds));
    }
    __syncthreads();
    for (int col = threadIdx.x; col < ncol; col += blockDim.x) {
      const int nb = col / T.ntile_n, row = col - nb * T.ntile_n;
      const int part = row / part_rows, prow = row - part * part_rows;
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float cs32 = 0.0f, sn32 = 0.0f;
        if (valid[u] && col < T.n3) {
          const double2 z = cmul(u4[u * nu + (col >> 4)], v4[u * 16 + (col & 15)]);
          cs32 = static_cast<float>(z.x);
          sn32 = static_cast<float>(z.y);
        }
        split_pair<kBf16>(cs32, sn32, hi[u], lo[u]);
      }
      uint8_t* base = T.cimg + ((static_cast<size_t>(nb) * T.stages + k) * T.parts + part) *
                                   (2u * part_rows * kRowBytes);
      const uint32_t off = swz64(static_cast<uint32_t>(prow), static_cast<uint32_t>(chunk));
      *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(part_rows) * kRowBytes + off) =
          *reinterpret_cast<const uint4*>(lo);
    }
  }
}

// The same factored builders with a warp, not a block, per harmonic (R/S)
// or per 4-harmonic chunk (C): each warp keeps its own factor tables and
// synchronises with __syncwarp only. Small fields have few entries per
// harmonic (a 64-point axis: 40 sincos and 128 entries), so a block per
// harmonic leaves most threads waiting at its two barriers; with a warp per
// harmonic four harmonics are in flight per block. Every entry is computed
// by the same FP64 operations as above, so the images are bit-identical.
constexpr int kBuilderWarps = 4;

__global__ void __launch_bounds__(32 * kBuilderWarps) tc_build_rs_warps(const TableJob j0, const TableJob* jobs) {
  extern __shared__ double2 fsh[];
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const int nr = T.bi * T.ti, ns = T.bj * T.tj;
  const int nur = (nr + 15) / 16, nus = (ns + 15) / 16;
  const int nfac = nur + nus + 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* ur = fsh + warp * nfac;
  double2* vr = ur + nur;
  double2* us = vr + 16;
  double2* vs = us + nus;
  const double offr = T.off[T.ax_r], offs = T.off[T.ax_s];
  for (int h = blockIdx.x * kBuilderWarps + warp; h < T.stages * kStageHarm; h += gridDim.x * kBuilderWarps) {
    const bool valid = h < T.nh;
    double kv[3] = {0.0, 0.0, 0.0}, c = 0.0, a = 0.0, b = 0.0;
    if (valid) harmonic_k(T, h, kv, c, a, b);
    const double kr = kv[T.ax_r], ks = kv[T.ax_s];
    __syncwarp();  // the previous harmonic's entries are written
    for (int e = lane; e < nfac; e += 32) {
      if (e < nur) {
        ur[e] = expi(kr * ((16.0 * e + offr) * T.ds) + c);
      } else if (e < nur + 16) {
        vr[e - nur] = expi(kr * ((e - nur) * T.ds));
      } else if (e < nur + 16 + nus) {
        us[e - nur - 16] = expi(ks * ((16.0 * (e - nur - 16) + offs) * T.ds));
      } else {
        vs[e - nur - 16 - nus] = expi(ks * ((e - nur - 16 - nus) * T.ds));
      }
    }
    __syncwarp();
    const int k = h / kStageHarm, hp = h - k * kStageHarm;
    for (int e = lane; e < nr + ns; e += 32) {
      const bool is_r = e < nr;
      const int idx = is_r ? e : e - nr;
      const int tw = is_r ? T.ti : T.tj;
      const int blk = idx / tw, t = idx - blk * tw;
      float2 out = make_float2(0.0f, 0.0f);
      if (valid && idx < (is_r ? T.n1 : T.n2)) {
        if (is_r) {
          const double2 z = cmul(ur[idx >> 4], vr[idx & 15]);
          out = make_float2(static_cast<float>(b * z.x + a * z.y), static_cast<float>(b * z.y - a * z.x));
        } else {
          const double2 z = cmul(us[idx >> 4], vs[idx & 15]);
          out = make_float2(static_cast<float>(z.x), static_cast<float>(z.y));
        }
      }
      const size_t q = ((static_cast<size_t>(blk) * T.stages + k) * kStageHarm + hp) * tw + t;
      (is_r ? T.rimg : T.simg)[q] = out;
    }
  }
}

template <bool kBf16>
__global__ void __launch_bounds__(32 * kBuilderWarps) tc_build_c_warps(const TableJob j0, const TableJob* jobs) {
  extern __shared__ double2 fsh[];
  const TableJob& T = jobs ? jobs[blockIdx.y] : j0;
  const int ncol = T.bn * T.ntile_n;
  const int nu = (ncol + 15) / 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2* u4 = fsh + warp * 4 * (nu + 16);  // [4][nu]
  double2* v4 = u4 + 4 * nu;                 // [4][16]
  const double offc = T.off[T.ax_c];
  const int part_rows = T.ntile_n / T.parts;
  for (int j = blockIdx.x * kBuilderWarps + warp; j < T.stages * 4; j += gridDim.x * kBuilderWarps) {
    const int k = j >> 2, chunk = j & 3;
    bool valid[4];
    double kc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int h = k * kStageHarm + chunk * 4 + u;
      valid[u] = h < T.nh;
      double kv[3] = {0.0, 0.0, 0.0}, c, a, b;
      if (valid[u]) harmonic_k(T, h, kv, c, a, b);
      kc[u] = kv[T.ax_c];
    }
    __syncwarp();  // the previous chunk's entries are written
    for (int e = lane; e < 4 * (nu + 16); e += 32) {
      const int u = e / (nu + 16), r = e - u * (nu + 16);
      if (r < nu) u4[u * nu + r] = expi(kc[u] * ((16.0 * r + offc) * T.ds));
      else v4[u * 16 + (r - nu)] = expi(kc[u] * ((r - nu) * T.ds));
    }
    __syncwarp();
    for (int col = lane; col < ncol; col += 32) {
      const int nb = col / T.ntile_n, row = col - nb * T.ntile_n;
      const int part = row / part_rows, prow = row - part * part_rows;
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float cs32 = 0.0f, sn32 = 0.0f;
        if (valid[u] && col < T.n3) {
          const double2 z = cmul(u4[u * nu + (col >> 4)], v4[u * 16 + (col & 15)]);
          cs32 = static_cast<float>(z.x);
          sn32 = static_cast<float>(z.y);
        }
        split_pair<kBf16>(cs32, sn32, hi[u], lo[u]);
      }
      uint8_t* base = T.cimg + ((static_cast<size_t>(nb) * T.stages + k) * T.parts + part) *
                                   (2u * part_rows * kRowBytes);
      const uint32_t off = swz64(static_cast<uint32_t>(prow), static_cast<uint32_t>(chunk));
      *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
      *reinterpret_cast<uint4*>(base + static_cast<size_t>(part_rows) * kRowBytes + off) =
          *reinterpret_cast<const uint4*>(lo);
    }
  }
}

// Shared memory of the factored builders for a plan (image widths as
// make_job sets them, padded to whole row blocks).
size_t factor_smem_rs(const TcPlan& p) {
  const int ni = p.pair_i ? 2 * p.bix : p.bi;
  const int nj = (p.pair && !p.pair_i) ? 2 * p.bjx : p.bj;
  return sizeof(double2) * (static_cast<size_t>((ni * p.ti + 15) / 16) + (nj * p.tj + 15) / 16 + 32);
}
size_t factor_smem_c(const TcPlan& p) {
  return sizeof(double2) * 4 * (static_cast<size_t>((p.bn * p.ntile_n + 15) / 16) + 16);
}

// Enqueues the R/S and C image builders for nfields fields (jobs == nullptr:
// the single field T) given their largest stage count and shared-memory
// needs. The factored builders walk harmonics one block at a time, each
// step latency-bound (a sincos and two barriers), so they get many small
// blocks: ~64 per SM over all fields.
// With `fork`, the C-image builder runs on fork->side beside the R/S builder
// (the two are independent: R/S are issue-bound FP64 work, C writes its
// images at a good share of HBM bandwidth) and `stream` joins it afterwards.
void launch_table_builders(const TableJob& T, const TableJob* jobs, int nfields, int max_stages, size_t smem_rs,
                           size_t smem_c, int nsm, cudaStream_t stream, bool bf16, const BuilderFork* fork = nullptr) {
  const bool forked = fork && fork->side && fork->fork && fork->join &&
                      cudaEventRecord(fork->fork, stream) == cudaSuccess &&
                      cudaStreamWaitEvent(fork->side, fork->fork, 0) == cudaSuccess;
  const cudaStream_t cs = forked ? fork->side : stream;
  const int per_field = std::max(1, nsm * 64 / std::max(1, nfields));
  const int grid_old = std::max(1, std::min(64, nsm * 8 / std::max(1, nfields)));
  // Builder form: warps while each warp's factor tables fit (default), else
  // blocks, else direct; SCARF3D_B200_TABLE_BUILDER=block|direct forces a
  // form (the forms are compared in tests).
  static const int forced = [] {
    const char* e = std::getenv("SCARF3D_B200_TABLE_BUILDER");
    if (!e) return 0;
    if (!std::strcmp(e, "block")) return 1;
    if (!std::strcmp(e, "direct")) return 2;
    return 0;
  }();
  const size_t warps_limit = static_cast<size_t>(kFactorSmem) / kBuilderWarps;
  if (forced == 0 && smem_rs <= warps_limit)
    tc_build_rs_warps<<<dim3(std::min((max_stages * kStageHarm + kBuilderWarps - 1) / kBuilderWarps, per_field),
                             nfields),
                        32 * kBuilderWarps, kBuilderWarps * smem_rs, stream>>>(T, jobs);
  else if (forced <= 1 && smem_rs <= static_cast<size_t>(kFactorSmem))
    tc_build_rs_factored<<<dim3(std::min(max_stages * kStageHarm, per_field), nfields), 128, smem_rs, stream>>>(
        T, jobs);
  else
    tc_build_rs<<<dim3(jobs ? grid_old : nsm * 8, nfields), 256, 0, stream>>>(T, jobs);
  // The C image's operand type (FP16 or BF16 hi/lo) is uniform over a launch.
  const dim3 g_warps(std::min((max_stages * 4 + kBuilderWarps - 1) / kBuilderWarps, per_field), nfields);
  const dim3 g_fact(std::min(max_stages * 4, per_field), nfields);
  const dim3 g_old(jobs ? grid_old : nsm * 8, nfields);
  if (forced == 0 && smem_c <= warps_limit) {
    if (bf16)
      tc_build_c_warps<true><<<g_warps, 32 * kBuilderWarps, kBuilderWarps * smem_c, cs>>>(T, jobs);
    else
      tc_build_c_warps<false><<<g_warps, 32 * kBuilderWarps, kBuilderWarps * smem_c, cs>>>(T, jobs);
  } else if (forced <= 1 && smem_c <= static_cast<size_t>(kFactorSmem)) {
    if (bf16)
      tc_build_c_factored<true><<<g_fact, 128, smem_c, cs>>>(T, jobs);
    else
      tc_build_c_factored<false><<<g_fact, 128, smem_c, cs>>>(T, jobs);
  } else {
    if (bf16)
      tc_build_c<true><<<g_old, 256, 0, cs>>>(T, jobs);
    else
      tc_build_c<false><<<g_old, 256, 0, cs>>>(T, jobs);
  }
  if (forked) {
    cudaEventRecord(fork->join, cs);
    cudaStreamWaitEvent(stream, fork->join, 0);
  }
}

// One work item: field descriptor and the tile's block coordinates.
struct Item {
  TcField f;
  int ib, jb, nt;
  int local;   // item index within its field
  int seg;     // harmonic segment (0 without a split)
  int k0, k1;  // stages [k0, k1) of the segment
};

__device__ __forceinline__ Item decode_item(const TcKernelArgs& A, int idx) {
  Item it;
  int fid = 0, local = idx;
  if (A.items) {
    const int2 e = A.items[idx];
    fid = e.x;
    local = e.y;
  }
  it.f = A.fields ? A.fields[fid] : A.f0;
  it.local = local;
  const int tiles_m = it.f.bix * it.f.bjx;
  const int per_seg = tiles_m * it.f.bn;
  it.seg = local / per_seg;
  it.k0 = static_cast<int>(static_cast<long long>(it.seg) * it.f.stages / it.f.split);
  it.k1 = static_cast<int>(static_cast<long long>(it.seg + 1) * it.f.stages / it.f.split);
  const int lt = local - it.seg * per_seg;
  it.nt = lt / tiles_m;
  const int mt = lt - it.nt * tiles_m;
  // Within a column tile, bands of `band` row blocks along i, each walked
  // over every j (the next band in the opposite j direction).
  const int g = min(it.f.band, it.f.bix);
  const int b = mt / (g * it.f.bjx);
  const int gb = min(g, it.f.bix - b * g);
  const int o = mt - b * g * it.f.bjx;
  const int jo = o / gb;
  it.ib = b * g + (o - jo * gb);
  it.jb = (b & 1) ? it.f.bjx - 1 - jo : jo;
  return it;
}

// Number of stages of work item idx (its harmonic segment), read without
// copying the field descriptor (the generator warps only count stages).
__device__ __forceinline__ int item_stages(const TcKernelArgs& A, int idx) {
  int fid = 0, local = idx;
  if (A.items) {
    const int2 e = A.items[idx];
    fid = e.x;
    local = e.y;
  }
  const TcField& f = A.fields ? A.fields[fid] : A.f0;
  const int split = f.split;
  if (split <= 1) return f.stages;
  const int seg = local / (f.bix * f.bjx * f.bn);
  return static_cast<int>(static_cast<long long>(seg + 1) * f.stages / split -
                          static_cast<long long>(seg) * f.stages / split);
}

// W (16 or 32) columns of a chunk drain: all TMEM loads issued before one
// wait, so each round trip to tensor memory covers W columns.
template <int W>
__device__ __forceinline__ void drain_cols(uint32_t lane_base, uint32_t master_col, int c0, bool first, bool last,
                                           bool row_ok, float* dst, long long plane, int k0, int n3, float scaling) {
  uint32_t v[W], m[W];
#pragma unroll
  for (int h = 0; h < W / 16; ++h) {
    tmem_ld_32x32b_x16(lane_base + c0 + 16 * h, *reinterpret_cast<uint32_t(*)[16]>(v + 16 * h));
    if (!first) tmem_ld_32x32b_x16(lane_base + master_col + c0 + 16 * h, *reinterpret_cast<uint32_t(*)[16]>(m + 16 * h));
  }
  tmem_wait_ld();
  if (!first) {
#pragma unroll
    for (int c = 0; c < W; ++c) v[c] = __float_as_uint(__fadd_rn(__uint_as_float(m[c]), __uint_as_float(v[c])));
  }
  if (!last) {
#pragma unroll
    for (int h = 0; h < W / 16; ++h)
      tmem_st_32x32b_x16(lane_base + master_col + c0 + 16 * h, *reinterpret_cast<const uint32_t(*)[16]>(v + 16 * h));
  } else if (row_ok) {
    // The scaling of scarflib_srm.f90:847, applied once to the sum.
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int kcol = k0 + c0 + c;
      if (kcol < n3) dst[plane * kcol] = __fmul_rn(__uint_as_float(v[c]), scaling);
    }
  }
}

// One chunk drain of the epilogue for the 32 rows of this warp: the TMEM
// chunk accumulator is added (round to nearest) into the FP32 master at
// master_col, or, for the last chunk, master + chunk is scaled and stored.
__device__ __forceinline__ void drain_chunk(uint32_t lane_base, uint32_t master_col, int ntile_n, bool first,
                                            bool last, bool row_ok, float* dst, long long plane, int k0, int n3,
                                            float scaling) {
  int c0 = 0;
  for (; c0 + 32 <= ntile_n; c0 += 32)
    drain_cols<32>(lane_base, master_col, c0, first, last, row_ok, dst, plane, k0, n3, scaling);
  if (c0 < ntile_n) drain_cols<16>(lane_base, master_col, c0, first, last, row_ok, dst, plane, k0, n3, scaling);
  if (!last) tmem_wait_st();
}

// Slab accounting after a warp stored its 32 rows of row tile (ib, jb) of
// column tile nt: the last of the slab's 4 x tiles arrivals raises the host
// flag. System-scope fences order the field stores before the count and the
// count before the flag, so the host may copy the slab out once it sees it.
__device__ __forceinline__ void signal_slab(const TcKernelArgs& A, const TcField& f, int ib, int jb, int nt,
                                            int lane) {
  __threadfence_system();
  __syncwarp();
  if (lane == 0 && ib < f.bi && jb < f.bj) {
    const int jb0 = (jb / A.slab_jbs) * A.slab_jbs;
    const int slab = nt * A.slab_spn + jb / A.slab_jbs;
    const int expect = 4 * f.bi * min(A.slab_jbs, f.bj - jb0);
    if (atomicAdd(&A.slab_cnt[slab], 1) == expect - 1) {
      __threadfence_system();
      A.slab_flag[slab] = 1;
    }
  }
}

// Statistics of the values one warp stored for its 32 rows of an item (one
// row per lane, columns k0 .. min(k0 + ntile_n, n3) - 1), read back after the
// accumulator is released (the warp just stored them: L2 hits), accumulated
// in FP64 about the row's first value, merged over the warp in a fixed order
// and written by lane 0 into the item's record.
__device__ __forceinline__ void record_stats(Moments* rec, const float* dst, long long plane, int k0, int ntile_n,
                                             int n3, bool row_ok, int lane) {
  double s1 = 0.0, s2 = 0.0, cnt = 0.0, shift = 0.0;
  if (row_ok) {
    const int kend = min(k0 + ntile_n, n3);
    if (k0 < kend) shift = static_cast<double>(__ldcg(dst + plane * k0));
    for (int k = k0; k < kend; ++k) {
      const double d = static_cast<double>(__ldcg(dst + plane * k)) - shift;
      s1 += d;
      s2 = fma(d, d, s2);
      cnt += 1.0;
    }
  }
  const Moments m = warp_moments(moments_from_shifted(cnt, shift, s1, s2));
  if (lane == 0) *rec = m;
}

// The field's last item is stored: the last epilogue warp to arrive raises
// the field's host flag. System-scope fences order the field stores before
// the count and the count before the flag, as for slabs.
__device__ __forceinline__ void signal_field(const TcField& f, int lane) {
  __threadfence_system();
  __syncwarp();
  if (lane == 0 && atomicAdd(f.done_cnt, 1) == f.done_expect - 1) {
    __threadfence_system();
    *f.done_flag = 1;
  }
}

// A operand of one stage into shared memory: row r of the tile (the
// (ii, jj) point of the row block), kGenHarm harmonics from h0, 16-bit hi and lo
// images in the 64-B-swizzled K-major layout.
template <bool kBf16>
__device__ __forceinline__ void generate_a_smem(const TcKernelArgs& A, uint8_t* st, const uint8_t* rs, int r, int ii,
                                                int jj, int h0) {
  // rs: the stage's R tile [16][ti] followed by its S tile [16][tj] (float2)
  const float2* rt = reinterpret_cast<const float2*>(rs) + h0 * A.ti + ii;
  const float2* stt = reinterpret_cast<const float2*>(rs) + kStageHarm * A.ti + h0 * A.tj + jj;
  typename OperandPair<kBf16>::T2 hv[kGenHarm], lv[kGenHarm];
  gen_products<kBf16>(rt, stt, A.ti, A.tj, hv, lv);
  uint8_t* a_hi = st + A.off_a;
  uint8_t* a_lo = a_hi + kATileBytes;
#pragma unroll
  for (int cc = 0; cc < kGenHarm / 4; ++cc) {
    const uint32_t off = swz64(static_cast<uint32_t>(r), static_cast<uint32_t>(h0 / 4 + cc));
    *reinterpret_cast<uint4*>(a_hi + off) = *reinterpret_cast<const uint4*>(hv + 4 * cc);
    *reinterpret_cast<uint4*>(a_lo + off) = *reinterpret_cast<const uint4*>(lv + 4 * cc);
  }
  fence_proxy_async_smem();
}

// TMEM columns (512 allocated). Shared-memory A: chunk accumulator [0, 256),
// FP32 master [256, 512). TMEM A: accumulator [0, 192), master [192, 384) and
// an A ring of kTmemAStages stages [384, 512), each stage holding the hi half
// (16 columns: 32 fp16 along K) then the lo half.
constexpr int kMaxNSmemA = 256;
constexpr int kMaxNTmemA = 192;
constexpr int kTmemAStages = 4;
constexpr uint32_t kTmemACol0 = 384;
constexpr uint32_t kTmemAStageCols = 32;

// ------------------------------------------------------------- main kernel --
// kTmemA selects where the generated A operand lives: shared memory (the
// tensor core reads both operands from shared memory) or tensor memory
// (tcgen05.st from the generator registers, MMA in its TMEM-A form). The
// TMEM-A form takes the A tile's writes and its three operand reads per
// stage off the shared-memory port, which is the pipeline's bottleneck.
template <bool kTmemA, bool kBf16>
__global__ void __launch_bounds__(kThreads, 1) srm_tc_kernel(const TcKernelArgs A) {
  constexpr uint32_t kMasterCol = kTmemA ? kMaxNTmemA : kMaxNSmemA;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int S = A.nstage_buf;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + A.bars_off);  // bulk copies landed
  uint64_t* agen = full + S;                                         // A tile generated
  uint64_t* empty = agen + S;                                        // stage consumed by MMA
  uint64_t* accf = empty + S;                                        // chunk accumulated
  uint64_t* acce = accf + 1;                                         // chunk drained
  uint64_t* fin = acce + 1;                                          // MMA drain at exit
  uint64_t* item_full = fin + 1;                                     // item slot written [kItemRing]
  uint64_t* item_empty = item_full + kItemRing;                      // item slot read [kItemRing]
  int* item_slot = reinterpret_cast<int*>(item_empty + kItemRing);   // [kItemRing]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(item_slot + kItemRing);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&agen[s], kGenWarps);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 4);
    mbar_init(fin, 1);
    for (int q = 0; q < kItemRing; ++q) {
      mbar_init(&item_full[q], 1);
      mbar_init(&item_empty[q], kItemConsumers);
    }
    fence_mbar_init();
  }
  if (warp == 2) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  bool ok = true;

  // Consumer side of the item ring: the next item index (or -1 when the
  // queue is exhausted). Lane 0 of each consumer warp acknowledges the slot.
  auto next_item = [&](uint32_t it, int& idx) -> bool {
    const int q = it % kItemRing;
    if (!warp_wait_bounded(&item_full[q], (it / kItemRing) & 1, A.status, false)) return false;
    idx = *reinterpret_cast<volatile int*>(&item_slot[q]);
    __syncwarp();
    if (lane == 0) mbar_arrive(&item_empty[q]);
    return true;
  };

  if (warp == 0) {
    // ------------------------------------------------------ producer -------
    // One thread; stage slot and phase advance incrementally.
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0, issued = 0;
      for (uint32_t it = 0; ok; ++it) {
        const int q = it % kItemRing;
        if (!mbar_wait_bounded(&item_empty[q], ((it / kItemRing) & 1) ^ 1, A.status)) {
          ok = false;
          break;
        }
        int idx = atomicAdd(A.queue, 1);
        if (idx >= A.num_items) idx = -1;
        item_slot[q] = idx;
        mbar_arrive(&item_full[q]);  // release: the slot write is visible to waiters
        if (idx < 0) break;
        const Item w = decode_item(A, idx);
        const uint32_t bbytes = 2u * w.f.ntile_n * kRowBytes;
        const uint32_t rbytes = kStageHarm * A.ti * 8u;
        const uint32_t sbytes = kStageHarm * A.tj * 8u;
        const uint8_t* csrc = w.f.cimg + static_cast<size_t>(w.nt) * w.f.stages * bbytes;
        const float2* rsrc = w.f.rimg + static_cast<size_t>(w.ib) * w.f.stages * kStageHarm * A.ti;
        const float2* ssrc = w.f.simg + static_cast<size_t>(w.jb) * w.f.stages * kStageHarm * A.tj;
        for (int k = w.k0; k < w.k1; ++k) {
          if (!mbar_wait_bounded(&empty[s], ph ^ 1, A.status)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s * A.stage_bytes;
          mbar_arrive_expect_tx(&full[s], bbytes + rbytes + sbytes);
          bulk_g2s(st + A.off_b, csrc + static_cast<size_t>(k) * bbytes, bbytes, &full[s]);
          bulk_g2s(st + A.off_r, rsrc + static_cast<size_t>(k) * kStageHarm * A.ti, rbytes, &full[s]);
          bulk_g2s(st + A.off_s, ssrc + static_cast<size_t>(k) * kStageHarm * A.tj, sbytes, &full[s]);
          ++issued;
          if (++s == S) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if (!ok) {
        // Let every issued copy land before shared memory is released: the
        // last min(issued, S) stages, each in the phase it was issued in.
        const uint32_t n_in_flight = issued < static_cast<uint32_t>(S) ? issued : S;
        for (uint32_t b = 1; b <= n_in_flight; ++b) {
          const uint32_t c = issued - b;
          mbar_wait_drain(&full[c % S], (c / S) & 1);
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------- MMA issuer ----
    // The K loop of an item runs in chunks of chunk_stages stages, each
    // accumulated from zero in the TMEM chunk buffer (columns from 0). At the
    // end of a chunk the epilogue adds the buffer into an FP32 master
    // accumulator held in TMEM from column kMasterCol (round to nearest), or, for
    // the last chunk, writes master + chunk to the field. The tensor core's
    // own FP32 accumulation is not round-to-nearest, so its error grows with
    // the number of accumulation steps into one buffer; chunking bounds it.
    // One thread issues; stage slot and phase advance incrementally.
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0, chunk = 0;
      bool issued_any = false;
      // Stage slot's B image landed and its A tile generated. Both phases are
      // probed back to back first (their round trips overlap); the bounded
      // waits run only when one is still open.
      auto stage_inputs_ready = [&](int sl, uint32_t par) -> bool {
        const bool f = mbar_test_wait(&full[sl], par);
        const bool g = mbar_test_wait(&agen[sl], par);
        if (f && g) return true;
        return mbar_wait_bounded(&full[sl], par, A.status) && mbar_wait_bounded(&agen[sl], par, A.status);
      };
      for (uint32_t it = 0; ok; ++it) {
        const int q = it % kItemRing;
        if (!mbar_wait_bounded(&item_full[q], (it / kItemRing) & 1, A.status)) {
          ok = false;
          break;
        }
        const int idx = *reinterpret_cast<volatile int*>(&item_slot[q]);
        mbar_arrive(&item_empty[q]);
        if (idx < 0) break;
        const Item w = decode_item(A, idx);
        const uint32_t b_lo_off = A.off_b + w.f.ntile_n * kRowBytes;
        for (int c0 = w.k0; c0 < w.k1 && ok; c0 += w.f.chunk_stages, ++chunk) {
          const int c1 = min(w.k1, c0 + w.f.chunk_stages);
          // The previous chunk must be drained before the buffer restarts.
          if (chunk > 0 && !mbar_wait_bounded(acce, (chunk - 1) & 1, A.status)) {
            ok = false;
            break;
          }
          // Inputs of the chunk's first stage. Each later stage's inputs are
          // checked between the two K halves of the stage before it, while
          // the tensor core still holds queued MMAs: an issuing thread that
          // checked them after its last MMA would leave the tensor pipe idle
          // for the round trips of the checks.
          if (!stage_inputs_ready(s, ph)) {
            ok = false;
            break;
          }
          for (int k = c0; k < c1; ++k) {
            tc_fence_after();
            const uint32_t st = smem_u32(smem + s * A.stage_bytes);
            const uint32_t b_hi = st + A.off_b, b_lo = st + b_lo_off;
            const int s_next = (s + 1 == S) ? 0 : s + 1;
            const uint32_t ph_next = (s + 1 == S) ? (ph ^ 1u) : ph;
            bool next_ok = true;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
              const uint64_t dbh = umma_smem_desc(b_hi + 32 * kk, 16, 512, kSwizzle64);
              const uint64_t dbl = umma_smem_desc(b_lo + 32 * kk, 16, 512, kSwizzle64);
              const uint32_t acc = (k > c0 || kk > 0) ? 1u : 0u;
              if constexpr (kTmemA) {
                const uint32_t ta = tmem_base + kTmemACol0 + s * kTmemAStageCols + 8 * kk;
                umma_f16_ts(tmem_base, ta, dbh, w.f.idesc, acc);
                if (w.f.terms == 3) umma_f16_ts(tmem_base, ta, dbl, w.f.idesc, 1u);
                umma_f16_ts(tmem_base, ta + 16, dbh, w.f.idesc, 1u);
              } else {
                const uint32_t a_hi = st + A.off_a, a_lo = a_hi + kATileBytes;
                const uint64_t dah = umma_smem_desc(a_hi + 32 * kk, 16, 512, kSwizzle64);
                const uint64_t dal = umma_smem_desc(a_lo + 32 * kk, 16, 512, kSwizzle64);
                umma_f16(tmem_base, dah, dbh, w.f.idesc, acc);
                if (w.f.terms == 3) umma_f16(tmem_base, dah, dbl, w.f.idesc, 1u);
                umma_f16(tmem_base, dal, dbh, w.f.idesc, 1u);
              }
              if (kk == 0 && k + 1 < c1) next_ok = stage_inputs_ready(s_next, ph_next);
            }
            umma_commit(&empty[s]);
            issued_any = true;
            s = s_next;
            ph = ph_next;
            if (!next_ok) {
              ok = false;
              break;
            }
          }
          if (!ok) break;
          umma_commit(accf);
        }
      }
      if (issued_any) {
        // All MMAs of this CTA complete before tensor memory is released.
        umma_commit(fin);
        mbar_wait_drain(fin, 0);
      }
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4) {
    // --------------------------------------------------------- epilogue ----
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const int ii = r & (A.ti - 1);
    const int jj = r >> A.ti_shift;
    const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(q * 32) << 16);
    uint32_t chunk = 0;
    for (uint32_t it = 0; ok; ++it) {
      int idx;
      if (!next_item(it, idx)) {
        ok = false;
        break;
      }
      if (idx < 0) break;
      const Item w = decode_item(A, idx);
      const int i = w.ib * A.ti + ii;
      const int j = w.jb * A.tj + jj;
      const bool row_ok = (i < w.f.n1) && (j < w.f.n2);
      const long long plane = w.f.sc;
      float* dst = w.f.field + i * w.f.sr + j * w.f.ss;
      const int k0 = w.nt * w.f.ntile_n;
      // A split item stores its segment's unscaled partial sums.
      float* out = w.f.split > 1 ? w.f.partial + w.seg * w.f.seg_stride + (dst - w.f.field) : dst;
      const float out_scale = w.f.split > 1 ? 1.0f : w.f.scaling;
      for (int s0 = w.k0; s0 < w.k1; s0 += w.f.chunk_stages, ++chunk) {
        const bool first = (s0 == w.k0);
        const bool last = (s0 + w.f.chunk_stages >= w.k1);
        if (!warp_wait_bounded(accf, chunk & 1, A.status, false)) {
          ok = false;
          break;
        }
        tc_fence_after();
        drain_chunk(lane_base, kMasterCol, w.f.ntile_n, first, last, row_ok, out, plane, k0, w.f.n3, out_scale);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce);
        if (last && A.slab_cnt) signal_slab(A, w.f, w.ib, w.jb, w.nt, lane);
        if (last && w.f.done_flag) signal_field(w.f, lane);
        if (last && w.f.stats)  // (never with a split: out is the field then)
          record_stats(w.f.stats + w.local * 4 + q, out, plane, k0, w.f.ntile_n, w.f.n3, row_ok, lane);
      }
    }
  } else if (warp >= kGenWarp0) {
    // -------------------------------------------------------- generators ---
    // Thread g owns row r of the A tile (TMEM lane r: warp % 4 is the lane
    // quadrant) and kGenHarm consecutive harmonics of every stage.
    const int g = threadIdx.x - kGenWarp0 * 32;
    const int r = g & (kRows - 1);
    const int h0 = (g >> 7) * kGenHarm;
    const int ii = r & (A.ti - 1);
    const int jj = r >> A.ti_shift;
    uint32_t cnt = 0;
    for (uint32_t it = 0; ok; ++it) {
      int idx;
      if (!next_item(it, idx)) {
        ok = false;
        break;
      }
      if (idx < 0) break;
      const int stages = item_stages(A, idx);
      for (int k = 0; k < stages; ++k, ++cnt) {
        const int s = cnt % S;
        const uint32_t ph = (cnt / S) & 1;
        if (!warp_wait_bounded(&full[s], ph, A.status, false)) {
          ok = false;
          break;
        }
        uint8_t* st = smem + s * A.stage_bytes;
        const float2* rt = reinterpret_cast<const float2*>(st + A.off_r) + h0 * A.ti + ii;
        const float2* stt = reinterpret_cast<const float2*>(st + A.off_s) + h0 * A.tj + jj;
        typename OperandPair<kBf16>::T2 hv[kGenHarm], lv[kGenHarm];
        gen_products<kBf16>(rt, stt, A.ti, A.tj, hv, lv);
        if constexpr (kTmemA) {
          // Harmonic h = column h of the stage's hi half (16 + h: lo half).
          // The slot's previous MMAs completed before its bulk copies were
          // issued (empty -> full).
          tc_fence_after();
          const uint32_t ta = tmem_base + (static_cast<uint32_t>(r & ~31) << 16) + kTmemACol0 +
                              s * kTmemAStageCols + h0;
          tmem_st_cols<kGenHarm>(ta, reinterpret_cast<const uint32_t*>(hv));
          tmem_st_cols<kGenHarm>(ta + 16, reinterpret_cast<const uint32_t*>(lv));
          tmem_wait_st();
          tc_fence_before();
        } else {
          uint8_t* a_hi = st + A.off_a;
          uint8_t* a_lo = a_hi + kATileBytes;
#pragma unroll
          for (int cc = 0; cc < kGenHarm / 4; ++cc) {
            const uint32_t off = swz64(static_cast<uint32_t>(r), static_cast<uint32_t>(h0 / 4 + cc));
            *reinterpret_cast<uint4*>(a_hi + off) = *reinterpret_cast<const uint4*>(hv + 4 * cc);
            *reinterpret_cast<uint4*>(a_lo + off) = *reinterpret_cast<const uint4*>(lv + 4 * cc);
          }
          fence_proxy_async_smem();
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&agen[s]);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

// -------------------------------------------------------- CTA-pair kernel --
// The tile of a work item is split over the two CTAs of a cluster: 256 rows
// (row blocks jb = 2 jbp + rank, or ib = 2 ibp + rank when the field has a
// single row block along j) x N columns. Each CTA generates its 128 rows of
// A, stages half of the B image (N / 2 rows) and drains its own accumulators;
// the even CTA issues one cta_group::2 MMA per K step for both. Per SM this
// halves the B traffic of the one-CTA form, and the pair MMA runs at the
// tensor core's full rate down to small N.
//
// Two rings per CTA decouple the inputs: the small factor tiles (R, S) run
// up to nrs stages ahead so the generators never wait on copies, and the
// A / B stage ring (nstage_buf slots) feeds the MMA.
//
// Barriers (the same offsets in both CTAs):
//   item ring    the even CTA's R/S producer takes items from the queue and
//                publishes each in both CTAs; the other consumers of both
//                CTAs release slots on the even CTA's item_empty.
//   rs_full/rs_empty[r]  local: R/S tiles of stage r landed / consumed.
//   b_full[s]    local: this CTA's B half of stage s landed.
//   agen[s]      local generators wrote stage s's A rows; the even CTA's
//                also counts the odd CTA's forwarder, which relays the odd
//                CTA's agen[s] and b_full[s] with one cluster-scope arrive.
//   empty[s]     both: the pair MMAs of stage s completed (multicast commit).
//   accf         both: a chunk is accumulated (multicast commit).
//   acce         even CTA: the epilogues of both CTAs drained the chunk.
template <bool kBf16>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1) srm_tc_pair_kernel(const TcKernelArgs A) {
  constexpr uint32_t kMasterCol = kMaxNSmemA;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int S = A.nstage_buf;
  const int NR = A.nrs;
  uint64_t* b_full = reinterpret_cast<uint64_t*>(smem + A.bars_off);
  uint64_t* agen = b_full + S;
  uint64_t* empty = agen + S;
  uint64_t* rs_full = empty + S;
  uint64_t* rs_empty = rs_full + NR;
  uint64_t* accf = rs_empty + NR;
  uint64_t* acce = accf + 1;
  uint64_t* fin = acce + 1;
  uint64_t* item_full = fin + 1;
  uint64_t* item_empty = item_full + kItemRing;
  int* item_slot = reinterpret_cast<int*>(item_empty + kItemRing);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(item_slot + kItemRing);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const bool even = rank == 0;
  // Consumers of one item: B producers (2), the even CTA's MMA thread, the
  // odd CTA's R/S producer and forwarder, epilogue (2 x 4) and generator
  // (2 x kGenWarps) warps. The even CTA's R/S producer publishes.
  constexpr int kPairConsumers = 2 + 1 + 2 + 2 * 4 + 2 * kGenWarps;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&agen[s], even ? kGenWarps + 1 : kGenWarps);
      mbar_init(&empty[s], 1);
    }
    for (int r = 0; r < NR; ++r) {
      mbar_init(&rs_full[r], 1);
      mbar_init(&rs_empty[r], kGenWarps);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 8);
    mbar_init(fin, 1);
    for (int q = 0; q < kItemRing; ++q) {
      mbar_init(&item_full[q], 1);
      mbar_init(&item_empty[q], kPairConsumers);
    }
    fence_mbar_init();
  }
  if (warp == 2) {
    tmem_alloc_pair(tmem_slot, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // barrier initialisation and TMEM of both CTAs visible to the pair
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  bool ok = true;

  const uint32_t agen0 = cluster_map(agen, 0);
  const uint32_t acce0 = cluster_map(acce, 0);
  const uint32_t item_empty0 = cluster_map(item_empty, 0);

  // Item ring, consumer side (one thread or a whole warp).
  auto take_item = [&](uint32_t it, int& idx) -> bool {
    const int q = it % kItemRing;
    if (!mbar_wait_bounded_cluster(&item_full[q], (it / kItemRing) & 1, A.status)) return false;
    idx = *reinterpret_cast<volatile int*>(&item_slot[q]);
    return true;
  };
  auto release_item = [&](uint32_t it) { mbar_arrive_cluster(item_empty0 + 8u * (it % kItemRing)); };
  // Whole-warp consumers: lane 0 waits and releases, the warp shares the item.
  auto take_item_warp = [&](uint32_t it, int& idx) -> bool {
    const int q = it % kItemRing;
    if (!warp_wait_bounded(&item_full[q], (it / kItemRing) & 1, A.status, true)) return false;
    idx = *reinterpret_cast<volatile int*>(&item_slot[q]);
    __syncwarp();
    if (lane == 0) release_item(it);
    return true;
  };
  auto tile_of = [&](const Item& w, int& ib, int& jb) {
    ib = w.f.pair_i ? 2 * w.ib + static_cast<int>(rank) : w.ib;
    jb = w.f.pair_i ? w.jb : 2 * w.jb + static_cast<int>(rank);
  };

  if (warp == 2) {
    // ------------------------------------------------- R / S producer ------
    if (lane == 0) {
      int r = 0;
      uint32_t rph = 0, issued = 0;
      const uint32_t peer_full = cluster_map(item_full, 1);
      const uint32_t peer_slot = cluster_map(item_slot, 1);
      for (uint32_t it = 0; ok; ++it) {
        const int q = it % kItemRing;
        int idx;
        if (even) {
          if (!mbar_wait_bounded_cluster(&item_empty[q], ((it / kItemRing) & 1) ^ 1, A.status)) {
            ok = false;
            break;
          }
          idx = atomicAdd(A.queue, 1);
          if (idx >= A.num_items) idx = -1;
          item_slot[q] = idx;
          st_cluster_u32(peer_slot + 4u * q, static_cast<uint32_t>(idx));
          mbar_arrive(&item_full[q]);
          mbar_arrive_cluster(peer_full + 8u * q);  // release: the remote slot store first
        } else {
          if (!take_item(it, idx)) {
            ok = false;
            break;
          }
          release_item(it);
        }
        if (idx < 0) break;
        const Item w = decode_item(A, idx);
        int ib, jb;
        tile_of(w, ib, jb);
        const uint32_t rbytes = kStageHarm * A.ti * 8u;
        const uint32_t sbytes = kStageHarm * A.tj * 8u;
        const float2* rsrc = w.f.rimg + static_cast<size_t>(ib) * w.f.stages * kStageHarm * A.ti;
        const float2* ssrc = w.f.simg + static_cast<size_t>(jb) * w.f.stages * kStageHarm * A.tj;
        for (int k = w.k0; k < w.k1; ++k) {
          if (!mbar_wait_bounded(&rs_empty[r], rph ^ 1, A.status)) {
            ok = false;
            break;
          }
          uint8_t* rs = smem + A.rs_base + r * A.rs_bytes;
          mbar_arrive_expect_tx(&rs_full[r], rbytes + sbytes);
          bulk_g2s(rs, rsrc + static_cast<size_t>(k) * kStageHarm * A.ti, rbytes, &rs_full[r]);
          bulk_g2s(rs + rbytes, ssrc + static_cast<size_t>(k) * kStageHarm * A.tj, sbytes, &rs_full[r]);
          ++issued;
          if (++r == NR) {
            r = 0;
            rph ^= 1;
          }
        }
      }
      if (!ok) {
        const uint32_t n_in_flight = issued < static_cast<uint32_t>(NR) ? issued : NR;
        for (uint32_t b = 1; b <= n_in_flight; ++b) {
          const uint32_t c = issued - b;
          mbar_wait_drain(&rs_full[c % NR], (c / NR) & 1);
        }
      }
    }
    __syncwarp();
  } else if (warp == 0) {
    // ------------------------------------------------------ B producer -----
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0, issued = 0;
      for (uint32_t it = 0; ok; ++it) {
        int idx;
        if (!take_item(it, idx)) {
          ok = false;
          break;
        }
        release_item(it);
        if (idx < 0) break;
        const Item w = decode_item(A, idx);
        const uint32_t bbytes = w.f.ntile_n * kRowBytes;  // this CTA's half: N / 2 rows, hi and lo
        const uint8_t* csrc = w.f.cimg + (static_cast<size_t>(w.nt) * w.f.stages * 2 + rank) * bbytes;
        for (int k = w.k0; k < w.k1; ++k) {
          if (!mbar_wait_bounded_cluster(&empty[s], ph ^ 1, A.status)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&b_full[s], bbytes);
          bulk_g2s(smem + s * A.stage_bytes + A.off_b, csrc + static_cast<size_t>(k) * 2 * bbytes, bbytes, &b_full[s]);
          ++issued;
          if (++s == S) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if (!ok) {
        const uint32_t n_in_flight = issued < static_cast<uint32_t>(S) ? issued : S;
        for (uint32_t b = 1; b <= n_in_flight; ++b) {
          const uint32_t c = issued - b;
          mbar_wait_drain(&b_full[c % S], (c / S) & 1);
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------- MMA issuer (even CTA) -----
    if (even && lane == 0) {
      int s = 0;
      uint32_t ph = 0, chunk = 0;
      bool issued_any = false;
      // This CTA's B half landed and both CTAs' A rows (and the odd CTA's B
      // half, relayed by its forwarder) are in place.
      auto stage_inputs_ready = [&](int sl, uint32_t par) -> bool {
        const bool f = mbar_test_wait(&b_full[sl], par);
        const bool g = mbar_test_wait_cluster(&agen[sl], par);
        if (f && g) return true;
        return mbar_wait_bounded(&b_full[sl], par, A.status) && mbar_wait_bounded_cluster(&agen[sl], par, A.status);
      };
      for (uint32_t it = 0; ok; ++it) {
        int idx;
        if (!take_item(it, idx)) {
          ok = false;
          break;
        }
        release_item(it);
        if (idx < 0) break;
        const Item w = decode_item(A, idx);
        const uint32_t b_lo_off = A.off_b + (w.f.ntile_n / 2) * kRowBytes;
        for (int c0 = w.k0; c0 < w.k1 && ok; c0 += w.f.chunk_stages, ++chunk) {
          const int c1 = min(w.k1, c0 + w.f.chunk_stages);
          if (chunk > 0 && !mbar_wait_bounded_cluster(acce, (chunk - 1) & 1, A.status)) {
            ok = false;
            break;
          }
          // As in the one-CTA form: the next stage's inputs are checked
          // between the K halves of the current stage.
          if (!stage_inputs_ready(s, ph)) {
            ok = false;
            break;
          }
          for (int k = c0; k < c1; ++k) {
            tc_fence_after();
            const uint32_t st = smem_u32(smem + s * A.stage_bytes);
            const uint32_t a_hi = st + A.off_a, a_lo = a_hi + kATileBytes;
            const uint32_t b_hi = st + A.off_b, b_lo = st + b_lo_off;
            const int s_next = (s + 1 == S) ? 0 : s + 1;
            const uint32_t ph_next = (s + 1 == S) ? (ph ^ 1u) : ph;
            bool next_ok = true;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
              const uint64_t dah = umma_smem_desc(a_hi + 32 * kk, 16, 512, kSwizzle64);
              const uint64_t dal = umma_smem_desc(a_lo + 32 * kk, 16, 512, kSwizzle64);
              const uint64_t dbh = umma_smem_desc(b_hi + 32 * kk, 16, 512, kSwizzle64);
              const uint64_t dbl = umma_smem_desc(b_lo + 32 * kk, 16, 512, kSwizzle64);
              umma_f16_pair(tmem_base, dah, dbh, w.f.idesc, (k > c0 || kk > 0) ? 1u : 0u);
              if (w.f.terms == 3) umma_f16_pair(tmem_base, dah, dbl, w.f.idesc, 1u);
              umma_f16_pair(tmem_base, dal, dbh, w.f.idesc, 1u);
              if (kk == 0 && k + 1 < c1) next_ok = stage_inputs_ready(s_next, ph_next);
            }
            umma_commit_pair_both(&empty[s]);
            issued_any = true;
            s = s_next;
            ph = ph_next;
            if (!next_ok) {
              ok = false;
              break;
            }
          }
          if (!ok) break;
          umma_commit_pair_both(accf);
        }
      }
      if (issued_any) {
        umma_commit_pair_local(fin);
        mbar_wait_drain(fin, 0);
      }
    }
    __syncwarp();
  } else if (warp == 3) {
    // ------------------------------------------- forwarder (odd CTA) -------
    // One cluster-scope arrive per stage on the even CTA's agen[s] once this
    // CTA's A rows and B half of stage s are in place.
    if (!even && lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      for (uint32_t it = 0; ok; ++it) {
        int idx;
        if (!take_item(it, idx)) {
          ok = false;
          break;
        }
        release_item(it);
        if (idx < 0) break;
        const int stages = item_stages(A, idx);
        for (int k = 0; k < stages; ++k) {
          if (!mbar_wait_bounded(&agen[s], ph, A.status) || !mbar_wait_bounded(&b_full[s], ph, A.status)) {
            ok = false;
            break;
          }
          // This CTA's A rows (generic stores, proxy fence, local release)
          // and B half (bulk-copy completion) are in place: a plain signal
          // suffices, and only this SM's tensor core reads them.
          mbar_arrive_cluster_relaxed(agen0 + 8u * s);
          if (++s == S) {
            s = 0;
            ph ^= 1;
          }
        }
      }
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4) {
    // --------------------------------------------------------- epilogue ----
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const int ii = r & (A.ti - 1);
    const int jj = r >> A.ti_shift;
    const uint32_t lane_base = tmem_base + (static_cast<uint32_t>(q * 32) << 16);
    uint32_t chunk = 0;
    for (uint32_t it = 0; ok; ++it) {
      int idx;
      if (!take_item_warp(it, idx)) {
        ok = false;
        break;
      }
      if (idx < 0) break;
      const Item w = decode_item(A, idx);
      int ib, jb;
      tile_of(w, ib, jb);
      const int i = ib * A.ti + ii;
      const int j = jb * A.tj + jj;
      const bool row_ok = (i < w.f.n1) && (j < w.f.n2);
      const long long plane = w.f.sc;
      float* dst = w.f.field + i * w.f.sr + j * w.f.ss;
      const int k0 = w.nt * w.f.ntile_n;
      // A split item stores its segment's unscaled partial sums.
      float* out = w.f.split > 1 ? w.f.partial + w.seg * w.f.seg_stride + (dst - w.f.field) : dst;
      const float out_scale = w.f.split > 1 ? 1.0f : w.f.scaling;
      for (int s0 = w.k0; s0 < w.k1; s0 += w.f.chunk_stages, ++chunk) {
        const bool first = (s0 == w.k0);
        const bool last = (s0 + w.f.chunk_stages >= w.k1);
        if (!warp_wait_bounded(accf, chunk & 1, A.status, true)) {
          ok = false;
          break;
        }
        tc_fence_after();
        drain_chunk(lane_base, kMasterCol, w.f.ntile_n, first, last, row_ok, out, plane, k0, w.f.n3, out_scale);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(acce0);
        if (last && A.slab_cnt) signal_slab(A, w.f, ib, jb, w.nt, lane);
        if (last && w.f.done_flag) signal_field(w.f, lane);
        if (last && w.f.stats)  // (never with a split: out is the field then)
          record_stats(w.f.stats + (w.local * 2 + static_cast<int>(rank)) * 4 + q, out, plane, k0, w.f.ntile_n,
                       w.f.n3, row_ok, lane);
      }
    }
  } else if (warp >= kGenWarp0) {
    // -------------------------------------------------------- generators ---
    const int g = threadIdx.x - kGenWarp0 * 32;
    const int r = g & (kRows - 1);
    const int h0 = (g >> 7) * kGenHarm;
    const int ii = r & (A.ti - 1);
    const int jj = r >> A.ti_shift;
    int s = 0, rr = 0;
    uint32_t ph = 0, rph = 0;
    for (uint32_t it = 0; ok; ++it) {
      int idx;
      if (!take_item_warp(it, idx)) {
        ok = false;
        break;
      }
      if (idx < 0) break;
      const int stages = item_stages(A, idx);
      for (int k = 0; k < stages; ++k) {
        // factor tiles in place, and the A slot's previous MMAs complete
        if (!warp_wait_bounded(&rs_full[rr], rph, A.status, false) ||
            !warp_wait_bounded(&empty[s], ph ^ 1, A.status, true)) {
          ok = false;
          break;
        }
        generate_a_smem<kBf16>(A, smem + s * A.stage_bytes, smem + A.rs_base + rr * A.rs_bytes, r, ii, jj, h0);
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&agen[s]);
          mbar_arrive(&rs_empty[rr]);
        }
        if (++s == S) {
          s = 0;
          ph ^= 1;
        }
        if (++rr == NR) {
          rr = 0;
          rph ^= 1;
        }
      }
    }
  }

  // Both CTAs stay resident until the pair is done with each other's shared
  // and tensor memory.
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();
  if (warp == 2) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

// Ordered sum of the split segments' partial sums, then the scaling of
// scarflib_srm.f90:847 (segments added in index order: deterministic).
__global__ void tc_split_reduce(const float* __restrict__ partial, int split, long long n, float* field,
                                float scaling) {
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += stride) {
    float v = partial[p];
    for (int sgm = 1; sgm < split; ++sgm) v = __fadd_rn(v, partial[sgm * n + p]);
    field[p] = __fmul_rn(v, scaling);
  }
}

int ilog2(int v) {
  int s = 0;
  while ((1 << s) < v) ++s;
  return s;
}

// 512 harmonics per chunk keeps the accumulation error of the tensor core
// below ~4e-6 of the field's standard deviation at any harmonic count.
constexpr int kDefaultChunkStages = 32;
int g_chunk_stages = kDefaultChunkStages;
int g_variant = kTcVariantSingle;
int g_prec_bf16 = 1, g_prec_terms = 3;  // operand precision of plans made from now on (BF16 x 3 by default)

TableJob make_job(const scarf_srm_setup& s, const int fs[3], float ds, const float* d_table, int nh,
                  const TcPlan& p, void* d_work) {
  uint8_t* work = static_cast<uint8_t*>(d_work);
  TableJob T{};
  T.table = d_table;
  T.nh = nh;
  T.stages = p.stages;
  for (int i = 0; i < 9; ++i) T.m[i] = s.m[i];
  for (int i = 0; i < 3; ++i) T.bar[i] = s.bar[i];
  T.ds = ds;
  for (int a = 0; a < 3; ++a) T.off[a] = fs[a] - 1;  // 0-based t -> (t + fs - 1) * ds
  T.ax_r = p.ax_r;
  T.ax_s = p.ax_s;
  T.ax_c = p.ax_c;
  T.n1 = p.n1;
  T.n2 = p.n2;
  T.n3 = p.n3;
  T.ti = p.ti;
  T.tj = p.tj;
  T.bi = p.pair_i ? 2 * p.bix : p.bi;
  T.bj = (p.pair && !p.pair_i) ? 2 * p.bjx : p.bj;
  T.ntile_n = p.ntile_n;
  T.bn = p.bn;
  T.parts = p.pair ? 2 : 1;
  T.bf16 = p.bf16;
  T.rimg = reinterpret_cast<float2*>(work + p.off_r);
  T.simg = reinterpret_cast<float2*>(work + p.off_s);
  T.cimg = work + p.off_c;
  return T;
}

TcField make_field(const scarf_srm_setup& s, const TcPlan& p, const TableJob& T, float* d_field) {
  TcField f{};
  f.n1 = p.n1;
  f.n2 = p.n2;
  f.n3 = p.n3;
  f.sr = p.sr;
  f.ss = p.ss;
  f.sc = p.sc;
  f.bi = p.bi;
  f.bj = p.bj;
  f.bix = p.bix;
  f.bjx = p.bjx;
  f.pair_i = p.pair_i;
  f.bn = p.bn;
  f.split = 1;
  f.band = p.bix;
  f.ntile_n = p.ntile_n;
  f.stages = p.stages;
  f.chunk_stages = std::max(1, p.chunk_stages);
  f.idesc = umma_idesc_f16_f32(p.pair ? 2 * kRows : kRows, static_cast<uint32_t>(p.ntile_n), p.bf16 != 0);
  f.terms = p.terms;
  f.bf16 = p.bf16;
  f.scaling = s.scaling;
  f.rimg = T.rimg;
  f.simg = T.simg;
  f.cimg = T.cimg;
  f.field = d_field;
  return f;
}

constexpr int kMaxDynSmem = 227 * 1024;

// Shared-memory carve-up for a launch with row tiles ti x tj and column
// tiles up to ntile_max; returns the dynamic shared-memory size (0 if the
// ring cannot hold two stages). With A in tensor memory a stage holds only
// the B image and the factor tiles, and the ring depth is the TMEM A ring's;
// a CTA of a pair holds half of the B image.
size_t compute_layout(TcKernelArgs& A, int ti, int tj, int ntile_max, bool tmem_a, bool pair) {
  A.ti = ti;
  A.tj = tj;
  A.ti_shift = ilog2(ti);
  const uint32_t budget = kMaxDynSmem - 1024u - 1024u;
  if (pair) {
    // A / B ring: this CTA's half of the B image, then the A tile (hi, lo).
    A.off_b = 0;
    A.off_a = (ntile_max * kRowBytes + 1023u) & ~1023u;
    A.off_r = A.off_s = 0;
    A.stage_bytes = A.off_a + 2u * kATileBytes;
    // R / S ring: up to 16 stages ahead (at least 4), ~48 KB.
    A.rs_bytes = (kStageHarm * (ti + tj) * 8u + 127u) & ~127u;
    A.nrs = std::max(4, std::min(16, static_cast<int>((48u * 1024u) / A.rs_bytes)));
    const uint32_t rs_total = A.nrs * A.rs_bytes;
    if (rs_total >= budget) return 0;
    const int nbuf = std::min(8, static_cast<int>((budget - rs_total) / A.stage_bytes));
    if (nbuf < 2) return 0;
    A.nstage_buf = nbuf;
    A.rs_base = nbuf * A.stage_bytes;
    A.bars_off = (A.rs_base + rs_total + 7u) & ~7u;
    return 1024 + A.bars_off + (3 * nbuf + 2 * A.nrs + 3 + 2 * kItemRing) * 8 + kItemRing * 4 + 16;
  }
  const uint32_t b_bytes = 2u * ntile_max * kRowBytes;
  A.off_b = 0;
  A.off_a = (b_bytes + 1023u) & ~1023u;
  A.off_r = A.off_a + (tmem_a ? 0u : 2u * kATileBytes);
  A.off_s = A.off_r + kStageHarm * ti * 8u;
  A.stage_bytes = (A.off_s + kStageHarm * tj * 8u + 1023u) & ~1023u;
  const int nbuf = std::min(tmem_a ? kTmemAStages : 8, static_cast<int>(budget / A.stage_bytes));
  if (nbuf < 2) return 0;
  A.nstage_buf = nbuf;
  A.bars_off = nbuf * A.stage_bytes;
  return 1024 + A.bars_off + (3 * nbuf + 3 + 2 * kItemRing) * 8 + kItemRing * 4 + 16;
}

// The kernel's dynamic shared-memory limit, raised once per device so that
// launches themselves make no attribute calls.
template <bool kBf16>
cudaError_t set_smem_attributes() {
  cudaError_t e = cudaFuncSetAttribute(srm_tc_kernel<false, kBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMaxDynSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(srm_tc_kernel<true, kBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(srm_tc_pair_kernel<kBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  return e;
}

cudaError_t ensure_smem_attribute() {
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  e = set_smem_attributes<false>();
  if (e == cudaSuccess) e = set_smem_attributes<true>();
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

int device_sms() {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

// Persistent launch: one CTA (or CTA pair) per SM (pair), at most one per item.
template <bool kBf16>
void launch_tc_kernel_typed(const TcKernelArgs& A, bool tmem_a, bool pair, int nsm, size_t smem, cudaStream_t stream) {
  if (pair) {
    const int pairs = std::max(1, std::min(A.num_items, nsm / 2));
    srm_tc_pair_kernel<kBf16><<<2 * pairs, kThreads, smem, stream>>>(A);
  } else if (tmem_a) {
    srm_tc_kernel<true, kBf16><<<std::min(A.num_items, nsm), kThreads, smem, stream>>>(A);
  } else {
    srm_tc_kernel<false, kBf16><<<std::min(A.num_items, nsm), kThreads, smem, stream>>>(A);
  }
}

void launch_tc_kernel(const TcKernelArgs& A, bool tmem_a, bool pair, int nsm, size_t smem, cudaStream_t stream) {
  if (A.bf16)
    launch_tc_kernel_typed<true>(A, tmem_a, pair, nsm, smem, stream);
  else
    launch_tc_kernel_typed<false>(A, tmem_a, pair, nsm, smem, stream);
}

}  // namespace

int tc_get_variant() { return g_variant; }

void tc_set_variant(int v) { g_variant = v; }

bool tc_set_precision(int bf16, int terms) {
  if ((bf16 != 0 && bf16 != 1) || (terms != 2 && terms != 3)) return false;
  g_prec_bf16 = bf16;
  g_prec_terms = terms;
  return true;
}

void tc_set_chunk_harmonics(int harmonics) {
  g_chunk_stages = harmonics > 0 ? (harmonics + kStageHarm - 1) / kStageHarm : kDefaultChunkStages;
}

bool tc_make_plan(int ndim, const int n[3], int nh, TcPlan* P, int tj_force, bool permute, int variant, int split) {
  if (nh <= 0 || n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return false;
  TcPlan p{};
  // Rows (i, j) over two axes, columns k over the third. By default k = z
  // (y in 2D, whose single z plane becomes j) and i = x. With `permute` the
  // longest axis becomes the column axis (ties keep z, then y), for wide
  // column tiles: generation and the per-instruction MMA cost amortise over
  // more columns. The rows take the other two axes, the faster-varying one as
  // i; with x as the column axis the field stores are strided, a small cost
  // next to the sum.
  int ax_c = (ndim == 3) ? 2 : 1;
  if (permute) {
    const int cand[3] = {ax_c, ax_c == 2 ? 1 : 2, 0};  // preference on ties
    for (int c : cand)
      if (c < (ndim == 3 ? 3 : 2) && n[c] > n[ax_c]) ax_c = c;
  }
  p.ax_c = ax_c;
  p.ax_r = (ax_c == 0) ? 1 : 0;
  p.ax_s = (ax_c == 2) ? 1 : 2;
  const long long stride[3] = {1, n[0], static_cast<long long>(n[0]) * n[1]};
  p.n1 = n[p.ax_r];
  p.n2 = n[p.ax_s];
  p.n3 = n[p.ax_c];
  p.sr = stride[p.ax_r];
  p.ss = stride[p.ax_s];
  p.sc = stride[p.ax_c];
  if (tj_force > 0) {
    if (tj_force > kRows || (tj_force & (tj_force - 1))) return false;
    p.tj = tj_force;
  } else {
    p.tj = 1;
    while (p.tj < 8 && p.tj * 2 <= p.n2) p.tj *= 2;
  }
  p.ti = kRows / p.tj;
  p.bi = (p.n1 + p.ti - 1) / p.ti;
  p.bj = (p.n2 + p.tj - 1) / p.tj;
  const int form = (variant >= 0) ? variant : g_variant;
  p.pair = form == kTcVariantPair ? 1 : 0;
  p.tmem_a = form == kTcVariantSingleTmemA ? 1 : 0;
  p.pair_i = (p.pair && p.bj == 1) ? 1 : 0;  // one row block along j (2D): pair along i
  p.bix = (p.pair && p.pair_i) ? (p.bi + 1) / 2 : p.bi;
  p.bjx = (p.pair && !p.pair_i) ? (p.bj + 1) / 2 : p.bj;
  const int max_n = p.tmem_a ? kMaxNTmemA : kMaxNSmemA;
  const int n3_16 = (p.n3 + 15) / 16 * 16;
  p.bn = (n3_16 + max_n - 1) / max_n;
  p.ntile_n = ((p.n3 + p.bn - 1) / p.bn + 15) / 16 * 16;
  p.bf16 = g_prec_bf16;
  p.terms = g_prec_terms;
  p.nh = nh;
  p.nh_pad = (nh + kStageHarm - 1) / kStageHarm * kStageHarm;
  p.stages = p.nh_pad / kStageHarm;
  p.chunk_stages = g_chunk_stages;
  auto align = [](size_t v) { return (v + 255) / 256 * 256; };
  size_t off = 0;
  p.off_r = off;
  off = align(off + static_cast<size_t>(p.pair_i ? 2 * p.bix : p.bi) * p.stages * kStageHarm * p.ti * sizeof(float2));
  p.off_s = off;
  off = align(off + static_cast<size_t>((p.pair && !p.pair_i) ? 2 * p.bjx : p.bj) * p.stages * kStageHarm * p.tj *
                        sizeof(float2));
  p.off_c = off;
  off = align(off + static_cast<size_t>(p.bn) * p.stages * 2 * p.ntile_n * kRowBytes);
  // Harmonic split (single-CTA forms; at most one segment per stage).
  p.split = std::max(1, std::min(split, p.stages));
  if (p.pair) p.split = 1;
  p.off_partial = off;
  if (p.split > 1)
    off = align(off + sizeof(float) * static_cast<size_t>(p.split) * n[0] * n[1] * n[2]);
  p.off_status = off;  // status word, then the work-queue counter
  off = align(off + 256);
  p.bytes = off;
  *P = p;
  return true;
}

void tc_slab_layout(const TcPlan& p, int target_items, TcSlabSignal* sig) {
  sig->jbs = std::max(1, std::min(p.bj, target_items / std::max(1, p.bi)));
  sig->spn = (p.bj + sig->jbs - 1) / sig->jbs;
  sig->nslabs = sig->spn * p.bn;
}

TcSlab tc_slab_extent(const TcPlan& p, const TcSlabSignal& sig, int q) {
  const int nt = q / sig.spn, jb0 = (q % sig.spn) * sig.jbs;
  TcSlab e;
  e.z0 = nt * p.ntile_n;
  e.z1 = std::min(p.n3, e.z0 + p.ntile_n);
  e.y0 = jb0 * p.tj;
  e.y1 = std::min(p.n2, (jb0 + sig.jbs) * p.tj);
  return e;
}

// Item order of a single-field launch. The items in flight at once (one per
// SM, or per CTA pair) each stream their R, S and C factor tiles through all
// harmonics; in natural order they cover every row block along i, and the
// tiles of one wave of items overflow L2 before the next wave reads them
// again. In bands of g row blocks along i, consecutive waves share the band's
// R tiles and the column tile's C tiles, which then stay in L2. The widest g
// whose per-wave footprint fits in 3/4 of L2 is taken (natural order when
// even one row block's does not); SCARF3D_B200_ITEM_BAND overrides it.
int tc_item_band(const TcPlan& p, int nsm) {
  if (const char* e = std::getenv("SCARF3D_B200_ITEM_BAND")) {
    const int g = std::atoi(e);
    if (g > 0) return g;
  }
  static int l2 = -1;
  if (l2 < 0) {
    int dev = 0, v = 0;
    l2 = (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev) == cudaSuccess)
             ? v
             : 0;
  }
  if (l2 <= 0) return p.bix;
  const int conc = std::max(1, p.pair ? nsm / 2 : nsm);
  const double rb = 16.0 * p.ti * sizeof(float2) * ((p.pair && p.pair_i) ? 2 : 1);
  const double sb = 16.0 * p.tj * sizeof(float2) * ((p.pair && !p.pair_i) ? 2 : 1);
  const double cb = 2.0 * p.ntile_n * kRowBytes;
  auto footprint = [&](int g) {
    const int jbs = std::min(p.bjx, (conc + g - 1) / g);
    return static_cast<double>(p.stages) * (g * rb + jbs * sb + cb);
  };
  const double limit = 0.75 * static_cast<double>(l2);
  if (footprint(p.bix) <= limit) return p.bix;
  int g = 1;
  while (2 * g < p.bix) g *= 2;
  for (; g >= 1; g /= 2)
    if (footprint(g) <= limit) return g;
  return p.bix;
}

long long tc_stat_records(const TcPlan& p) {
  return static_cast<long long>(p.bix) * p.bjx * p.bn * (p.pair ? 8 : 4);
}

cudaError_t launch_tc_structured(const scarf_srm_setup& s, const int fs[3], const int n[3], float ds,
                                 const float* d_table, int nh, float* d_field, void* d_work, const TcPlan& p,
                                 int* d_status, cudaStream_t stream, cudaEvent_t ev_main0, cudaEvent_t ev_main1,
                                 const TcSlabSignal* slabs, StatRecord* d_stats) {
  const TableJob T = make_job(s, fs, ds, d_table, nh, p, d_work);
  const int nsm = device_sms();
  launch_table_builders(T, nullptr, 1, p.stages, factor_smem_rs(p), factor_smem_c(p), nsm, stream, p.bf16 != 0);
  cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) return le;

  TcKernelArgs A{};
  A.f0 = make_field(s, p, T, d_field);
  A.bf16 = p.bf16;
  // Slab copies need whole column tiles to finish early: natural order then.
  A.f0.band = (slabs && slabs->nslabs > 0) ? p.bix : tc_item_band(p, nsm);
  const long long npts = static_cast<long long>(n[0]) * n[1] * n[2];
  if (p.split > 1) {
    // Statistics and slab signals need the final values in the kernel.
    if (d_stats || (slabs && slabs->nslabs > 0)) return cudaErrorInvalidValue;
    A.f0.split = p.split;
    A.f0.partial = reinterpret_cast<float*>(static_cast<uint8_t*>(d_work) + p.off_partial);
    A.f0.seg_stride = npts;
  }
  A.f0.stats = d_stats;
  A.fields = nullptr;
  A.items = nullptr;
  A.num_items = p.bix * p.bjx * p.bn * p.split;
  A.status = d_status;
  A.queue = d_status + 1;
  const size_t smem = compute_layout(A, p.ti, p.tj, p.ntile_n, p.tmem_a != 0, p.pair != 0);
  if (!smem) return cudaErrorInvalidConfiguration;
  cudaError_t e = ensure_smem_attribute();
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(A.queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  if (slabs && slabs->nslabs > 0) {
    e = cudaMemsetAsync(slabs->d_cnt, 0, sizeof(int) * slabs->nslabs, stream);
    if (e != cudaSuccess) return e;
    A.slab_cnt = slabs->d_cnt;
    A.slab_flag = slabs->flag_dev;
    A.slab_jbs = slabs->jbs;
    A.slab_spn = slabs->spn;
  }
  if (ev_main0) cudaEventRecord(ev_main0, stream);
  launch_tc_kernel(A, p.tmem_a != 0, p.pair != 0, nsm, smem, stream);
  if (p.split > 1) {
    const long long blocks = std::min<long long>((npts + 255) / 256, static_cast<long long>(nsm) * 16);
    tc_split_reduce<<<static_cast<unsigned>(std::max(1LL, blocks)), 256, 0, stream>>>(A.f0.partial, p.split, npts,
                                                                                       d_field, s.scaling);
  }
  if (ev_main1) cudaEventRecord(ev_main1, stream);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- batches --
size_t tc_batch_plan(const TcBatchInput* in, int nfields, TcBatchPlan* out) {
  TcBatchPlan bp;
  bp.nfields = nfields;
  auto align = [](size_t v) { return (v + 255) / 256 * 256; };
  size_t off = 0;
  bp.off_fields = off;
  off = align(off + sizeof(TcField) * nfields);
  bp.off_jobs = off;
  off = align(off + sizeof(TableJob) * nfields);
  long long items = 0;
  int ti = 0, tj = 0, ntile_max = 16;
  for (int f = 0; f < nfields; ++f) {
    TcPlan p{};
    if (!tc_make_plan(in[f].s->ndim, in[f].n, in[f].nh, &p, in[f].tj, true)) return 0;
    if (f == 0) {
      ti = p.ti;
      tj = p.tj;
      bp.tmem_a = p.tmem_a;
      bp.pair = p.pair;
    } else if (p.ti != ti || p.tj != tj || p.tmem_a != bp.tmem_a || p.pair != bp.pair) {
      return 0;  // one row-tile shape and A placement per launch
    }
    ntile_max = std::max(ntile_max, p.ntile_n);
    items += static_cast<long long>(p.bix) * p.bjx * p.bn;
    bp.field_off.push_back(off);
    bp.plans.push_back(p);
    off = align(off + p.bytes);
  }
  bp.ti = ti;
  bp.tj = tj;
  bp.ntile_max = ntile_max;
  for (const TcPlan& p : bp.plans) {
    bp.smem_rs = std::max(bp.smem_rs, factor_smem_rs(p));
    bp.smem_c = std::max(bp.smem_c, factor_smem_c(p));
    bp.max_stages = std::max(bp.max_stages, p.stages);
  }
  bp.num_items = static_cast<int>(items);
  bp.off_items = off;
  off = align(off + sizeof(int2) * static_cast<size_t>(items));
  bp.off_done = off;
  off = align(off + sizeof(int) * static_cast<size_t>(nfields));
  bp.off_status = off;
  off = align(off + 256);
  bp.bytes = off;
  if (out) *out = bp;
  return bp.bytes;
}

cudaError_t tc_batch_upload(const TcBatchInput* in, const TcBatchPlan& bp, void* d_work, int* done_flags_dev) {
  uint8_t* work = static_cast<uint8_t*>(d_work);
  std::vector<TcField> fields(bp.nfields);
  std::vector<TableJob> jobs(bp.nfields);
  std::vector<int2> items;
  items.reserve(bp.num_items);
  for (int f = 0; f < bp.nfields; ++f) {
    jobs[f] = make_job(*in[f].s, in[f].fs, in[f].ds, in[f].d_table, in[f].nh, bp.plans[f], work + bp.field_off[f]);
    fields[f] = make_field(*in[f].s, bp.plans[f], jobs[f], in[f].d_field);
    const int nit = bp.plans[f].bix * bp.plans[f].bjx * bp.plans[f].bn;
    if (done_flags_dev) {
      fields[f].done_cnt = reinterpret_cast<int*>(work + bp.off_done) + f;
      fields[f].done_flag = done_flags_dev + f;
      fields[f].done_expect = (bp.plans[f].pair ? 8 : 4) * nit;  // epilogue warps per item
    }
    for (int l = 0; l < nit; ++l) items.push_back(make_int2(f, l));
  }
  // Longest items first (the dynamic queue then balances the tail).
  std::stable_sort(items.begin(), items.end(),
                   [&](const int2& a, const int2& b) { return bp.plans[a.x].stages > bp.plans[b.x].stages; });
  cudaError_t e = cudaMemcpy(work + bp.off_fields, fields.data(), sizeof(TcField) * bp.nfields,
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(work + bp.off_jobs, jobs.data(), sizeof(TableJob) * bp.nfields, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(work + bp.off_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = ensure_smem_attribute();
  return e;
}

cudaError_t tc_batch_launch(const TcBatchPlan& bp, void* d_work, cudaStream_t stream, cudaEvent_t ev_main0,
                            cudaEvent_t ev_main1, const BuilderFork* fork) {
  uint8_t* work = static_cast<uint8_t*>(d_work);
  const int nsm = device_sms();
  const TableJob* jobs = reinterpret_cast<const TableJob*>(work + bp.off_jobs);
  TableJob none{};
  int* status = reinterpret_cast<int*>(work + bp.off_status);
  cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(int), stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(work + bp.off_done, 0, sizeof(int) * bp.nfields, stream);  // field completion counts
  if (e != cudaSuccess) return e;
  launch_table_builders(none, jobs, bp.nfields, bp.max_stages, bp.smem_rs, bp.smem_c, nsm, stream,
                        bp.nfields > 0 && bp.plans[0].bf16 != 0, fork);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  TcKernelArgs A{};
  A.fields = reinterpret_cast<const TcField*>(work + bp.off_fields);
  A.bf16 = bp.nfields > 0 ? bp.plans[0].bf16 : 0;
  A.items = reinterpret_cast<const int2*>(work + bp.off_items);
  A.num_items = bp.num_items;
  A.status = status;
  A.queue = status + 1;
  const size_t smem = compute_layout(A, bp.ti, bp.tj, bp.ntile_max, bp.tmem_a != 0, bp.pair != 0);
  if (!smem) return cudaErrorInvalidConfiguration;
  if (ev_main0) cudaEventRecord(ev_main0, stream);
  launch_tc_kernel(A, bp.tmem_a != 0, bp.pair != 0, nsm, smem, stream);
  if (ev_main1) cudaEventRecord(ev_main1, stream);
  return cudaGetLastError();
}

}  // namespace scarf
