// Device side of the harmonic sampler: the rejection tests of the sampling
// loop (scarflib_srm.f90:731-745) evaluated for a whole range of uniform
// pairs at once.
//
// Thread t owns pairs [q0, q0 + P) of the stream, jumps a copy of the
// generator to draw 2*q0 and tests each pair exactly as the host does: the
// same integer recursion and output power, the same float mapping, u in FP32
// with the reference's operation order. Only the spectrum (powf / expf) may
// differ from the host's libm by a few ulps, so a decision whose margin
// |r2 - d| is below a relative bound that covers those ulps is flagged
// "uncertain" and left to the host. Certain rejections are dropped; accepted
// and uncertain pairs are written, in stream order, with the raw floats of
// the pair and of the three pairs that follow it (angles, a, b), which is
// everything the host walk needs.
//
// Most pairs are certain rejections that the raw draws already show: the
// host gives each field a table of thresholds on y2 per bin of y1 (an upper
// bound of the spectrum over the bin's u interval, with room for the FP32
// evaluation), and a pair with y2 at or above its bin's threshold is dropped
// before any floating-point work. Every other pair takes the full test, so
// the decisions are those of the full test for every pair.
//
// Two passes over the same range: the first counts candidates per thread,
// the host turns the counts into offsets, the second writes them.
//
// The generator (yarn2.cuh) evaluates its output transform from 18 KB of
// tables that every block holds in shared memory: two large tables in global
// memory made each draw two dependent random L2 reads, which bounded the
// scan.
#include <cuda_runtime.h>

#include <cstdint>

#include "srm_kernels.h"
#include "yarn2.cuh"

namespace scarf {
namespace {

using namespace yarn2;

__device__ uint32_t g_pow[kPowWords];  // g^k, g^(k 2^11), g^(k 2^22) mod m

// The block's copy of g_pow in shared memory.
__device__ __forceinline__ void load_pow(uint32_t* sp) {
  for (int i = threadIdx.x; i < kPowWords; i += blockDim.x) sp[i] = g_pow[i];
  __syncthreads();
}

// 0 = certain reject, 1 = certain accept, 2 = uncertain.
__device__ __forceinline__ int classify(const SamplerArgs& A, float r1, float r2) {
  const float u = __fadd_rn(__fmul_rn(r1, __fsub_rn(A.kmax, A.kmin)), A.kmin);
  float fv;
  if (A.acf == 0) {
    fv = __fdiv_rn(1.0f, powf(__fadd_rn(1.0f, __fmul_rn(u, u)), A.nu));
  } else {
    fv = expf(__fmul_rn(-0.25f, __fmul_rn(u, u)));
  }
  double srm = static_cast<double>(u) * static_cast<double>(fv);
  if (A.ndim == 3) srm = srm * static_cast<double>(u);
  const float d = static_cast<float>(srm * static_cast<double>(A.cnst));
  if (r2 < d * (1.0f - A.margin)) return 1;
  if (r2 >= d * (1.0f + A.margin)) return 0;
  return 2;
}

// Pairs [q0, q1) of local thread t of one field's pass: count (write = 0),
// write the candidate entries at the thread's offset (write = 1), or write
// up to A.cap candidate keys (pair index << 2 | flag, 8 bytes) into the
// thread's own slot keys + t * cap while counting them all (write = 2: one
// scan instead of two; a count above cap tells the host to redo that field;
// the gather launch rebuilds full entries from the keys).
__device__ __forceinline__ void sample_range(const SamplerArgs& A, long long t, int write, const uint32_t* sp,
                                             const uint32_t* thr) {
  const long long q0 = A.q_begin + t * A.pairs_per_thread;
  long long q1 = q0 + A.pairs_per_thread;
  if (q1 > A.q_begin + A.q_count) q1 = A.q_begin + A.q_count;
  Gen g{A.r0, A.r1, sp};
  g.jump(2ull * static_cast<uint64_t>(q0));
  int count = 0;
  long long slot = write == 1 ? A.offsets[t] : (write == 2 ? t * A.cap : 0);
  const long long slot_end = write == 2 ? slot + A.cap : (1ll << 62);
  const int npairs = q1 > q0 ? static_cast<int>(q1 - q0) : 0;  // at most pairs_per_thread
  for (int i = 0; i < npairs; ++i) {
    const uint32_t y1 = g.next();
    const uint32_t y2 = g.next();
    if (thr && y2 >= thr[y1 >> kRejectShift]) continue;
    const long long q = q0 + i;
    const float r1 = to_u01(y1);
    const float r2 = to_u01(y2);
    const int c = classify(A, r1, r2);
    if (c == 0) continue;
    ++count;
    if (write == 2) {
      if (slot < slot_end) A.keys[slot++] = (static_cast<unsigned long long>(q) << 2) | static_cast<unsigned>(c);
    } else if (write && slot < slot_end) {
      SampleEntry e;
      e.q = q;
      e.flag = c;
      e.r[0] = r1;
      e.r[1] = r2;
      Gen look = g;  // the three pairs after q, without disturbing the scan
      for (int k = 2; k < 8; ++k) e.r[k] = to_u01(look.next());
      A.out[slot++] = e;
    }
  }
  if (write != 1) A.counts[t] = count;
}

__global__ void sampler_kernel(const SamplerArgs A) {
  __shared__ uint32_t sp[kPowWords];
  __shared__ uint32_t sthr[kRejectBins];
  if (A.reject)
    for (int i = threadIdx.x; i < kRejectBins; i += blockDim.x) sthr[i] = A.reject[i];
  load_pow(sp);
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= A.nthreads) return;
  sample_range(A, t, A.write, sp, A.reject ? sthr : nullptr);
}

// The field f with tbeg[f] <= t < tbeg[f + 1] (binary search over the prefix).
__device__ __forceinline__ int field_of(const long long* tbeg, int nfields, long long t) {
  int lo = 0, hi = nfields - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tbeg[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Passes of many fields in one launch: global thread t belongs to field
// field_of(t). The block keeps the reject thresholds of its first thread's
// field and of the next field in shared memory (a block spans at most those
// two unless fields have fewer threads than a block; threads of any further
// field read their field's table from global memory).
__global__ void sampler_batch_kernel(const SamplerArgs* fields, const long long* tbeg, int nfields,
                                     long long total, int write) {
  __shared__ uint32_t sp[kPowWords];
  __shared__ uint32_t sthr[2][kRejectBins];
  const long long tb = static_cast<long long>(blockIdx.x) * blockDim.x;
  const int f0 = field_of(tbeg, nfields, tb);
  for (int i = threadIdx.x; i < 2 * kRejectBins; i += blockDim.x) {
    const int f = f0 + i / kRejectBins;
    const uint32_t* src = f < nfields ? fields[f].reject : nullptr;
    sthr[i / kRejectBins][i % kRejectBins] = src ? src[i % kRejectBins] : 0xFFFFFFFFu;
  }
  load_pow(sp);
  const long long t = tb + threadIdx.x;
  if (t >= total) return;
  const int f = field_of(tbeg, nfields, t);
  const SamplerArgs A = fields[f];
  const uint32_t* thr = f - f0 < 2 ? sthr[f - f0] : A.reject;
  sample_range(A, t - tbeg[f], write, sp, thr);
}

// Compacts the per-thread slots of a write = 2 pass: thread t's min(count,
// cap) keys become entries at dst + offsets[t] (global thread index t), the
// pair and the three after it drawn again by jumping a generator copy from
// one candidate to the next.
__global__ void sampler_gather_kernel(const SamplerArgs* fields, const long long* tbeg, int nfields, long long total,
                                      const long long* offsets, SampleEntry* dst) {
  __shared__ uint32_t sp[kPowWords];
  load_pow(sp);
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int lo = field_of(tbeg, nfields, t);
  const SamplerArgs& A = fields[lo];
  const long long tl = t - tbeg[lo];
  const int n = min(A.counts[tl], A.cap);
  const unsigned long long* src = A.keys + tl * A.cap;
  SampleEntry* o = dst + offsets[t];
  Gen g{A.r0, A.r1, sp};
  unsigned long long at = 0;  // draw index g stands at; keys ascend in q
  for (int i = 0; i < n; ++i) {
    const unsigned long long key = src[i];
    const unsigned long long q = key >> 2;
    g.jump(2ull * q - at);
    at = 2ull * q;
    SampleEntry e;
    e.q = static_cast<long long>(q);
    e.flag = static_cast<int>(key & 3u);
    e.pad = 0;
    Gen look = g;  // candidates may follow each other within 4 pairs
    for (int k = 0; k < 8; ++k) e.r[k] = to_u01(look.next());
    o[i] = e;
  }
}

}  // namespace

cudaError_t sampler_upload_tables(const uint32_t* pow3) {
  return cudaMemcpyToSymbol(g_pow, pow3, sizeof(uint32_t) * kPowWords);
}

cudaError_t launch_sampler_batch(const SamplerArgs* d_fields, const long long* d_tbeg, int nfields, long long total,
                                 int write, cudaStream_t stream) {
  const int block = 128;
  const long long blocks = (total + block - 1) / block;
  if (blocks <= 0 || nfields <= 0) return cudaSuccess;
  sampler_batch_kernel<<<static_cast<unsigned>(blocks), block, 0, stream>>>(d_fields, d_tbeg, nfields, total, write);
  return cudaGetLastError();
}

cudaError_t launch_sampler_gather(const SamplerArgs* d_fields, const long long* d_tbeg, int nfields, long long total,
                                  const long long* d_offsets, SampleEntry* d_dst, cudaStream_t stream) {
  const int block = 128;
  const long long blocks = (total + block - 1) / block;
  if (blocks <= 0 || nfields <= 0) return cudaSuccess;
  sampler_gather_kernel<<<static_cast<unsigned>(blocks), block, 0, stream>>>(d_fields, d_tbeg, nfields, total,
                                                                             d_offsets, d_dst);
  return cudaGetLastError();
}

cudaError_t launch_sampler(const SamplerArgs& A, cudaStream_t stream) {
  const int block = 128;
  const long long blocks = (A.nthreads + block - 1) / block;
  if (blocks <= 0) return cudaSuccess;
  sampler_kernel<<<static_cast<unsigned>(blocks), block, 0, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace scarf
