// Launchers of the SRM device kernels (host-callable, no allocation inside).
#pragma once

#include <cstddef>
#include <vector>

#include <cuda_runtime.h>

#include "scarf3d_b200.h"

namespace scarf {

// Process-unique id of the current CUDA context (0 when it cannot be read),
// for caches of per-context state (cuda_context.cpp).
unsigned long long current_context_id();

// Statistics records written by the summation kernels when asked for: one
// (count, mean, M2) triple (FP64) per epilogue warp and work item of the
// tensor-core form, or per block of the direct form, merged in record order by
// launch_stats_records (srm_stats.cu). Layout of struct Moments (common.cuh).
struct StatRecord {
  double n, mean, m2;
};

// ---- direct sum (srm_direct.cu) ----
// sin/cos of the direct sum: 1 = Cody-Waite reduction + SFU (default),
// 0 = CUDA's sincosf.
void direct_set_sincos(int fast);
int direct_get_sincos();
// d_stats (optional): direct_stat_records(npts) records.
long long direct_stat_records(long long npts);
cudaError_t launch_direct_structured(const scarf_srm_setup& s, const int fs[3], const int n[3], float ds,
                                     const float* d_table, int nh, float* d_field, int* d_status,
                                     cudaStream_t stream, StatRecord* d_stats = nullptr);
cudaError_t launch_direct_points(const scarf_srm_setup& s, const float* d_x, const float* d_y, const float* d_z,
                                 long long npts, const float* d_table, int nh, float* d_field, int* d_status,
                                 cudaStream_t stream, StatRecord* d_stats = nullptr);

// ---- factorised tensor-core form (srm_tc.cu) ----
// Geometry of one structured field in the factorised form:
//   out[i*sr + j*ss + k*sc] = scale * Re sum_h R_h(i) S_h(j) C_h(k)
// with (i, j, k) along the physical axes (ax_r, ax_s, ax_c): (x, y, z) by
// default ((x, z, y) in 2D, the single z plane as j); a permuting plan takes
// the longest axis as k: (x, z, y) or (y, z, x).
struct TcPlan {
  int n1, n2, n3;        // logical extents
  int ti, tj;            // row tile = ti x tj = 128 rows over (i, j)
  int bi, bj;            // number of row blocks along i and j
  int ntile_n;           // column tile width (multiple of 16, <= 256)
  int bn;                // number of column blocks
  int nh;                // harmonics
  int nh_pad;            // padded to a multiple of the stage size
  int stages;            // nh_pad / kStageHarm
  int chunk_stages;      // stages per TMEM accumulation chunk (FP32 sum of chunks)
  int tmem_a;            // 1: A operand generated into tensor memory (ntile_n <= 192)
  int pair;              // 1: CTA-pair form (M = 256 over two SMs, each holding half of B)
  int pair_i;            // pairs split along i (when bj == 1) instead of j
  int bf16;              // operands split into BF16 (else FP16)
  int terms;             // split products per K step: 3, or 2 (the A-hi x B-lo product dropped)
  int split;             // harmonic segments per tile (1: none)
  int bix, bjx;          // item grid (bi x bj, halved along the pair axis, rounded up)
  int ax_r, ax_s, ax_c;  // physical axis (0 x, 1 y, 2 z) of i (row-fast), j (row-slow), k (column)
  long long sr, ss, sc;  // field strides of i, j, k in elements
  size_t off_r, off_s, off_c, off_partial, off_status, bytes;  // workspace layout
};

// Kernel form for plans made from now on (SCARF_TC_* of scarf3d_b200.h).
constexpr int kTcVariantPair = 0;         // cta_group::2 pairs, A in shared memory
constexpr int kTcVariantSingle = 1;       // one CTA per tile, A in shared memory (default)
constexpr int kTcVariantSingleTmemA = 2;  // one CTA per tile, A in tensor memory
void tc_set_variant(int v);
// Operand precision of plans made from now on: FP16 (bf16 = 0) or BF16 split
// operands, 3 or 2 split products. False for other values.
bool tc_set_precision(int bf16, int terms);
int tc_get_variant();

// tj_force > 0 fixes the row tile to (128 / tj_force) x tj_force.
// permute: let the longest axis be the column axis (device-field entry
// points; the default layout keeps k = z, which the slab copy-out relies on).
// variant >= 0 selects the kernel form (kTcVariant*) instead of the global one.
// split > 1 divides the harmonics over that many work items per tile
// (single-CTA forms), their partial sums reduced in order after the kernel.
bool tc_make_plan(int ndim, const int n[3], int nh, TcPlan* plan, int tj_force = 0, bool permute = false,
                  int variant = -1, int split = 1);

// ---- autotuning (tc_tune.cpp) ----
// A tuned plan choice for one shape bucket (grid extents rounded up to a
// multiple of 16): kernel form, row tile (128 / tile_j) x tile_j, and whether
// the longest axis is the column axis.
struct TcChoice {
  int variant, tile_j, permute;
  float ms;
  int split;  // harmonic segments per tile (device-field plans only)
};
// The tuned choice for a grid when tuned plans are enabled and its bucket has
// an entry (fixed_columns: the caller keeps k = z, as scarf_execute does).
bool tc_tuned_choice(int ndim, const int n[3], bool fixed_columns, TcChoice* c);
// Plan of the device-field entry points (scarf_srm_tc_structured and the
// allocation-free variant): a tuned choice for the grid's bucket when tuned
// plans are enabled, else the default plan with the longest axis as columns.
// The same rule sizes scarf_srm_tc_workspace_bytes.
bool device_field_plan(int ndim, const int n[3], int nh, TcPlan* p);
// Harmonics accumulated in tensor memory before each FP32 drain (rounded up
// to whole pipeline stages); 0 restores the default.
void tc_set_chunk_harmonics(int harmonics);
// Slab-wise completion signal of a single-field launch. Slab q covers column
// tile q / spn and row blocks j in [(q % spn) * jbs, +jbs): rows x columns
// that are one strided block of the column-major field. The kernel sets
// flag[q] = 1 (host-mapped memory) once every item of slab q is stored.
struct TcSlab {
  int z0, z1;  // column (plan axis 3) range
  int y0, y1;  // row-block j range in grid rows (plan axis 2)
};
struct TcSlabSignal {
  int* d_cnt = nullptr;    // >= nslabs device counters (zeroed by the launch)
  int* flag_dev = nullptr; // device address of >= nslabs host-mapped ints, zeroed by the caller
  int jbs = 0, spn = 0, nslabs = 0;
};
// Slab layout of a plan with about target_items work items per slab.
void tc_slab_layout(const TcPlan& p, int target_items, TcSlabSignal* sig);
TcSlab tc_slab_extent(const TcPlan& p, const TcSlabSignal& sig, int q);

// Status word at d_status[0]; d_status[1] is used as the work-queue counter.
// d_stats (optional): tc_stat_records(plan) records of the stored field.
long long tc_stat_records(const TcPlan& plan);
cudaError_t launch_tc_structured(const scarf_srm_setup& s, const int fs[3], const int n[3], float ds,
                                 const float* d_table, int nh, float* d_field, void* d_work, const TcPlan& plan,
                                 int* d_status, cudaStream_t stream, cudaEvent_t ev_main0 = nullptr,
                                 cudaEvent_t ev_main1 = nullptr, const TcSlabSignal* slabs = nullptr,
                                 StatRecord* d_stats = nullptr);

// Batched form: many fields in one persistent launch fed by a device work
// queue. All fields of a batch share one row-tile shape.
struct TcBatchInput {
  const scarf_srm_setup* s;
  int fs[3], n[3];
  float ds;
  const float* d_table;
  int nh;
  float* d_field;
  int tj;  // row-tile shape (0 = automatic)
};
struct TcBatchPlan {
  int nfields = 0, num_items = 0, ti = 0, tj = 0, ntile_max = 0, tmem_a = 0, pair = 0;
  size_t smem_rs = 0, smem_c = 0;  // shared memory of the factored table builders (largest field)
  int max_stages = 0;              // largest stage count of the fields
  size_t off_fields = 0, off_jobs = 0, off_items = 0, off_done = 0, off_status = 0, bytes = 0;
  std::vector<TcPlan> plans;
  std::vector<size_t> field_off;
};
// Workspace bytes (0 if the fields cannot share one launch).
size_t tc_batch_plan(const TcBatchInput* in, int nfields, TcBatchPlan* out);
// Host -> device upload of descriptors, table jobs and the work list
// (synchronous; not for use inside stream capture). With done_flags_dev
// (device address of nfields host-mapped ints) each field raises its flag
// once all of its items are stored.
cudaError_t tc_batch_upload(const TcBatchInput* in, const TcBatchPlan& plan, void* d_work,
                            int* done_flags_dev = nullptr);
// A second stream and two events with which the C-image builder runs beside
// the R/S builder (fork after the stream's prior work, join before the
// persistent kernel); all null: both builders in order on the stream.
struct BuilderFork {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
// Enqueue only: status/queue reset, table builds, persistent kernel.
cudaError_t tc_batch_launch(const TcBatchPlan& plan, void* d_work, cudaStream_t stream,
                            cudaEvent_t ev_main0 = nullptr, cudaEvent_t ev_main1 = nullptr,
                            const BuilderFork* fork = nullptr);

// ---- device side of the harmonic sampler (srm_sampler.cu) ----
struct SampleEntry {
  long long q;  // pair index in the stream
  int flag;     // 1 = accepted, 2 = to be decided on the host
  int pad;
  float r[8];   // pairs q, q+1, q+2, q+3
};
// Bins of the scan's certain-reject test: the first draw's raw output
// y1 < 2^31 falls in bin y1 >> kRejectShift.
constexpr int kRejectShift = 23;
constexpr int kRejectBins = 1 << (31 - kRejectShift);
struct SamplerArgs {
  unsigned long long r0, r1;  // generator state after seeding (pair 0 next)
  const unsigned int* reject; // [kRejectBins] certain-reject thresholds on y2 (NULL: none)
  long long q_begin, q_count;
  int pairs_per_thread;
  long long nthreads;
  float kmin, kmax, cnst, nu, margin;
  int ndim, acf;
  int write;                 // 0: count per thread, 1: write entries
  int* counts;               // [nthreads]
  const long long* offsets;  // [nthreads]
  SampleEntry* out;
  int cap;                   // batch mode 2: candidates per thread slot (keys + t * cap), counts kept in full
  unsigned long long* keys;  // batch mode 2: candidate keys (pair index << 2 | flag)
};
// Output-transform tables of the generator: g^k (k < 2048), g^(k 2^11)
// (k < 2048) and g^(k 2^22) (k < 512) mod 2^31 - 1, 4 608 words in that order.
cudaError_t sampler_upload_tables(const unsigned int* pow3);

// Bounded-wait self-test (srm_selftest.cu): `blocks` blocks wait on an
// mbarrier that nothing arrives on; d_scratch is 16 device bytes. On return
// *status is the status word the waits wrote, *waited_ns the longest wait,
// and *timed_out whether a wait ran out and said so.
cudaError_t run_wait_limit_probe(int blocks, void* d_scratch, cudaStream_t stream, int* status,
                                 unsigned long long* waited_ns, bool* timed_out);
cudaError_t launch_sampler(const SamplerArgs& args, cudaStream_t stream);
// One pass for each of nfields fields in a single launch: d_fields[f] holds
// field f's pass (its counts / offsets pointers already at the field's slice),
// d_tbeg the prefix of the fields' thread counts (nfields + 1 entries).
cudaError_t launch_sampler_batch(const SamplerArgs* d_fields, const long long* d_tbeg, int nfields, long long total,
                                 int write, cudaStream_t stream);
// Compaction after a write = 2 batch pass (see SamplerArgs::cap): each
// kept key becomes a full entry, its draws regenerated from the stream.
cudaError_t launch_sampler_gather(const SamplerArgs* d_fields, const long long* d_tbeg, int nfields, long long total,
                                  const long long* d_offsets, SampleEntry* d_dst, cudaStream_t stream);

// ---- statistics and post-processing (srm_stats.cu) ----
size_t stats_partials_bytes(long long n);
// Two passes (mean, then centred sums) in FP64; writes mean/var (FP32
// results as the reference returns them) to d_out[0..1] (float).
cudaError_t launch_field_stats(const float* d_field, long long n, double* d_partials, float* d_out,
                               cudaStream_t stream);
// Merge `count` statistics records in record order (one block, fixed tree)
// into the FP32 mean and unbiased variance at d_out[0..1], as
// launch_field_stats reports them.
cudaError_t launch_stats_records(const StatRecord* d_rec, long long count, float* d_out, cudaStream_t stream);
// Rescale (when rescale != 0, scarflib_srm.f90:897-912) and the taper of
// every point of interest (scarflib_common.f90:881-994), in the reference's
// order, in one pass over the field. d_poi: npoi x 3 floats.
// Structured fields (d_x null) take coordinates (i + fs - 2) dh from the
// index; point sets read d_x, d_y, d_z.
struct FinalizeArgs {
  int rescale;
  float scaling, mean;  // field * scaling - mean
  const float* d_poi;
  int npoi;
  float mute, taper;
  int n0, n1, o0, o1, o2;  // structured: extents and fs - 1
  float dh;
  const float *d_x, *d_y, *d_z;
};
cudaError_t launch_finalize_field(float* d_field, long long n, const FinalizeArgs& a, cudaStream_t stream);

// ---- FIM, the Fourier integral method (fim.cu) ----
struct FimInputs {
  int ndim, acf, pad, rescale, seed;
  float ds, dh, sigma, hurst, mute, taper;
  float cl[3], nc[3], fc[3];  // nc/fc: extent of the external points (the internal grid covers it)
  int structured;             // 1: external grid fs..fe at step ds; 0: the points d_x, d_y, d_z
  int fs[3], fe[3];
  const float *d_x, *d_y, *d_z;
  long long npts;
  const float* poi;  // host, npoi points of poi_stride floats
  int npoi, poi_stride;
};
// Internal (FFT) grid: points per axis, offset of its first node, and the
// reference's info(1:2) flags (scarflib_fim.f90:787-818).
struct FimGrid {
  int npts[3];
  float off_axis[3];
  float info0, info1;
};
void fim_grid(const FimInputs& in, FimGrid* g);
size_t fim_workspace_bytes(const FimGrid& g, int npoi);
// The whole FIM into the device field of the external points; stats as the
// reference's info(1:8). d_work: fim_workspace_bytes, 256-byte aligned. On
// failure *what names the failing step. Synchronises `st`.
cudaError_t fim_run(const FimInputs& in, const FimGrid& g, void* d_work, float* d_field, float stats[8],
                    cudaStream_t st, const char** what);
// Frees the FIM's cached cuFFT plans of the current device.
void release_fim_plans();

}  // namespace scarf
