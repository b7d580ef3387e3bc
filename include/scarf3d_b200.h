/*
 * scarf3d_b200.h -- extended C ABI of the B200 SRM library.
 *
 * The reference-compatible entry points (scarf_opt_init, scarf_cart_initialize,
 * scarf_nocart_initialize, scarf_execute, scarf_finalize, scarf_io_one,
 * scarf_io_slice) are declared in scarf3d.h. This header adds status-returning
 * variants, configuration the reference fixes at compile time, and the
 * building blocks of the SRM path (setup, sampler, device sums, statistics)
 * with plain pointers and sizes. Device pointers are CUDA device addresses of
 * the current device; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).
 *
 * Every int-returning function returns SCARF_OK (0) or a negative status and
 * records a message readable with scarf_last_error() (per thread).
 */
#ifndef SCARF3D_B200_H_
#define SCARF3D_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCARF_OK 0
#define SCARF_ERR_ARG (-1)         /* invalid argument                          */
#define SCARF_ERR_STATE (-2)       /* call order (execute before initialize ...) */
#define SCARF_ERR_CUDA (-3)        /* CUDA runtime error                        */
#define SCARF_ERR_UNSUPPORTED (-4) /* e.g. method = FIM, acf = user-defined      */
#define SCARF_ERR_DEVICE (-5)      /* a kernel reported a stalled pipeline       */
#define SCARF_ERR_NOMEM (-6)       /* host or device allocation failed           */

/* Summation form used by scarf_execute / scarf_execute_ex. */
#define SCARF_FORM_AUTO 0   /* tensor-core form for structured grids, else direct */
#define SCARF_FORM_DIRECT 1 /* FP32 direct sum (any point set)                    */
#define SCARF_FORM_TC 2     /* factorised tcgen05 split-16-bit form (structured)   */

/* Flags for scarf_execute_ex. */
#define SCARF_FIELD_ON_DEVICE 1    /* `field` is a device pointer (no D2H copy)      */
#define SCARF_TAPER_UNSTRUCTURED 2 /* apply POI taper on unstructured meshes too    */

/* SRM inputs (scarflib.f90:67-87, SRM fields only). cl[2] <= 0 selects 2D. */
typedef struct scarf_srm_params {
  int acf;     /* 0 = von Karman, 1 = Gaussian                        */
  int nharm;   /* number of harmonics (reference constant: 10000)     */
  int seed;
  int rescale; /* 1 = rescale discrete std to sigma                   */
  float hurst, sigma, ds, dh;
  float cl[3], nc[3], fc[3];
  float alpha, beta, gamma; /* rotation angles, degrees           */
} scarf_srm_params;

/* Derived scalars (scarflib_srm.f90:617-720). m is row-major
 * (m[3*r+c] = matrix(r+1,c+1)). scaling includes the quadrature ratio. */
typedef struct scarf_srm_setup {
  int ndim;
  float kmin, kmax, kc, nu, cnst, scaling, scaling0;
  float m[9];
  float bar[3];
  float info0, info1;
  float intg_band, intg_full;
  int ier_band, ier_full;
} scarf_srm_setup;

const char *scarf_last_error(void);

/* ---- configuration of the reference-compatible API ---------------------- */
/* Harmonic count (replaces the constant nharm = 10000, scarflib_srm.f90:90). */
int scarf_set_nharm(int nharm);
int scarf_get_nharm(void);
/* SCARF_FORM_*. */
int scarf_set_form(int form);
/* Install the reference's own uniform source (prng.cpp set_seed / srng,
 * TRNG4 yarn2 + uniform01_dist<>) so that harmonics are drawn exactly as
 * the reference draws them. NULL, NULL restores the built-in generator. */
int scarf_set_uniform_source(void (*set_seed)(int), void (*srng)(float *));
/* Stream for all device work of the reference-compatible API. */
int scarf_set_stream(void *stream);
/* Host threads for the sampler (0 = automatic). */
int scarf_set_host_threads(int nthreads);
/* When enabled, the dominant summation kernel of each call is bracketed by
 * CUDA events on its launch stream; scarf_last_kernel_ms() returns the last
 * such duration in milliseconds. */
int scarf_set_kernel_timing(int enable);
float scarf_last_kernel_ms(void);
/* Cap on the device memory the library allocates for itself (tables,
 * staging fields, sampler and tuning scratch), summed over all devices;
 * 0 = no cap (default). A call that would pass the cap fails with
 * SCARF_ERR_NOMEM and leaves the library usable; buffers the caller passes
 * in (device fields, batch workspaces) do not count. Buffers are kept
 * between calls and only grow, so the cap bounds the high-water mark. */
int scarf_set_device_memory_cap(size_t bytes);
/* Device bytes the library holds now. */
size_t scarf_device_memory_in_use(void);
/* Frees the device buffers the library keeps between calls (they are
 * allocated again on demand), and the FIM's cuFFT plans of the current
 * device (kept between calls; their work areas are cuFFT's own allocations,
 * outside the cap); waits for the library's device work first. */
int scarf_release_device_memory(void);
/* Self-test of the bounded waits inside every pipeline kernel: `blocks`
 * blocks (1..1024) wait on an mbarrier that nothing arrives on, through the
 * same bounded wait (limit 2 s) the pipeline kernels use. Returns SCARF_OK
 * when a wait ran out and wrote the timeout code into the status word, as
 * designed; *device_status (if non-NULL) receives the status word and
 * *waited_s (if non-NULL) the longest wait in seconds. Nothing faults: the
 * context stays usable. No counterpart in the reference. */
int scarf_selftest_wait_limit(int blocks, int *device_status, double *waited_s);
/* Harmonics accumulated in tensor memory before each FP32 drain of the
 * tensor-core form (0 = default, 512). The tensor core's FP32 accumulation
 * does not round to nearest, so its error grows with this length. */
int scarf_set_tc_chunk(int harmonics);

/* Host-field output of scarf_execute on a structured mesh with the
 * tensor-core form, no rescale and no taper: the field is copied to the host
 * in slabs (a column tile x a run of row blocks, about items_per_slab work
 * items of 128 x <=256 points each) while the kernel computes the rest.
 * 1 = default slab size (64 items), >= 2 = that size, 0 = copy the whole
 * field after the kernel. The field is identical either way. */
int scarf_set_output_overlap(int items_per_slab);

/* Kernel form of the tensor-core sum, for plans made after the call. All
 * give identical sums (the same products accumulated in the same order per
 * output point).
 *   SCARF_TC_SINGLE       (default) one CTA per 128-row tile, A in shared
 *                         memory;
 *   SCARF_TC_PAIR         a cluster of two CTAs per 256-row tile,
 *                         cta_group::2 MMAs, each SM staging half of B;
 *   SCARF_TC_SINGLE_TMEM_A one CTA per tile, A in tensor memory (column
 *                         tiles <= 192). */
#define SCARF_TC_PAIR 0
#define SCARF_TC_SINGLE 1
#define SCARF_TC_SINGLE_TMEM_A 2
int scarf_set_tc_variant(int variant);
/* Operand precision of the tensor-core form for plans made afterwards (no
 * counterpart in the reference, which sums in FP32). Each FP32 operand is
 * split into hi + lo 16-bit parts, operand_type SCARF_TC_BF16 (default) or
 * SCARF_TC_FP16, and terms = 3 (hi.hi + hi.lo + lo.hi, default) or 2 (hi.hi +
 * lo.hi) products are accumulated in FP32. Measured against FP64 over whole
 * fields (512^3 x 20 000 and 2048x2048x512 x 50 000): BF16 x 3 ~5e-6 rel-RMS,
 * FP16 x 3 ~3.6e-6 at ~2.5 % more time under the power cap; both meet 1e-5.
 * Two products miss it (FP16 ~1.6e-4, BF16 ~1.3e-3). */
#define SCARF_TC_FP16 0
#define SCARF_TC_BF16 1
int scarf_set_tc_precision(int operand_type, int terms);

/* Autotuning of the tensor-core form. No counterpart in the reference (its
 * SRM has one CPU code path). A tuning times every candidate plan -- kernel
 * form (SCARF_TC_*), row tile (128 / tile_j) x tile_j with tile_j in
 * {1, 2, 4, 8, 16}, and for device fields whether the longest axis is the
 * column axis -- on the caller's grid and harmonic table (at most 2 048
 * harmonics of it; table builds and kernel), on the current GPU, and records
 * the fastest for the grid's shape bucket (extents rounded up to a multiple
 * of 16, per GPU name and driver); the default plan is kept unless a
 * candidate beats it by 3 %. With scarf_set_tc_autotune(1), plans made afterwards
 * (scarf_srm_tc_workspace_bytes / scarf_srm_tc_structured, and
 * scarf_execute for fixed_columns = 1 tunings) follow the recorded choice
 * of their bucket; other buckets keep the default plans. Tuned plans compute
 * the same sum; a different column axis changes how the per-axis factors
 * combine, so results may differ at the rounding level (within the
 * tensor-core tolerance). The tuning allocates its own device scratch. */
typedef struct scarf_tc_tuning {
  int variant; /* SCARF_TC_*                                     */
  int tile_j;  /* row tile (128 / tile_j) x tile_j                */
  int permute; /* 1: longest axis as column axis (device fields)  */
  float ms;    /* kernel time of the chosen plan on the probe      */
  int split;   /* harmonic segments per tile (1: none; device fields) */
} scarf_tc_tuning;
/* 0 = default plans (the initial state), 1 = follow recorded tunings. */
int scarf_set_tc_autotune(int mode);
/* Tunings are also appended to this text file and read from it now (NULL:
 * memory only). */
int scarf_set_tc_tune_cache(const char *path);
/* The plan scarf_srm_tc_structured would use for this grid now (ms = 0;
 * permute = 1 when the column axis is not z, or y in 2D). */
int scarf_srm_tc_plan_info(int ndim, const int n[3], int nh, scarf_tc_tuning *out);
/* Tune one structured grid (device table, nh rows); fixed_columns = 1 keeps
 * z as the column axis (the layout scarf_execute uses). */
int scarf_srm_tc_autotune(const scarf_srm_setup *s, const int fs[3], const int n[3], float ds, const float *d_table,
                          int nh, int fixed_columns, void *stream, scarf_tc_tuning *out);

/* The FIM's internal (FFT) grid for a domain nc..fc (no counterpart in the
 * reference; it lets a caller size the device memory of method 0): points
 * per axis, offset of the first node, and the reference's info(1:2) flags
 * (scarflib_fim.f90:787-818). ndim 2 or 3; pad as scarf_opt.pad. */
int scarf_fim_internal_grid(int ndim, const float nc[3], const float fc[3], float dh, const float cl[3], int pad,
                            int npts[3], float off_axis[3], float flags[2]);
/* Device bytes the FIM workspace of that grid takes (spectrum, transform
 * output, statistics records, points of interest; cuFFT's own work area
 * comes on top). */
size_t scarf_fim_workspace_bytes(const int npts[3], int npoi);

/* Status-returning scarf_execute (c_binding.c:138-143); stats[8] as the
 * reference fills it (stats[4] host seconds, stats[5] device seconds). */
int scarf_execute_ex(int seed, float *field, float stats[8], int flags);

/* ---- contexts (no counterpart in the reference) ---------------------------
 * A context is one independent library instance: the object that an
 * initialize call sets up (scarflib.f90:87 keeps one for the whole process),
 * the scarf_set_* settings that shape an execute (nharm, form, stream, host
 * threads, sampler, uniform source, kernel timing, output overlap) and the
 * device buffers of its execute path. Every thread starts on the process-wide
 * default context, on which the reference-compatible API acts; a thread that
 * makes another context current runs every entry point of this header and of
 * scarf3d.h on it. Entry points are serialised inside the library, so any
 * thread may call them; contexts let several meshes stay initialised at once
 * (one per context) and give each thread its own. The kernel-form settings
 * (scarf_set_tc_variant, _precision, _chunk, _autotune, scarf_set_direct_sincos)
 * stay process-wide. */
struct scarf_opt;
typedef struct scarf_ctx scarf_ctx;
scarf_ctx *scarf_ctx_create(void);
/* Finalises the context and frees its device buffers; NULL and the default
 * context are ignored. A calling thread that had it current returns to the
 * default; no other thread may still have it current. */
void scarf_ctx_destroy(scarf_ctx *ctx);
/* Makes ctx the calling thread's current context (NULL: the default). */
int scarf_ctx_make_current(scarf_ctx *ctx);
/* scarf_cart_initialize, scarf_nocart_initialize, scarf_execute_ex and
 * scarf_finalize on an explicit context, with a status. */
int scarf_ctx_cart_initialize(scarf_ctx *ctx, int nd, const int fs[], const int fe[], float ds, int acf,
                              const float cl[], float sigma, const struct scarf_opt *opt);
int scarf_ctx_nocart_initialize(scarf_ctx *ctx, int nd, int npts, const float *x, const float *y, const float *z,
                                float dh, int acf, const float cl[], float sigma, const struct scarf_opt *opt);
int scarf_ctx_execute(scarf_ctx *ctx, int seed, float *field, float stats[8], int flags);
int scarf_ctx_finalize(scarf_ctx *ctx);

/* ---- building blocks ----------------------------------------------------- */
int scarf_srm_compute_setup(const scarf_srm_params *p, scarf_srm_setup *s);
/* table: nharm rows {v1,v2,v3,a,b} (FP32); *n_kept = rows written. */
int scarf_srm_sample(const scarf_srm_params *p, const scarf_srm_setup *s, float *table, int *n_kept,
                     long long *pairs_used);

/* The same table as scarf_srm_sample (built-in generator), with the rejection
 * tests of the sampling loop (scarflib_srm.f90:731-745) evaluated on the
 * current GPU; the host walks the accepted pairs and decides the pairs whose
 * test lies within float rounding of its threshold, so the table is bit-
 * identical to the host loop's. *host_decided receives that pair count. */
int scarf_srm_sample_device(const scarf_srm_params *p, const scarf_srm_setup *s, float *table, int *n_kept,
                            long long *pairs_used, long long *host_decided, void *stream);

/* scarf_srm_sample_device for nfields fields at once (p[f], s[f] -> tables[f]
 * with room for p[f].nharm rows; n_kept[f], pairs_used[f] per field, may be
 * NULL for pairs_used; *host_decided sums the host-decided pairs). The first
 * pass of every field runs in one scan launch and one compaction launch; the
 * tables are bit-identical to scarf_srm_sample_device's. */
int scarf_srm_sample_device_batch(int nfields, const scarf_srm_params *p, const scarf_srm_setup *s,
                                  float *const *tables, int *n_kept, long long *pairs_used, long long *host_decided,
                                  void *stream);

/* The device scan's certain-reject table of one field (256 entries): a pair
 * whose second raw draw y2 is >= thr[y1 >> 23] (y1 the first raw draw) fails
 * the rejection test r2 < d(u) whatever the spectrum's FP32 rounding, and is
 * dropped before the spectrum is evaluated. 0xFFFFFFFF: never dropped early.
 * Exposed so that the bound can be checked on the host. */
int scarf_srm_sampler_reject_table(const scarf_srm_params *p, const scarf_srm_setup *s, unsigned int thr[256]);

/* Where scarf_execute draws its harmonics: SCARF_SAMPLER_AUTO (device,
 * unless a uniform source was installed), _HOST or _DEVICE. */
#define SCARF_SAMPLER_AUTO 0
#define SCARF_SAMPLER_HOST 1
#define SCARF_SAMPLER_DEVICE 2
int scarf_set_sampler(int where);
/* Upper bound on the uniform pairs one device pass tests (0 = sized from the
 * acceptance rate); further passes are chained as needed. */
int scarf_set_sampler_pass_pairs(long long pairs);

/* FP32 direct sum, structured block: field[i + n0*(j + n1*k)] for the grid
 * x = (i + fs[0] - 1) * ds (0-based i), likewise y, z; scaled by s->scaling.
 * d_table: nh rows of 5 floats on the device. */
int scarf_srm_direct_structured(const scarf_srm_setup *s, const int fs[3], const int n[3], float ds,
                                const float *d_table, int nh, float *d_field, void *stream);
/* sin/cos of the FP32 direct sum (no counterpart in the reference, which
 * calls the Fortran intrinsics): SCARF_SINCOS_FAST (default) reduces each
 * phase to [-pi, pi] by Cody-Waite's method (2 pi in three floats, FMA) and
 * takes the SFU's sin and cos (~6e-7 absolute per term; fields within ~4e-7
 * rel-RMS of the reference's FP32 arithmetic); SCARF_SINCOS_ACCURATE uses
 * CUDA's sincosf (~1 ulp; ~2e-7 rel-RMS) at about half the speed. */
#define SCARF_SINCOS_ACCURATE 0
#define SCARF_SINCOS_FAST 1
int scarf_set_direct_sincos(int mode);
/* FP32 direct sum over npts points (x, y, z device arrays). */
int scarf_srm_direct_points(const scarf_srm_setup *s, const float *d_x, const float *d_y, const float *d_z,
                            long long npts, const float *d_table, int nh, float *d_field, void *stream);

/* Factorised tensor-core form (structured only). d_work must hold
 * scarf_srm_tc_workspace_bytes(...) bytes of device memory (256-B aligned). */
size_t scarf_srm_tc_workspace_bytes(int ndim, const int n[3], int nh);
int scarf_srm_tc_structured(const scarf_srm_setup *s, const int fs[3], const int n[3], float ds,
                            const float *d_table, int nh, float *d_field, void *d_work, size_t work_bytes,
                            void *stream);

/* Batched tensor-core form: many structured fields (uneven sizes, spectra,
 * harmonic counts) in one persistent launch that pulls 128-row output tiles
 * from a device work queue, longest first. All fields of a batch must share
 * one row-tile shape (3-D fields with n[1] >= 8 do by default; 2-D fields
 * form their own batches). No counterpart in the reference, whose SRM
 * produces one field per call (scarflib_srm.f90:505). */
typedef struct scarf_tc_field {
  const scarf_srm_setup *setup; /* read during create only          */
  int fs[3];
  int n[3];
  float ds;
  const float *d_table; /* nh rows of 5 floats, device            */
  int nh;
  float *d_field; /* n[0]*n[1]*n[2] floats, device            */
  int tile_j;     /* row tile (128/tile_j) x tile_j; 0 = auto   */
} scarf_tc_field;
typedef struct scarf_tc_batch scarf_tc_batch;
size_t scarf_srm_tc_batch_workspace_bytes(const scarf_tc_field *fields, int nfields);
/* Plans the batch and uploads its descriptors into d_work (synchronous; call
 * outside stream capture). Tables and outputs must stay valid while the
 * batch is launched. */
int scarf_srm_tc_batch_create(const scarf_tc_field *fields, int nfields, void *d_work, size_t work_bytes,
                              scarf_tc_batch **batch);
/* Enqueues the batch on `stream` (table builds + one persistent kernel);
 * makes no synchronising or allocating call. */
int scarf_srm_tc_batch_launch(const scarf_tc_batch *batch, void *stream);
/* Synchronises `stream` and reports a kernel-side pipeline failure. With host
 * outputs set, it first copies each field to its host buffer as soon as
 * the launch has stored that field, while the launch computes the others. */
int scarf_srm_tc_batch_wait(const scarf_tc_batch *batch, void *stream);
/* host_fields[f] (nfields host buffers of n[0]*n[1]*n[2] floats, page-locked
 * for full copy speed; NULL turns the copy-out off): every
 * scarf_srm_tc_batch_wait after a launch copies the fields there, field by
 * field as they complete (the launch raises one host-mapped flag per field).
 * Re-uploads the descriptors (synchronous; call outside stream capture).
 * No counterpart in the reference. */
int scarf_srm_tc_batch_set_host_outputs(scarf_tc_batch *batch, float *const *host_fields);
void scarf_srm_tc_batch_destroy(scarf_tc_batch *batch);
/* Times the batch's candidate plans (kernel form SCARF_TC_SINGLE or
 * SCARF_TC_PAIR, tile_j in {1, 2, 4, 8, 16} for every field) on the fields'
 * own tables, overwriting their outputs, and returns the fastest (the
 * default, one-CTA form with the automatic tile_j, unless beaten by 3 %): create the
 * batch with each field's tile_j set to out->tile_j after
 * scarf_set_tc_variant(out->variant). Synchronises `stream`; allocates its
 * own device scratch. */
int scarf_srm_tc_batch_autotune(const scarf_tc_field *fields, int nfields, void *stream, scarf_tc_tuning *out);

/* Same tensor-core sum as scarf_srm_tc_structured, for callers that cannot
 * allocate device memory (their memory belongs to another allocator, or a
 * per-step cudaMalloc/cudaFree synchronisation is unacceptable). No
 * counterpart in the reference. Scratch lives in a fixed device array of
 * scarf_srm_tc_noalloc_capacity_bytes() (64 MiB) that every GPU loading the
 * library holds until exit; a grid and harmonic count whose
 * scarf_srm_tc_workspace_bytes() exceeds it returns SCARF_ERR_ARG. The plan
 * is the one scarf_srm_tc_structured runs (tuned plans included). The first
 * call in each device context looks up the array's device address; make that
 * first call on a device before any stream capture begins there. Every
 * call reads its status word back and synchronises `stream`. All calls on a
 * device share the array: calls that overlap on the GPU race and must be
 * serialised. */
size_t scarf_srm_tc_noalloc_capacity_bytes(void);
int scarf_srm_tc_structured_noalloc(const scarf_srm_setup *s, const int fs[3], const int n[3], float ds,
                                    const float *d_table, int nh, float *d_field, void *stream);

/* Field statistics as the reference computes them (FP64 sums, FP32 results):
 * mean and unbiased variance (scarflib_common.f90:694-817). d_work must hold
 * scarf_field_stats_workspace_bytes(n) bytes. Synchronises the stream. */
size_t scarf_field_stats_workspace_bytes(long long n);
int scarf_field_stats(const float *d_field, long long n, void *d_work, size_t work_bytes, float *mean,
                      float *var, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SCARF3D_B200_H_ */
