// C ABI of the B200 SRM library: the reference-compatible scarf_* entry
// points (module-global state, as scarflib.f90:87 and f_binding.f90:44-47
// keep it) and the extended, status-returning API of scarf3d_b200.h.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "scarf3d.h"
#include "scarf3d_b200.h"
#include "srm_host.h"
#include "srm_kernels.h"

namespace scarf {
namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // a failed cudaMalloc leaves no sticky error
    return fail(SCARF_ERR_NOMEM, "%s: %s (library device memory in use: %zu bytes)", what, cudaGetErrorString(e),
                scarf::device_memory_in_use());
  }
  return fail(SCARF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// A device-sampler failure: out of device memory (or over the library's
// cap) when an allocation on this thread said so, else a CUDA error.
int sampler_fail(const char* what) {
  if (scarf::take_device_alloc_failure())
    return fail(SCARF_ERR_NOMEM, "%s: out of device memory (library device memory in use: %zu bytes)", what,
                scarf::device_memory_in_use());
  return fail(SCARF_ERR_CUDA, "%s: CUDA error", what);
}

#define SCARF_CUDA(call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);    \
  } while (0)

// ------------------------------------------------------------------ config --
// Work items per output slab of the overlapped copy-out: the last slab is
// copied after the kernel ends, so slabs are kept small (64 items of a
// 512^3 field: 8 MB).
constexpr int kDefaultSlabItems = 64;
struct Config {
  int nharm = 10000;  // scarflib_srm.f90:90
  int form = SCARF_FORM_AUTO;
  UniformSource src;
  cudaStream_t stream = nullptr;
  int threads = 0;
  int sampler = SCARF_SAMPLER_AUTO;
  bool kernel_timing = false;
  int overlap_items = kDefaultSlabItems;  // work items per slab copied out while the kernel runs; 0 = off
};

// ------------------------------------------- reference-style global object --
struct Object {
  bool ready = false;
  bool structured = true;
  int nd = 3;
  int method = 0;
  int acf = 0, rescale = 0, pad = 0;
  int fs[3] = {1, 1, 1}, fe[3] = {1, 1, 1};
  float ds = 0, dh = 0, sigma = 0, hurst = 0, mute = -999.0f, taper = -999.0f;
  float alpha = 0, beta = 0, gamma = 0;
  float cl[3] = {0, 0, 0}, nc[3] = {0, 0, 0}, fc[3] = {0, 0, 0};
  int npts = 0;
  const float *x = nullptr, *y = nullptr, *z = nullptr;  // borrowed (scarflib.f90:233-237)
  std::vector<float> z2d;                                // 2D meshes: z = 0 (:239-240)
  const float* poi = nullptr;                            // borrowed, [nd x npoi]
  int npoi = 0;
  const void* pinned[3] = {nullptr, nullptr, nullptr};  // coordinate arrays this library page-locked
};

// The caller's coordinate arrays stay borrowed for the life of the mesh and
// every execute reads them anew (as the reference's does), so the library
// page-locks them there: each execute's upload is then an asynchronous copy
// that runs while the harmonics are sampled. Arrays that share pages are
// registered as one range; arrays that are managed or already page-locked
// memory, or that cannot be registered, are copied as they are.
void unpin_points(Object& o) {
  bool any = false;
  for (auto& p : o.pinned) {
    if (p) cudaHostUnregister(const_cast<void*>(p));
    any = any || p;
    p = nullptr;
  }
  if (any) (void)cudaGetLastError();
}

void pin_points(Object& o) {
  const float* arr[3] = {o.x, o.y, o.nd == 3 ? o.z : nullptr};
  const uintptr_t bytes = sizeof(float) * static_cast<uintptr_t>(o.npts);
  constexpr uintptr_t kPage = 4096;
  // Byte ranges of the arrays not yet page-locked; ranges whose pages touch
  // are registered as one (a second registration of a page fails).
  struct Range { uintptr_t lo, hi; };
  Range r[3];
  int n = 0;
  for (int c = 0; c < 3; ++c) {
    if (!arr[c]) continue;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, arr[c]) != cudaSuccess) {
      (void)cudaGetLastError();
      return;  // no usable device: nothing to gain
    }
    if (at.type != cudaMemoryTypeUnregistered) continue;  // device, managed or already page-locked
    const uintptr_t lo = reinterpret_cast<uintptr_t>(arr[c]);
    r[n++] = {lo, lo + bytes};
  }
  std::sort(r, r + n, [](const Range& a, const Range& b) { return a.lo < b.lo; });
  int m = 0;
  for (int i = 0; i < n; ++i) {
    if (m > 0 && r[i].lo / kPage <= (r[m - 1].hi - 1) / kPage) {
      r[m - 1].hi = std::max(r[m - 1].hi, r[i].hi);
    } else {
      r[m++] = r[i];
    }
  }
  for (int i = 0; i < m; ++i) {
    void* p = reinterpret_cast<void*>(r[i].lo);
    if (cudaHostRegister(p, r[i].hi - r[i].lo, cudaHostRegisterPortable) == cudaSuccess)
      o.pinned[i] = p;
    else
      (void)cudaGetLastError();
  }
}

void reset_object(Object& o) {
  unpin_points(o);
  o = Object();
}
std::mutex g_mu;  // every entry point that touches a context holds it

// --------------------------------------------------- per-device resources --
struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    scarf::device_free(p, bytes);
    p = nullptr;
    bytes = 0;
    const cudaError_t e = static_cast<cudaError_t>(scarf::device_alloc(&p, need));
    if (e == cudaSuccess) bytes = need;
    return e;
  }
  void release() {
    scarf::device_free(p, bytes);
    p = nullptr;
    bytes = 0;
  }
};

struct Resources {
  int device = -1;
  DeviceBuf status, stats, table, field, coords, work, slab_cnt, statrec, poi;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr, evs = nullptr;
  cudaEvent_t evp = nullptr;  // the coordinates' upload on the copy stream
  cudaStream_t copy_stream = nullptr;  // non-blocking: runs beside the legacy stream too
  int* slab_flags = nullptr;           // host-mapped, written by the kernel
  int* slab_flags_dev = nullptr;
  int slab_cap = 0;
  // Page-locked bounce ring for pageable host fields (kBounceSlots slots).
  char* bounce = nullptr;
  size_t bounce_slot = 0;
  cudaEvent_t bounce_ev[4] = {};
  void release() {
    if (bounce) cudaFreeHost(bounce);
    bounce = nullptr;
    bounce_slot = 0;
    for (auto& e : bounce_ev) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    if (slab_flags) cudaFreeHost(slab_flags);
    slab_flags = slab_flags_dev = nullptr;
    slab_cap = 0;
    slab_cnt.release();
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
    if (evs) cudaEventDestroy(evs);
    evs = nullptr;
    if (evp) cudaEventDestroy(evp);
    evp = nullptr;
    if (evk0) cudaEventDestroy(evk0);
    if (evk1) cudaEventDestroy(evk1);
    evk0 = evk1 = nullptr;
    status.release();
    stats.release();
    table.release();
    field.release();
    coords.release();
    work.release();
    statrec.release();
    poi.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
    device = -1;
  }
};
}  // namespace
}  // namespace scarf

// One library instance: the reference's global object, the settings and the
// device resources of its execute path. The legacy entry points act on the
// calling thread's current context (the process-wide default unless
// scarf_ctx_make_current chose another), so several meshes can be initialised
// at once, one per context (scarflib.f90:87 allows one).
struct scarf_ctx {
  scarf::Config cfg;
  scarf::Object obj;
  scarf::Resources res;
  float last_kernel_ms = 0.0f;
};

namespace scarf {
namespace {
scarf_ctx g_default_ctx;
thread_local scarf_ctx* t_ctx = &g_default_ctx;

// Makes `c` the calling thread's current context for one entry point's call.
class CtxScope {
 public:
  explicit CtxScope(scarf_ctx* c) : prev_(t_ctx) { t_ctx = c; }
  ~CtxScope() { t_ctx = prev_; }

 private:
  scarf_ctx* prev_;
};

int ensure_resources() {
  int dev = 0;
  SCARF_CUDA(cudaGetDevice(&dev));
  if (t_ctx->res.device != dev) {
    t_ctx->res.release();
    t_ctx->res.device = dev;
  }
  SCARF_CUDA(t_ctx->res.status.ensure(256));
  SCARF_CUDA(t_ctx->res.stats.ensure(stats_partials_bytes(0) + 256));
  if (!t_ctx->res.ev0) SCARF_CUDA(cudaEventCreate(&t_ctx->res.ev0));
  if (!t_ctx->res.ev1) SCARF_CUDA(cudaEventCreate(&t_ctx->res.ev1));
  if (!t_ctx->res.evk0) SCARF_CUDA(cudaEventCreate(&t_ctx->res.evk0));
  if (!t_ctx->res.evk1) SCARF_CUDA(cudaEventCreate(&t_ctx->res.evk1));
  return SCARF_OK;
}

// Slab flags (host-mapped) and device counters for at least n slabs, plus the
// copy stream and its join event.
int ensure_slab_resources(int n) {
  if (!t_ctx->res.copy_stream) SCARF_CUDA(cudaStreamCreateWithFlags(&t_ctx->res.copy_stream, cudaStreamNonBlocking));
  if (!t_ctx->res.evs) SCARF_CUDA(cudaEventCreateWithFlags(&t_ctx->res.evs, cudaEventDisableTiming));
  if (n > t_ctx->res.slab_cap) {
    if (t_ctx->res.slab_flags) cudaFreeHost(t_ctx->res.slab_flags);
    t_ctx->res.slab_flags = t_ctx->res.slab_flags_dev = nullptr;
    t_ctx->res.slab_cap = 0;
    void* h = nullptr;
    SCARF_CUDA(cudaHostAlloc(&h, sizeof(int) * n, cudaHostAllocMapped));
    t_ctx->res.slab_flags = static_cast<int*>(h);
    void* d = nullptr;
    SCARF_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    t_ctx->res.slab_flags_dev = static_cast<int*>(d);
    t_ctx->res.slab_cap = n;
  }
  SCARF_CUDA(t_ctx->res.slab_cnt.ensure(sizeof(int) * n));
  return SCARF_OK;
}

inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#else
  std::this_thread::yield();
#endif
}

// Copies the slabs of a running single-field launch to the host field in
// slab order, each as soon as the kernel has flagged it, on the copy stream.
// Once the launch stream is idle every remaining slab is copied without
// waiting (the status check that follows reports a failed launch).
// ------------------------------------------------ pageable host output --
// A device-to-host copy into pageable memory goes through the driver's own
// staging at a fraction of the link's rate. For pageable fields the copies go
// instead into a ring of page-locked slots at full rate, and the host's
// worker threads move each slot into the caller's array (in parallel pieces)
// while the next slots are in flight.
constexpr int kBounceSlots = 4;
constexpr size_t kBounceSlotCap = size_t(16) << 20;

bool is_pageable(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

int ensure_bounce(size_t slot_bytes) {
  slot_bytes = (slot_bytes + 4095) / 4096 * 4096;
  if (t_ctx->res.bounce && t_ctx->res.bounce_slot >= slot_bytes) return SCARF_OK;
  if (t_ctx->res.bounce) cudaFreeHost(t_ctx->res.bounce);
  t_ctx->res.bounce = nullptr;
  t_ctx->res.bounce_slot = 0;
  void* h = nullptr;
  SCARF_CUDA(cudaHostAlloc(&h, slot_bytes * kBounceSlots, cudaHostAllocDefault));
  t_ctx->res.bounce = static_cast<char*>(h);
  t_ctx->res.bounce_slot = slot_bytes;
  for (auto& e : t_ctx->res.bounce_ev)
    if (!e) SCARF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return SCARF_OK;
}

// A 2-D region (rows of `width` bytes, `height` rows) copied device -> a
// pageable host array through the ring. Regions are issued in order; each
// issue first completes the copy that last used its slot.
class BounceCopier {
 public:
  explicit BounceCopier(cudaStream_t cs) : cs_(cs) {}
  ~BounceCopier() { finish(); }
  int issue(char* dst, size_t dpitch, const char* src, size_t spitch, size_t width, size_t height) {
    const size_t cap = t_ctx->res.bounce_slot;
    const size_t rows_per = std::max<size_t>(1, cap / std::max<size_t>(width, 1));
    if (width > cap) {  // one row longer than a slot: split the row
      for (size_t r = 0; r < height; ++r)
        for (size_t o = 0; o < width; o += cap) {
          const int rc = issue_piece(dst + r * dpitch + o, dpitch, src + r * spitch + o, spitch,
                                     std::min(cap, width - o), 1);
          if (rc) return rc;
        }
      return SCARF_OK;
    }
    for (size_t r = 0; r < height; r += rows_per) {
      const int rc = issue_piece(dst + r * dpitch, dpitch, src + r * spitch, spitch, width,
                                 std::min(rows_per, height - r));
      if (rc) return rc;
    }
    return SCARF_OK;
  }
  // Moves every slot whose copy has already landed (oldest first) into the
  // caller's array, so that little is left for finish() once the last
  // region is issued.
  int poll() {
    for (int k = 0; k < kBounceSlots; ++k) {
      const int slot = (next_ + k) % kBounceSlots;
      if (!pend_[slot].busy) continue;
      if (cudaEventQuery(t_ctx->res.bounce_ev[slot]) != cudaSuccess) break;  // later copies queue behind it
      const int rc = complete(slot);
      if (rc) return rc;
    }
    return SCARF_OK;
  }
  int finish() {
    int rc = SCARF_OK;
    for (int k = 0; k < kBounceSlots; ++k) {
      const int c = complete((next_ + k) % kBounceSlots);
      if (c && !rc) rc = c;
    }
    return rc;
  }

 private:
  struct Pending {
    bool busy = false;
    char* dst = nullptr;
    size_t dpitch = 0, width = 0, height = 0;
  };
  int issue_piece(char* dst, size_t dpitch, const char* src, size_t spitch, size_t width, size_t height) {
    const int slot = next_;
    next_ = (next_ + 1) % kBounceSlots;
    int rc = complete(slot);
    if (rc) return rc;
    char* buf = t_ctx->res.bounce + static_cast<size_t>(slot) * t_ctx->res.bounce_slot;
    SCARF_CUDA(cudaMemcpy2DAsync(buf, width, src, spitch, width, height, cudaMemcpyDeviceToHost, cs_));
    SCARF_CUDA(cudaEventRecord(t_ctx->res.bounce_ev[slot], cs_));
    pend_[slot] = Pending{true, dst, dpitch, width, height};
    return SCARF_OK;
  }
  int complete(int slot) {
    Pending& q = pend_[slot];
    if (!q.busy) return SCARF_OK;
    q.busy = false;
    SCARF_CUDA(cudaEventSynchronize(t_ctx->res.bounce_ev[slot]));
    const char* buf = t_ctx->res.bounce + static_cast<size_t>(slot) * t_ctx->res.bounce_slot;
    constexpr size_t kPiece = size_t(1) << 20;
    const size_t per_row = (q.width + kPiece - 1) / kPiece;
    const Pending w = q;
    parallel_tasks(static_cast<int>(per_row * w.height), host_threads(), [&](int t) {
      const size_t r = static_cast<size_t>(t) / per_row, o = (static_cast<size_t>(t) % per_row) * kPiece;
      std::memcpy(w.dst + r * w.dpitch + o, buf + r * w.width + o, std::min(kPiece, w.width - o));
    });
    return SCARF_OK;
  }
  cudaStream_t cs_;
  int next_ = 0;
  Pending pend_[kBounceSlots];
};

int copy_slabs_out(const TcPlan& plan, const TcSlabSignal& sig, const float* d_field, float* field,
                   cudaStream_t st) {
  const bool bounce = is_pageable(field);
  if (bounce) {
    const TcSlab e0 = tc_slab_extent(plan, sig, 0);
    const size_t slab_bytes = static_cast<size_t>(e0.y1 - e0.y0) * plan.n1 * (e0.z1 - e0.z0) * sizeof(float);
    const int rc = ensure_bounce(std::min(kBounceSlotCap, std::max<size_t>(slab_bytes, 1 << 20)));
    if (rc) return rc;
  }
  BounceCopier bc(t_ctx->res.copy_stream);
  volatile int* flags = t_ctx->res.slab_flags;
  const size_t plane = static_cast<size_t>(plan.n1) * plan.n2;
  bool idle = false;
  for (int q = 0; q < sig.nslabs; ++q) {
    for (uint32_t spins = 0; !idle && !flags[q]; ++spins) {
      if ((spins & 1023u) == 1023u && cudaStreamQuery(st) != cudaErrorNotReady) {
        cudaGetLastError();
        idle = true;
      }
      if (bounce && (spins & 255u) == 255u) {
        // While the next slab computes, empty the slots that have landed.
        const int rc = bc.poll();
        if (rc) return rc;
      }
      cpu_relax();
    }
    const TcSlab e = tc_slab_extent(plan, sig, q);
    if (e.z1 <= e.z0 || e.y1 <= e.y0) continue;
    const size_t off = static_cast<size_t>(e.z0) * plane + static_cast<size_t>(e.y0) * plan.n1;
    const size_t width = static_cast<size_t>(e.y1 - e.y0) * plan.n1 * sizeof(float);
    if (bounce) {
      const int rc = bc.issue(reinterpret_cast<char*>(field + off), plane * sizeof(float),
                              reinterpret_cast<const char*>(d_field + off), plane * sizeof(float), width, e.z1 - e.z0);
      if (rc) return rc;
      continue;
    }
    SCARF_CUDA(cudaMemcpy2DAsync(field + off, plane * sizeof(float), d_field + off, plane * sizeof(float), width,
                                 e.z1 - e.z0, cudaMemcpyDeviceToHost, t_ctx->res.copy_stream));
  }
  return bc.finish();
}

// Whole field device -> host on `st` (after the kernels queued there): direct
// for page-locked or mapped memory, through the bounce ring for pageable.
int copy_field_out(float* field, const float* d_field, long long npts, cudaStream_t st) {
  const size_t bytes = sizeof(float) * static_cast<size_t>(npts);
  if (!is_pageable(field)) {
    SCARF_CUDA(cudaMemcpyAsync(field, d_field, bytes, cudaMemcpyDeviceToHost, st));
    return SCARF_OK;
  }
  int rc = ensure_bounce(std::min(kBounceSlotCap, std::max<size_t>(bytes / kBounceSlots, 1 << 20)));
  if (rc) return rc;
  BounceCopier bc(st);
  const size_t row = t_ctx->res.bounce_slot;
  const size_t rows = bytes / row, rest = bytes - rows * row;
  char* dst = reinterpret_cast<char*>(field);
  const char* src = reinterpret_cast<const char*>(d_field);
  if (rows) rc = bc.issue(dst, row, src, row, row, rows);
  if (!rc && rest) rc = bc.issue(dst + rows * row, rest, src + rows * row, rest, rest, 1);
  const int fr = bc.finish();
  return rc ? rc : fr;
}

// Events bracketing the dominant kernel of the next launch, when enabled.
cudaEvent_t kernel_ev0() { return t_ctx->cfg.kernel_timing ? t_ctx->res.evk0 : nullptr; }
cudaEvent_t kernel_ev1() { return t_ctx->cfg.kernel_timing ? t_ctx->res.evk1 : nullptr; }
void collect_kernel_time() {
  if (!t_ctx->cfg.kernel_timing) return;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, t_ctx->res.evk0, t_ctx->res.evk1) == cudaSuccess) t_ctx->last_kernel_ms = ms;
  cudaGetLastError();
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int check_device_status(const int* d_status, cudaStream_t st) {
  int h = 0;
  SCARF_CUDA(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCARF_CUDA(cudaStreamSynchronize(st));
  if (h != 0) return fail(SCARF_ERR_DEVICE, "device pipeline reported status %d (bounded wait expired)", h);
  return SCARF_OK;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

scarf_srm_params params_from_object(int seed) {
  scarf_srm_params p{};
  p.acf = t_ctx->obj.acf;
  p.nharm = t_ctx->cfg.nharm;
  p.seed = seed;
  p.rescale = t_ctx->obj.rescale;
  p.hurst = t_ctx->obj.hurst;
  p.sigma = t_ctx->obj.sigma;
  p.ds = t_ctx->obj.ds;
  p.dh = t_ctx->obj.dh;
  for (int c = 0; c < 3; ++c) {
    p.cl[c] = t_ctx->obj.cl[c];
    p.nc[c] = t_ctx->obj.nc[c];
    p.fc[c] = t_ctx->obj.fc[c];
  }
  p.alpha = t_ctx->obj.alpha;
  p.beta = t_ctx->obj.beta;
  p.gamma = t_ctx->obj.gamma;
  return p;
}

// Device copy of an unstructured mesh's coordinates (three arrays, each
// 16-byte aligned), issued on the copy stream; res.evp marks its end.
size_t coord_stride() { return (static_cast<size_t>(t_ctx->obj.npts) + 3) / 4 * 4; }

int upload_points() {
  const size_t npts = static_cast<size_t>(t_ctx->obj.npts);
  const size_t stride = coord_stride();
  SCARF_CUDA(t_ctx->res.coords.ensure(sizeof(float) * 3 * stride));
  if (!t_ctx->res.copy_stream) SCARF_CUDA(cudaStreamCreateWithFlags(&t_ctx->res.copy_stream, cudaStreamNonBlocking));
  if (!t_ctx->res.evp) SCARF_CUDA(cudaEventCreateWithFlags(&t_ctx->res.evp, cudaEventDisableTiming));
  float* c = static_cast<float*>(t_ctx->res.coords.p);
  cudaStream_t cs = t_ctx->res.copy_stream;
  SCARF_CUDA(cudaMemcpyAsync(c, t_ctx->obj.x, sizeof(float) * npts, cudaMemcpyDefault, cs));
  SCARF_CUDA(cudaMemcpyAsync(c + stride, t_ctx->obj.y, sizeof(float) * npts, cudaMemcpyDefault, cs));
  SCARF_CUDA(cudaMemcpyAsync(c + 2 * stride, t_ctx->obj.z, sizeof(float) * npts, cudaMemcpyDefault, cs));
  SCARF_CUDA(cudaEventRecord(t_ctx->res.evp, cs));
  return SCARF_OK;
}

// FIM (method 0) for the global object: scarf3d_structured_fim /
// scarf3d_unstructured_fim (scarflib_fim.f90:141-1104) on one device
// (fim.cu). The internal grid covers nc..fc; statistics, rescale and taper
// act on it, as the reference's do, before the external points take their
// nearest internal values. Point sets are not tapered unless
// SCARF_TAPER_UNSTRUCTURED is set: initialize_unstructured drops the POIs
// (scarflib.f90:273,283), for either method.
int fim_execute_impl(int seed, float* field, float stats[8], int flags) {
  cudaStream_t st = t_ctx->cfg.stream;
  FimInputs in{};
  in.ndim = t_ctx->obj.cl[2] > 0.0f ? 3 : 2;  // scarflib_fim.f90:770-774
  in.acf = t_ctx->obj.acf;
  in.pad = t_ctx->obj.pad;
  in.rescale = t_ctx->obj.rescale;
  in.seed = seed;
  in.ds = t_ctx->obj.ds;
  in.dh = t_ctx->obj.dh;
  in.sigma = t_ctx->obj.sigma;
  in.hurst = t_ctx->obj.hurst;
  in.mute = t_ctx->obj.mute;
  in.taper = t_ctx->obj.taper;
  for (int c = 0; c < 3; ++c) {
    in.cl[c] = t_ctx->obj.cl[c];
    in.nc[c] = t_ctx->obj.nc[c];
    in.fc[c] = t_ctx->obj.fc[c];
  }
  if (in.acf != 0 && in.acf != 1) return fail(SCARF_ERR_ARG, "FIM: acf must be 0 (von Karman) or 1 (Gaussian)");
  in.structured = t_ctx->obj.structured ? 1 : 0;
  long long npts;
  if (t_ctx->obj.structured) {
    npts = 1;
    for (int c = 0; c < 3; ++c) {
      in.fs[c] = t_ctx->obj.fs[c];
      in.fe[c] = t_ctx->obj.fe[c];
      npts *= t_ctx->obj.fe[c] - t_ctx->obj.fs[c] + 1;
    }
  } else {
    npts = t_ctx->obj.npts;
  }
  if (npts <= 0) return fail(SCARF_ERR_ARG, "empty point set");
  in.npts = npts;
  const bool taper_ok = t_ctx->obj.structured || (flags & SCARF_TAPER_UNSTRUCTURED);
  if (taper_ok && t_ctx->obj.poi && t_ctx->obj.npoi > 0) {
    in.poi = t_ctx->obj.poi;
    in.npoi = t_ctx->obj.npoi;
    in.poi_stride = t_ctx->obj.nd;
  }
  FimGrid g{};
  fim_grid(in, &g);
  for (int c = 0; c < 3; ++c)
    if (g.npts[c] <= 0) return fail(SCARF_ERR_ARG, "FIM: empty internal grid");
  const bool on_device = (flags & SCARF_FIELD_ON_DEVICE) || is_device_pointer(field);
  float* d_field = field;
  if (!on_device) {
    SCARF_CUDA(t_ctx->res.field.ensure(sizeof(float) * npts));
    d_field = static_cast<float*>(t_ctx->res.field.p);
  }
  if (!t_ctx->obj.structured) {
    const size_t stride = coord_stride();
    const int rc = upload_points();
    if (rc) return rc;
    SCARF_CUDA(cudaStreamWaitEvent(st, t_ctx->res.evp, 0));
    const float* c = static_cast<const float*>(t_ctx->res.coords.p);
    in.d_x = c;
    in.d_y = c + stride;
    in.d_z = c + 2 * stride;
  }
  SCARF_CUDA(t_ctx->res.work.ensure(fim_workspace_bytes(g, in.npoi)));
  const char* what = "";
  const cudaError_t e = fim_run(in, g, t_ctx->res.work.p, d_field, stats, st, &what);
  if (e != cudaSuccess) return fail(SCARF_ERR_CUDA, "FIM: %s: %s", what, cudaGetErrorString(e));
  if (!on_device) {
    const int rc = copy_field_out(field, d_field, npts, st);
    if (rc) return rc;
    SCARF_CUDA(cudaStreamSynchronize(st));
  }
  return SCARF_OK;
}

// The whole SRM execute (scarflib_srm.f90:505-929 / :105-499) for the global
// object. field: host or device memory of the local block / point set.
int execute_impl(int seed, float* field, float stats[8], int flags) {
  if (!t_ctx->obj.ready) return fail(SCARF_ERR_STATE, "scarf_execute called before scarf_*_initialize");
  if (!field || !stats) return fail(SCARF_ERR_ARG, "field and stats must not be NULL");
  int rc = ensure_resources();
  if (rc) return rc;
  scarf::take_device_alloc_failure();
  cudaStream_t st = t_ctx->cfg.stream;
  for (int i = 0; i < 8; ++i) stats[i] = 0.0f;
  if (t_ctx->obj.method == 0) return fim_execute_impl(seed, field, stats, flags);
  if (t_ctx->obj.method != 1) return fail(SCARF_ERR_UNSUPPORTED, "method must be 0 (FIM) or 1 (SRM)");
  // An unstructured mesh's coordinates go up while the harmonics are sampled.
  if (!t_ctx->obj.structured) {
    rc = upload_points();
    if (rc) return rc;
  }

  // Host: setup scalars and harmonic table.
  const double th0 = now_s();
  const scarf_srm_params p = params_from_object(seed);
  scarf_srm_setup s{};
  rc = srm_setup(p, &s);
  if (rc) return fail(rc, "invalid SRM parameters (acf %d, nharm %d)", p.acf, p.nharm);
  std::vector<float> table(5 * static_cast<size_t>(p.nharm));
  const int threads = t_ctx->cfg.threads > 0 ? t_ctx->cfg.threads : host_threads();
  long long pairs = 0;
  const bool on_gpu = !t_ctx->cfg.src.srng && t_ctx->cfg.sampler != SCARF_SAMPLER_HOST;
  const int nh = on_gpu ? srm_sample_device(p, s, table.data(), &pairs, st, nullptr)
                        : srm_sample(p, s, &t_ctx->cfg.src, threads, table.data(), &pairs);
  if (nh == -2) return sampler_fail("device sampler");
  if (nh < 0)
    return fail(SCARF_ERR_ARG,
                "rejection sampling infeasible: acceptance rate %.3g < %.1g (domain too small for the correlation "
                "lengths; stats[0] would flag it)",
                acceptance_rate(s), kMinAcceptance);
  const double t_host = now_s() - th0;

  // Device work.
  long long npts;
  int n[3] = {1, 1, 1};
  if (t_ctx->obj.structured) {
    for (int c = 0; c < 3; ++c) n[c] = t_ctx->obj.fe[c] - t_ctx->obj.fs[c] + 1;
    npts = static_cast<long long>(n[0]) * n[1] * n[2];
  } else {
    npts = t_ctx->obj.npts;
  }
  if (npts <= 0) return fail(SCARF_ERR_ARG, "empty point set");
  const bool on_device = (flags & SCARF_FIELD_ON_DEVICE) || is_device_pointer(field);
  SCARF_CUDA(t_ctx->res.table.ensure(sizeof(float) * 5 * std::max(nh, 1)));
  float* d_table = static_cast<float*>(t_ctx->res.table.p);
  int* d_status = static_cast<int*>(t_ctx->res.status.p);
  float* d_field = field;
  if (!on_device) {
    SCARF_CUDA(t_ctx->res.field.ensure(sizeof(float) * npts));
    d_field = static_cast<float*>(t_ctx->res.field.p);
  }
  SCARF_CUDA(cudaEventRecord(t_ctx->res.ev0, st));
  SCARF_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  if (nh > 0)
    SCARF_CUDA(cudaMemcpyAsync(d_table, table.data(), sizeof(float) * 5 * nh, cudaMemcpyHostToDevice, st));

  const float* dx = nullptr;
  const float* dy = nullptr;
  const float* dz = nullptr;
  const bool taper_ok = t_ctx->obj.structured || (flags & SCARF_TAPER_UNSTRUCTURED);
  const bool tapering = taper_ok && t_ctx->obj.poi && t_ctx->obj.npoi > 0;
  // Set once slab copies into the caller's buffer are in flight: every exit
  // from here on first waits for them.
  struct CopyJoin {
    bool active = false;
    ~CopyJoin() {
      if (active && t_ctx->res.copy_stream) cudaStreamSynchronize(t_ctx->res.copy_stream);
    }
  } copy_join;
  bool copied_out = false;  // field already on its way to the host (slab copies)
  // Statistics records written by the summation kernel (its epilogue reads
  // back what it stored), merged below: no further pass over the field.
  StatRecord* d_rec = nullptr;
  long long nrec = 0;
  auto want_records = [&](long long count) -> int {
    if (count <= 0) return SCARF_OK;
    SCARF_CUDA(t_ctx->res.statrec.ensure(sizeof(StatRecord) * static_cast<size_t>(count)));
    d_rec = static_cast<StatRecord*>(t_ctx->res.statrec.p);
    nrec = count;
    return SCARF_OK;
  };
  if (t_ctx->obj.structured) {
    const bool use_tc = (t_ctx->cfg.form != SCARF_FORM_DIRECT);
    TcPlan plan{};
    TcChoice tuned{};
    const bool have_tuned = use_tc && nh > 0 && tc_tuned_choice(s.ndim, n, true, &tuned);
    const bool planned = have_tuned ? tc_make_plan(s.ndim, n, nh, &plan, tuned.tile_j, false, tuned.variant)
                                    : tc_make_plan(s.ndim, n, nh, &plan);
    if (use_tc && nh > 0 && planned) {
      SCARF_CUDA(t_ctx->res.work.ensure(plan.bytes));
      // Without rescale or taper the field is final when the kernel stores
      // it: copy it out slab by slab while the kernel still runs.
      TcSlabSignal sig;
      const bool overlap = t_ctx->cfg.overlap_items > 0 && !on_device && p.rescale != 1 && !tapering;
      if (overlap) {
        tc_slab_layout(plan, t_ctx->cfg.overlap_items, &sig);
        rc = ensure_slab_resources(sig.nslabs);
        if (rc) return rc;
        std::memset(t_ctx->res.slab_flags, 0, sizeof(int) * sig.nslabs);
        sig.d_cnt = static_cast<int*>(t_ctx->res.slab_cnt.p);
        sig.flag_dev = t_ctx->res.slab_flags_dev;
      }
      rc = want_records(tc_stat_records(plan));
      if (rc) return rc;
      SCARF_CUDA(launch_tc_structured(s, t_ctx->obj.fs, n, p.ds, d_table, nh, d_field, t_ctx->res.work.p, plan, d_status, st,
                                      kernel_ev0(), kernel_ev1(), overlap ? &sig : nullptr, d_rec));
      if (overlap) {
        copy_join.active = true;
        rc = copy_slabs_out(plan, sig, d_field, field, st);
        if (rc) return rc;
        copied_out = true;
      }
    } else if (nh > 0) {
      rc = want_records(direct_stat_records(npts));
      if (rc) return rc;
      if (kernel_ev0()) SCARF_CUDA(cudaEventRecord(kernel_ev0(), st));
      SCARF_CUDA(launch_direct_structured(s, t_ctx->obj.fs, n, p.ds, d_table, nh, d_field, d_status, st, d_rec));
      if (kernel_ev1()) SCARF_CUDA(cudaEventRecord(kernel_ev1(), st));
    } else {
      SCARF_CUDA(cudaMemsetAsync(d_field, 0, sizeof(float) * npts, st));
    }
  } else {
    // The coordinates were issued on the copy stream before the sampling.
    const float* c = static_cast<const float*>(t_ctx->res.coords.p);
    const size_t stride = coord_stride();
    SCARF_CUDA(cudaStreamWaitEvent(st, t_ctx->res.evp, 0));
    dx = c;
    dy = c + stride;
    dz = c + 2 * stride;
    if (nh > 0) {
      rc = want_records(direct_stat_records(npts));
      if (rc) return rc;
      if (kernel_ev0()) SCARF_CUDA(cudaEventRecord(kernel_ev0(), st));
      SCARF_CUDA(launch_direct_points(s, dx, dy, dz, npts, d_table, nh, d_field, d_status, st, d_rec));
      if (kernel_ev1()) SCARF_CUDA(cudaEventRecord(kernel_ev1(), st));
    } else {
      SCARF_CUDA(cudaMemsetAsync(d_field, 0, sizeof(float) * npts, st));
    }
  }
  // Statistics (scarflib_srm.f90:877-895): single set, so the Chan merge
  // returns (var, mean) unchanged; std = sqrt(var) in FP32. The summation
  // kernel recorded per-tile moments as it stored the field; one small
  // kernel merges them (a field without harmonics takes the two FP64 passes
  // instead). The sum's status word comes back with them in one
  // synchronisation (after a failed sum the statistics are dropped).
  double* d_part = static_cast<double*>(t_ctx->res.stats.p);
  float* d_out = reinterpret_cast<float*>(static_cast<char*>(t_ctx->res.stats.p) + stats_partials_bytes(0));
  if (d_rec)
    SCARF_CUDA(launch_stats_records(d_rec, nrec, d_out, st));
  else
    SCARF_CUDA(launch_field_stats(d_field, npts, d_part, d_out, st));
  float mv[2];
  int dev_status = 0;
  SCARF_CUDA(cudaMemcpyAsync(&dev_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCARF_CUDA(cudaMemcpyAsync(mv, d_out, sizeof(mv), cudaMemcpyDeviceToHost, st));
  SCARF_CUDA(cudaStreamSynchronize(st));
  if (dev_status != 0)
    return fail(SCARF_ERR_DEVICE, "device pipeline reported status %d (bounded wait expired)", dev_status);
  if (nh > 0) collect_kernel_time();
  stats[0] = s.info0;
  stats[1] = s.info1;
  stats[2] = sqrtf(mv[1]);
  stats[3] = mv[0];

  // Rescale (:897-912) and taper (:920-925), in one pass over the field.
  std::vector<float> poi3;
  if (p.rescale == 1 || tapering) {
    FinalizeArgs fa{};
    if (p.rescale == 1) {
      fa.rescale = 1;
      fa.scaling = p.sigma / stats[2];  // scarflib_srm.f90:899, FP32 on the host
      fa.mean = stats[3];
      stats[2] = p.sigma;
      stats[3] = 0.0f;
    }
    if (tapering) {
      poi3.assign(3 * static_cast<size_t>(t_ctx->obj.npoi), 0.0f);
      for (int q = 0; q < t_ctx->obj.npoi; ++q)
        for (int c = 0; c < s.ndim; ++c) poi3[3 * q + c] = t_ctx->obj.poi[t_ctx->obj.nd * q + c];
      SCARF_CUDA(t_ctx->res.poi.ensure(sizeof(float) * poi3.size()));
      SCARF_CUDA(cudaMemcpyAsync(t_ctx->res.poi.p, poi3.data(), sizeof(float) * poi3.size(), cudaMemcpyHostToDevice, st));
      fa.d_poi = static_cast<const float*>(t_ctx->res.poi.p);
      fa.npoi = t_ctx->obj.npoi;
      fa.mute = t_ctx->obj.mute;
      fa.taper = t_ctx->obj.taper;
      if (t_ctx->obj.structured) {
        fa.n0 = n[0];
        fa.n1 = n[1];
        fa.o0 = t_ctx->obj.fs[0] - 1;
        fa.o1 = t_ctx->obj.fs[1] - 1;
        fa.o2 = t_ctx->obj.fs[2] - 1;
        fa.dh = p.ds;
      } else {
        fa.d_x = dx;
        fa.d_y = dy;
        fa.d_z = dz;
      }
    }
    SCARF_CUDA(launch_finalize_field(d_field, npts, fa, st));
  }
  if (copied_out) {
    // Device time ends with the last slab copy.
    SCARF_CUDA(cudaEventRecord(t_ctx->res.evs, st));
    SCARF_CUDA(cudaStreamWaitEvent(t_ctx->res.copy_stream, t_ctx->res.evs, 0));
    SCARF_CUDA(cudaEventRecord(t_ctx->res.ev1, t_ctx->res.copy_stream));
    SCARF_CUDA(cudaStreamSynchronize(t_ctx->res.copy_stream));
  } else {
    SCARF_CUDA(cudaEventRecord(t_ctx->res.ev1, st));
    if (!on_device) {
      rc = copy_field_out(field, d_field, npts, st);
      if (rc) return rc;
    }
  }
  SCARF_CUDA(cudaStreamSynchronize(st));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, t_ctx->res.ev0, t_ctx->res.ev1);
  stats[4] = static_cast<float>(t_host);
  stats[5] = ms * 1e-3f;
  return SCARF_OK;
}

void finalize_impl() {
  reset_object(t_ctx->obj);
  t_ctx->res.release();
}

}  // namespace

// Error recording for entry points defined in other translation units.
int record_error(int code, const char* msg) { return fail(code, "%s", msg); }

}  // namespace scarf

using namespace scarf;

// ======================================================================== //
// Reference-compatible entry points                                          //
// ======================================================================== //
extern "C" {

void scarf_opt_init(struct scarf_opt* var) {
  if (!var) return;
  std::memset(var, 0, sizeof(*var));
}

}  // extern "C"

namespace {
// The bodies of the initialize entry points, on the current context (the
// caller holds g_mu).
int cart_initialize_impl(const int nd, const int fs[], const int fe[], const real ds, const int acf,
                         const real cl[], const real sigma, const struct scarf_opt* var) {
  if ((nd != 2 && nd != 3) || !fs || !fe || !cl)
    return fail(SCARF_ERR_ARG, "scarf_cart_initialize: nd must be 2 or 3 and fs, fe, cl non-NULL");
  Object& o = t_ctx->obj;
  reset_object(o);
  o.structured = true;
  o.nd = nd;
  for (int c = 0; c < nd; ++c) {
    o.fs[c] = fs[c];
    o.fe[c] = fe[c];
    o.cl[c] = cl[c];
  }
  o.ds = ds;
  o.dh = ds;  // scarflib.f90:139
  o.acf = acf;
  o.sigma = sigma;
  for (int c = 0; c < 3; ++c) {  // scarflib.f90:157-158
    o.nc[c] = static_cast<float>(o.fs[c] - 1) * ds;
    o.fc[c] = static_cast<float>(o.fe[c] - 1) * ds;
  }
  if (var) {  // c_binding.c:89-103: a field is given when > 0 / != 0
    if (var->method == 1) o.method = 1;
    if (var->hurst > 0) o.hurst = var->hurst;
    if (var->dh > 0) o.dh = var->dh;
    if (var->poi && var->npoi > 0) {
      o.poi = var->poi;
      o.npoi = var->npoi;
    }
    if (var->mute > 0) o.mute = var->mute;
    if (var->taper > 0) o.taper = var->taper;
    if (var->rescale == 1) o.rescale = 1;
    if (var->pad == 1) o.pad = 1;
    if (var->nc && var->fc)
      for (int c = 0; c < nd; ++c) {
        o.nc[c] = var->nc[c];
        o.fc[c] = var->fc[c];
      }
    if (var->alpha != 0) o.alpha = var->alpha;
    if (var->beta != 0) o.beta = var->beta;
    if (var->gamma != 0) o.gamma = var->gamma;
  }
  o.ready = true;
  g_last_error.clear();
  return SCARF_OK;
}

int nocart_initialize_impl(const int nd, const int npts, const real* x, const real* y, const real* z,
                           const real dh, const int acf, const real cl[], const real sigma,
                           const struct scarf_opt* var) {
  if ((nd != 2 && nd != 3) || npts <= 0 || !x || !y || !cl || (nd == 3 && !z))
    return fail(SCARF_ERR_ARG, "scarf_nocart_initialize: invalid nd/npts or NULL coordinates");
  Object& o = t_ctx->obj;
  reset_object(o);
  o.structured = false;
  o.nd = nd;
  o.npts = npts;
  o.x = x;
  o.y = y;
  if (nd == 3) {
    o.z = z;
  } else {
    o.z2d.assign(static_cast<size_t>(npts), 0.0f);
    o.z = o.z2d.data();
  }
  for (int c = 0; c < nd; ++c) o.cl[c] = cl[c];
  o.dh = dh;
  o.ds = dh;  // scarflib.f90:249
  o.acf = acf;
  o.sigma = sigma;
  // nc / fc from the coordinate extrema (scarflib.f90:265-271).
  const float* ax[3] = {x, y, o.z};
  for (int c = 0; c < 3; ++c) {
    if (c >= nd) {
      o.nc[c] = o.fc[c] = 0.0f;
      continue;
    }
    float lo = ax[c][0], hi = ax[c][0];
    for (int i = 1; i < npts; ++i) {
      lo = std::min(lo, ax[c][i]);
      hi = std::max(hi, ax[c][i]);
    }
    o.nc[c] = lo;
    o.fc[c] = hi;
  }
  if (var) {
    if (var->method == 1) o.method = 1;
    if (var->hurst > 0) o.hurst = var->hurst;
    if (var->ds > 0) o.ds = var->ds;
    if (var->poi && var->npoi > 0) {
      o.poi = var->poi;
      o.npoi = var->npoi;
    }
    if (var->mute > 0) o.mute = var->mute;
    if (var->taper > 0) o.taper = var->taper;
    if (var->rescale == 1) o.rescale = 1;
    if (var->pad == 1) o.pad = 1;
    if (var->nc && var->fc)
      for (int c = 0; c < nd; ++c) {
        o.nc[c] = var->nc[c];
        o.fc[c] = var->fc[c];
      }
    if (var->alpha != 0) o.alpha = var->alpha;
    if (var->beta != 0) o.beta = var->beta;
    if (var->gamma != 0) o.gamma = var->gamma;
  }
  pin_points(o);
  o.ready = true;
  g_last_error.clear();
  return SCARF_OK;
}
}  // namespace

extern "C" {

void scarf_cart_initialize(const int nd, const int fs[], const int fe[], const real ds, const int acf,
                           const real cl[], const real sigma, struct scarf_opt* var) {
  std::lock_guard<std::mutex> lk(g_mu);
  cart_initialize_impl(nd, fs, fe, ds, acf, cl, sigma, var);
}

void scarf_nocart_initialize(const int nd, const int npts, const real* x, const real* y, const real* z,
                             const real dh, const int acf, const real cl[], const real sigma,
                             struct scarf_opt* var) {
  std::lock_guard<std::mutex> lk(g_mu);
  nocart_initialize_impl(nd, npts, x, y, z, dh, acf, cl, sigma, var);
}

void scarf_execute(const int seed, real* field, real stats[]) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int rc = execute_impl(seed, field, stats, 0);
  if (rc) std::fprintf(stderr, "scarf_execute: %s\n", g_last_error.c_str());
}

void scarf_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  finalize_impl();
}

// Raw column-major FP32 output of the local block placed in the global grid
// `npts` at its fs offset (the subarray view of scarflib_common.f90:363-399).
void scarf_io_one(const int nd, const int* npts, const real* field, const char fname[], const int* nwriters) {
  (void)nwriters;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!t_ctx->obj.ready || !t_ctx->obj.structured || !npts || !field || !fname) {
    fail(SCARF_ERR_STATE, "scarf_io_one: needs an initialized structured mesh");
    return;
  }
  long long gn[3] = {npts[0], nd > 1 ? npts[1] : 1, nd > 2 ? npts[2] : 1};
  int n[3];
  for (int c = 0; c < 3; ++c) n[c] = t_ctx->obj.fe[c] - t_ctx->obj.fs[c] + 1;
  const int fd = open(fname, O_CREAT | O_WRONLY, 0644);
  if (fd < 0) {
    fail(SCARF_ERR_ARG, "scarf_io_one: cannot open %s", fname);
    return;
  }
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j) {
      const long long gi = (t_ctx->obj.fs[0] - 1) + gn[0] * ((t_ctx->obj.fs[1] - 1 + j) + gn[1] * (t_ctx->obj.fs[2] - 1 + k));
      const real* src = field + static_cast<long long>(n[0]) * (j + static_cast<long long>(n[1]) * k);
      if (pwrite(fd, src, sizeof(real) * n[0], static_cast<off_t>(gi * sizeof(real))) < 0) {
        fail(SCARF_ERR_ARG, "scarf_io_one: write failed");
        close(fd);
        return;
      }
    }
  close(fd);
}

// One plane normal to `axis` ('x','y','z') at global index `plane`
// (scarflib_common.f90:527-646), written as a 2-D column-major FP32 array.
void scarf_io_slice(const int* npts, const char axis[], const int plane, const real* field, const char fname[]) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!t_ctx->obj.ready || !t_ctx->obj.structured || !npts || !axis || !field || !fname) {
    fail(SCARF_ERR_STATE, "scarf_io_slice: needs an initialized structured mesh");
    return;
  }
  const int cut = axis[0] == 'x' ? 0 : axis[0] == 'y' ? 1 : axis[0] == 'z' ? 2 : -1;
  if (cut < 0) return;
  if (plane < t_ctx->obj.fs[cut] || plane > t_ctx->obj.fe[cut]) return;
  int n[3];
  for (int c = 0; c < 3; ++c) n[c] = t_ctx->obj.fe[c] - t_ctx->obj.fs[c] + 1;
  const int d0 = cut == 0 ? 1 : 0, d1 = cut == 2 ? 1 : 2;
  const int cidx = plane - t_ctx->obj.fs[cut];
  const int fd = open(fname, O_CREAT | O_WRONLY, 0644);
  if (fd < 0) {
    fail(SCARF_ERR_ARG, "scarf_io_slice: cannot open %s", fname);
    return;
  }
  std::vector<real> row(n[d0]);
  for (int b = 0; b < n[d1]; ++b) {
    for (int a = 0; a < n[d0]; ++a) {
      int idx[3];
      idx[cut] = cidx;
      idx[d0] = a;
      idx[d1] = b;
      row[a] = field[idx[0] + static_cast<long long>(n[0]) * (idx[1] + static_cast<long long>(n[1]) * idx[2])];
    }
    const long long gi = (t_ctx->obj.fs[d0] - 1) + static_cast<long long>(npts[d0]) * (t_ctx->obj.fs[d1] - 1 + b);
    if (pwrite(fd, row.data(), sizeof(real) * n[d0], static_cast<off_t>(gi * sizeof(real))) < 0) break;
  }
  close(fd);
}

// ======================================================================== //
// Extended API                                                              //
// ======================================================================== //
const char* scarf_last_error(void) { return g_last_error.c_str(); }

int scarf_set_nharm(int nharm) {
  if (nharm <= 0) return fail(SCARF_ERR_ARG, "nharm must be positive");
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.nharm = nharm;
  return SCARF_OK;
}

int scarf_get_nharm(void) { return t_ctx->cfg.nharm; }

int scarf_set_form(int form) {
  if (form < SCARF_FORM_AUTO || form > SCARF_FORM_TC) return fail(SCARF_ERR_ARG, "unknown form %d", form);
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.form = form;
  return SCARF_OK;
}

int scarf_set_uniform_source(void (*set_seed)(int), void (*srng)(float*)) {
  if ((set_seed == nullptr) != (srng == nullptr))
    return fail(SCARF_ERR_ARG, "set_seed and srng must both be given or both be NULL");
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.src.set_seed = set_seed;
  t_ctx->cfg.src.srng = srng;
  return SCARF_OK;
}

int scarf_set_stream(void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.stream = static_cast<cudaStream_t>(stream);
  return SCARF_OK;
}

int scarf_set_host_threads(int nthreads) {
  if (nthreads < 0) return fail(SCARF_ERR_ARG, "nthreads must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.threads = nthreads;
  return SCARF_OK;
}

int scarf_execute_ex(int seed, float* field, float stats[8], int flags) {
  std::lock_guard<std::mutex> lk(g_mu);
  return execute_impl(seed, field, stats, flags);
}

scarf_ctx* scarf_ctx_create(void) {
  auto* c = new (std::nothrow) scarf_ctx();
  if (!c) fail(SCARF_ERR_NOMEM, "out of host memory");
  return c;
}

void scarf_ctx_destroy(scarf_ctx* ctx) {
  if (!ctx || ctx == &g_default_ctx) return;
  std::lock_guard<std::mutex> lk(g_mu);
  {
    CtxScope scope(ctx);
    finalize_impl();
  }
  if (t_ctx == ctx) t_ctx = &g_default_ctx;
  delete ctx;
}

int scarf_ctx_make_current(scarf_ctx* ctx) {
  t_ctx = ctx ? ctx : &g_default_ctx;
  return SCARF_OK;
}

int scarf_ctx_cart_initialize(scarf_ctx* ctx, int nd, const int fs[], const int fe[], float ds, int acf,
                              const float cl[], float sigma, const struct scarf_opt* opt) {
  if (!ctx) return fail(SCARF_ERR_ARG, "NULL context");
  std::lock_guard<std::mutex> lk(g_mu);
  CtxScope scope(ctx);
  return cart_initialize_impl(nd, fs, fe, ds, acf, cl, sigma, opt);
}

int scarf_ctx_nocart_initialize(scarf_ctx* ctx, int nd, int npts, const float* x, const float* y, const float* z,
                                float dh, int acf, const float cl[], float sigma, const struct scarf_opt* opt) {
  if (!ctx) return fail(SCARF_ERR_ARG, "NULL context");
  std::lock_guard<std::mutex> lk(g_mu);
  CtxScope scope(ctx);
  return nocart_initialize_impl(nd, npts, x, y, z, dh, acf, cl, sigma, opt);
}

int scarf_ctx_execute(scarf_ctx* ctx, int seed, float* field, float stats[8], int flags) {
  if (!ctx) return fail(SCARF_ERR_ARG, "NULL context");
  std::lock_guard<std::mutex> lk(g_mu);
  CtxScope scope(ctx);
  return execute_impl(seed, field, stats, flags);
}

int scarf_ctx_finalize(scarf_ctx* ctx) {
  if (!ctx) return fail(SCARF_ERR_ARG, "NULL context");
  std::lock_guard<std::mutex> lk(g_mu);
  CtxScope scope(ctx);
  finalize_impl();
  return SCARF_OK;
}

int scarf_srm_compute_setup(const scarf_srm_params* p, scarf_srm_setup* s) {
  if (!p || !s) return fail(SCARF_ERR_ARG, "NULL argument");
  const int rc = srm_setup(*p, s);
  if (rc) return fail(rc, "invalid SRM parameters");
  return SCARF_OK;
}

int scarf_set_sampler(int where) {
  if (where < SCARF_SAMPLER_AUTO || where > SCARF_SAMPLER_DEVICE) return fail(SCARF_ERR_ARG, "unknown sampler");
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.sampler = where;
  return SCARF_OK;
}

int scarf_set_sampler_pass_pairs(long long pairs) {
  if (pairs < 0) return fail(SCARF_ERR_ARG, "pairs must be >= 0");
  set_device_sampler_pass_cap(pairs);
  return SCARF_OK;
}

int scarf_srm_sample_device(const scarf_srm_params* p, const scarf_srm_setup* s, float* table, int* n_kept,
                            long long* pairs_used, long long* host_decided, void* stream) {
  if (!p || !s || !table) return fail(SCARF_ERR_ARG, "NULL argument");
  scarf::take_device_alloc_failure();
  long long used = 0, open = 0;
  const int kept = srm_sample_device(*p, *s, table, &used, stream, &open);
  if (kept == -1)
    return fail(SCARF_ERR_ARG, "rejection sampling infeasible: acceptance rate %.3g < %.1g", acceptance_rate(*s),
                kMinAcceptance);
  if (kept < 0) return sampler_fail("device sampler");
  if (n_kept) *n_kept = kept;
  if (pairs_used) *pairs_used = used;
  if (host_decided) *host_decided = open;
  return SCARF_OK;
}

int scarf_srm_sample_device_batch(int nfields, const scarf_srm_params* p, const scarf_srm_setup* s,
                                  float* const* tables, int* n_kept, long long* pairs_used, long long* host_decided,
                                  void* stream) {
  if (nfields < 0 || (nfields > 0 && (!p || !s || !tables || !n_kept)))
    return fail(SCARF_ERR_ARG, "invalid argument");
  for (int f = 0; f < nfields; ++f)
    if (!tables[f]) return fail(SCARF_ERR_ARG, "tables[%d] is NULL", f);
  scarf::take_device_alloc_failure();
  long long open = 0;
  const int rc = srm_sample_device_batch(nfields, p, s, tables, n_kept, pairs_used, stream, &open);
  if (rc <= -2 - nfields) return sampler_fail("batched device sampler");
  if (rc < 0) {
    const int f = -1 - rc;
    return fail(SCARF_ERR_ARG, "field %d: rejection sampling infeasible: acceptance rate %.3g < %.1g", f,
                acceptance_rate(s[f]), kMinAcceptance);
  }
  if (host_decided) *host_decided = open;
  return SCARF_OK;
}

int scarf_srm_sampler_reject_table(const scarf_srm_params* p, const scarf_srm_setup* s, unsigned int thr[256]) {
  static_assert(kRejectBins == 256, "the header declares 256 bins");
  if (!p || !s || !thr) return fail(SCARF_ERR_ARG, "NULL argument");
  sampler_reject_thresholds(*s, p->acf, kSamplerMargin, thr);
  return SCARF_OK;
}

int scarf_srm_sample(const scarf_srm_params* p, const scarf_srm_setup* s, float* table, int* n_kept,
                     long long* pairs_used) {
  if (!p || !s || !table) return fail(SCARF_ERR_ARG, "NULL argument");
  UniformSource src;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    src = t_ctx->cfg.src;
  }
  const int threads = t_ctx->cfg.threads > 0 ? t_ctx->cfg.threads : host_threads();
  long long used = 0;
  const int kept = srm_sample(*p, *s, &src, threads, table, &used);
  if (kept < 0)
    return fail(SCARF_ERR_ARG, "rejection sampling infeasible: acceptance rate %.3g < %.1g", acceptance_rate(*s),
                kMinAcceptance);
  if (n_kept) *n_kept = kept;
  if (pairs_used) *pairs_used = used;
  return SCARF_OK;
}

int scarf_srm_direct_structured(const scarf_srm_setup* s, const int fs[3], const int n[3], float ds,
                                const float* d_table, int nh, float* d_field, void* stream) {
  if (!s || !fs || !n || !d_field || (nh > 0 && !d_table) || nh < 0) return fail(SCARF_ERR_ARG, "invalid argument");
  if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return fail(SCARF_ERR_ARG, "empty grid");
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = ensure_resources();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_status = static_cast<int*>(t_ctx->res.status.p);
  SCARF_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  if (nh == 0) {
    SCARF_CUDA(cudaMemsetAsync(d_field, 0, sizeof(float) * n[0] * n[1] * n[2], st));
    return SCARF_OK;
  }
  if (kernel_ev0()) SCARF_CUDA(cudaEventRecord(kernel_ev0(), st));
  SCARF_CUDA(launch_direct_structured(*s, fs, n, ds, d_table, nh, d_field, d_status, st));
  if (kernel_ev1()) SCARF_CUDA(cudaEventRecord(kernel_ev1(), st));
  rc = check_device_status(d_status, st);
  if (!rc) collect_kernel_time();
  return rc;
}

int scarf_srm_direct_points(const scarf_srm_setup* s, const float* d_x, const float* d_y, const float* d_z,
                            long long npts, const float* d_table, int nh, float* d_field, void* stream) {
  if (!s || !d_x || !d_y || !d_z || !d_field || npts <= 0 || nh < 0 || (nh > 0 && !d_table))
    return fail(SCARF_ERR_ARG, "invalid argument");
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = ensure_resources();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_status = static_cast<int*>(t_ctx->res.status.p);
  SCARF_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  if (nh == 0) {
    SCARF_CUDA(cudaMemsetAsync(d_field, 0, sizeof(float) * npts, st));
    return SCARF_OK;
  }
  if (kernel_ev0()) SCARF_CUDA(cudaEventRecord(kernel_ev0(), st));
  SCARF_CUDA(launch_direct_points(*s, d_x, d_y, d_z, npts, d_table, nh, d_field, d_status, st));
  if (kernel_ev1()) SCARF_CUDA(cudaEventRecord(kernel_ev1(), st));
  rc = check_device_status(d_status, st);
  if (!rc) collect_kernel_time();
  return rc;
}

// Device-field entry points let the longest axis be the column axis
// (wider column tiles), or follow a tuned choice for the grid's bucket when
// tuned plans are enabled; the same rule sizes their workspace.
}  // extern "C"
namespace scarf {
bool device_field_plan(int ndim, const int n[3], int nh, TcPlan* p) {
  TcChoice c{};
  if (n[0] > 0 && n[1] > 0 && n[2] > 0 && tc_tuned_choice(ndim, n, false, &c))
    return tc_make_plan(ndim, n, nh, p, c.tile_j, c.permute != 0, c.variant, std::max(1, c.split));
  // SCARF3D_B200_TC_SPLIT=<n> splits the harmonics of untuned device-field
  // plans over n items per tile (tests compare split and unsplit sums).
  const char* e = std::getenv("SCARF3D_B200_TC_SPLIT");
  const int split = e ? std::max(1, std::atoi(e)) : 1;
  return tc_make_plan(ndim, n, nh, p, 0, true, -1, split);
}
}  // namespace scarf
extern "C" {
size_t scarf_srm_tc_workspace_bytes(int ndim, const int n[3], int nh) {
  TcPlan p{};
  if (!n || !device_field_plan(ndim, n, nh, &p)) return 0;
  return p.bytes;
}

int scarf_srm_tc_plan_info(int ndim, const int n[3], int nh, scarf_tc_tuning* out) {
  TcPlan p{};
  if (!n || !out || !device_field_plan(ndim, n, nh, &p)) return fail(SCARF_ERR_ARG, "invalid grid for the tensor-core form");
  out->variant = p.pair ? SCARF_TC_PAIR : (p.tmem_a ? SCARF_TC_SINGLE_TMEM_A : SCARF_TC_SINGLE);
  out->tile_j = p.tj;
  out->permute = p.ax_c != (ndim == 3 ? 2 : 1) ? 1 : 0;
  out->ms = 0.0f;
  out->split = p.split;
  return SCARF_OK;
}

int scarf_srm_tc_structured(const scarf_srm_setup* s, const int fs[3], const int n[3], float ds, const float* d_table,
                            int nh, float* d_field, void* d_work, size_t work_bytes, void* stream) {
  if (!s || !fs || !n || !d_field || !d_table || nh <= 0 || !d_work) return fail(SCARF_ERR_ARG, "invalid argument");
  TcPlan p{};
  if (!device_field_plan(s->ndim, n, nh, &p)) return fail(SCARF_ERR_ARG, "invalid grid for the tensor-core form");
  if (work_bytes < p.bytes) return fail(SCARF_ERR_ARG, "workspace too small: %zu < %zu", work_bytes, p.bytes);
  if (reinterpret_cast<uintptr_t>(d_work) & 255u) return fail(SCARF_ERR_ARG, "workspace must be 256-byte aligned");
  std::lock_guard<std::mutex> lk(g_mu);
  if (t_ctx->cfg.kernel_timing) {
    const int rc = ensure_resources();
    if (rc) return rc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_status = reinterpret_cast<int*>(static_cast<char*>(d_work) + p.off_status);
  SCARF_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  SCARF_CUDA(launch_tc_structured(*s, fs, n, ds, d_table, nh, d_field, d_work, p, d_status, st, kernel_ev0(),
                                  kernel_ev1()));
  const int rc = check_device_status(d_status, st);
  if (!rc) collect_kernel_time();
  return rc;
}

}  // extern "C"

struct scarf_tc_batch {
  scarf::TcBatchPlan plan;
  void* d_work = nullptr;
  // Kept for re-uploads of the descriptors (host outputs on or off).
  std::vector<scarf_srm_setup> setups;
  std::vector<scarf::TcBatchInput> in;
  // Overlapped copy-out to host buffers (scarf_srm_tc_batch_set_host_outputs).
  std::vector<float*> host;
  int* flags = nullptr;      // host-mapped, one per field
  int* flags_dev = nullptr;  // their device address
  cudaStream_t copy_stream = nullptr;
  scarf::BuilderFork fork;   // the C-image builder's stream beside the R/S builder
  ~scarf_tc_batch() {
    if (flags) cudaFreeHost(flags);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (fork.side) cudaStreamDestroy(fork.side);
    if (fork.fork) cudaEventDestroy(fork.fork);
    if (fork.join) cudaEventDestroy(fork.join);
  }
};

namespace {
std::vector<scarf::TcBatchInput> batch_inputs(const scarf_tc_field* fields, int nfields) {
  std::vector<scarf::TcBatchInput> in(nfields);
  for (int f = 0; f < nfields; ++f) {
    in[f].s = fields[f].setup;
    for (int c = 0; c < 3; ++c) {
      in[f].fs[c] = fields[f].fs[c];
      in[f].n[c] = fields[f].n[c];
    }
    in[f].ds = fields[f].ds;
    in[f].d_table = fields[f].d_table;
    in[f].nh = fields[f].nh;
    in[f].d_field = fields[f].d_field;
    in[f].tj = fields[f].tile_j;
  }
  return in;
}

bool batch_fields_valid(const scarf_tc_field* fields, int nfields) {
  if (!fields || nfields <= 0) return false;
  for (int f = 0; f < nfields; ++f)
    if (!fields[f].setup || !fields[f].d_table || !fields[f].d_field || fields[f].nh <= 0) return false;
  return true;
}
}  // namespace

extern "C" {

size_t scarf_srm_tc_batch_workspace_bytes(const scarf_tc_field* fields, int nfields) {
  if (!batch_fields_valid(fields, nfields)) return 0;
  const auto in = batch_inputs(fields, nfields);
  return tc_batch_plan(in.data(), nfields, nullptr);
}

int scarf_srm_tc_batch_create(const scarf_tc_field* fields, int nfields, void* d_work, size_t work_bytes,
                              scarf_tc_batch** batch) {
  if (!batch || !d_work || !batch_fields_valid(fields, nfields)) return fail(SCARF_ERR_ARG, "invalid argument");
  if (reinterpret_cast<uintptr_t>(d_work) & 255u) return fail(SCARF_ERR_ARG, "workspace must be 256-byte aligned");
  const auto in = batch_inputs(fields, nfields);
  auto* b = new (std::nothrow) scarf_tc_batch();
  if (!b) return fail(SCARF_ERR_NOMEM, "out of host memory");
  if (!tc_batch_plan(in.data(), nfields, &b->plan)) {
    delete b;
    return fail(SCARF_ERR_ARG, "fields cannot share one launch (row-tile shapes differ or a grid is empty)");
  }
  if (work_bytes < b->plan.bytes) {
    const size_t need = b->plan.bytes;
    delete b;
    return fail(SCARF_ERR_ARG, "workspace too small: %zu < %zu", work_bytes, need);
  }
  b->d_work = d_work;
  b->setups.resize(nfields);
  b->in = in;
  for (int f = 0; f < nfields; ++f) {
    b->setups[f] = *fields[f].setup;
    b->in[f].s = &b->setups[f];
  }
  cudaError_t e = tc_batch_upload(b->in.data(), b->plan, d_work);
  // Created here, outside any stream capture, for every later launch.
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->fork.side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork.join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "scarf_srm_tc_batch_create");
  }
  *batch = b;
  return SCARF_OK;
}

int scarf_srm_tc_batch_set_host_outputs(scarf_tc_batch* batch, float* const* host_fields) {
  if (!batch) return fail(SCARF_ERR_ARG, "NULL batch");
  const int nf = batch->plan.nfields;
  if (host_fields) {
    for (int f = 0; f < nf; ++f)
      if (!host_fields[f]) return fail(SCARF_ERR_ARG, "host output %d is NULL", f);
    if (!batch->flags) {
      void* h = nullptr;
      SCARF_CUDA(cudaHostAlloc(&h, sizeof(int) * nf, cudaHostAllocMapped));
      batch->flags = static_cast<int*>(h);
      void* d = nullptr;
      SCARF_CUDA(cudaHostGetDevicePointer(&d, h, 0));
      batch->flags_dev = static_cast<int*>(d);
    }
    if (!batch->copy_stream) SCARF_CUDA(cudaStreamCreateWithFlags(&batch->copy_stream, cudaStreamNonBlocking));
    std::memset(batch->flags, 0, sizeof(int) * nf);
    batch->host.assign(host_fields, host_fields + nf);
  } else {
    batch->host.clear();
  }
  SCARF_CUDA(tc_batch_upload(batch->in.data(), batch->plan, batch->d_work, host_fields ? batch->flags_dev : nullptr));
  return SCARF_OK;
}

int scarf_srm_tc_batch_launch(const scarf_tc_batch* batch, void* stream) {
  if (!batch) return fail(SCARF_ERR_ARG, "NULL batch");
  if (t_ctx->cfg.kernel_timing) {
    const int rc = ensure_resources();
    if (rc) return rc;
  }
  SCARF_CUDA(tc_batch_launch(batch->plan, batch->d_work, static_cast<cudaStream_t>(stream), kernel_ev0(),
                             kernel_ev1(), &batch->fork));
  return SCARF_OK;
}

int scarf_srm_tc_batch_wait(const scarf_tc_batch* batch, void* stream) {
  if (!batch) return fail(SCARF_ERR_ARG, "NULL batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!batch->host.empty()) {
    // Copy each field to its host buffer as soon as its flag rises, while
    // the launch computes the others; whatever is left when the stream
    // has finished (a failed launch) is copied then.
    const int nf = batch->plan.nfields;
    volatile int* flags = batch->flags;
    std::vector<char> copied(nf, 0);
    int left = nf;
    bool idle = false;
    for (uint32_t spins = 0; left > 0;) {
      bool progress = false;
      for (int f = 0; f < nf; ++f) {
        if (copied[f] || (!idle && !flags[f])) continue;
        const size_t bytes = sizeof(float) * static_cast<size_t>(batch->in[f].n[0]) * batch->in[f].n[1] *
                             batch->in[f].n[2];
        SCARF_CUDA(cudaMemcpyAsync(batch->host[f], batch->in[f].d_field, bytes, cudaMemcpyDeviceToHost,
                                   batch->copy_stream));
        copied[f] = 1;
        --left;
        progress = true;
      }
      if (!progress && (++spins & 1023u) == 0 && cudaStreamQuery(st) != cudaErrorNotReady) {
        cudaGetLastError();
        idle = true;
      }
      if (!progress) cpu_relax();
    }
    SCARF_CUDA(cudaStreamSynchronize(batch->copy_stream));
    std::memset(batch->flags, 0, sizeof(int) * nf);
  }
  const int* d_status = reinterpret_cast<const int*>(static_cast<const char*>(batch->d_work) + batch->plan.off_status);
  const int rc = check_device_status(d_status, st);
  if (!rc) collect_kernel_time();
  return rc;
}

void scarf_srm_tc_batch_destroy(scarf_tc_batch* batch) { delete batch; }

int scarf_set_kernel_timing(int enable) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.kernel_timing = enable != 0;
  return SCARF_OK;
}

int scarf_set_device_memory_cap(size_t bytes) {
  scarf::set_device_memory_cap(bytes);
  return SCARF_OK;
}

size_t scarf_device_memory_in_use(void) { return scarf::device_memory_in_use(); }

int scarf_release_device_memory(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (t_ctx->res.device >= 0) {
    int dev = 0;
    SCARF_CUDA(cudaGetDevice(&dev));
    SCARF_CUDA(cudaSetDevice(t_ctx->res.device));
    SCARF_CUDA(cudaDeviceSynchronize());
    t_ctx->res.release();
    SCARF_CUDA(cudaSetDevice(dev));
  }
  scarf::release_sampler_device_memory();
  scarf::release_fim_plans();
  return SCARF_OK;
}

int scarf_selftest_wait_limit(int blocks, int* device_status, double* waited_s) {
  if (blocks < 1 || blocks > 1024) return fail(SCARF_ERR_ARG, "blocks must be in 1..1024 (got %d)", blocks);
  void* d = nullptr;
  const cudaError_t ea = static_cast<cudaError_t>(scarf::device_alloc(&d, 16));
  if (ea != cudaSuccess) return cuda_fail(ea, "self-test scratch");
  struct Scratch {
    void* p;
    ~Scratch() { scarf::device_free(p, 16); }
  } scratch{d};
  int status = -1;
  unsigned long long waited = 0;
  bool timed_out = false;
  SCARF_CUDA(scarf::run_wait_limit_probe(blocks, d, t_ctx->cfg.stream, &status, &waited, &timed_out));
  if (device_status) *device_status = status;
  if (waited_s) *waited_s = static_cast<double>(waited) * 1e-9;
  if (!timed_out)
    return fail(SCARF_ERR_DEVICE, "bounded-wait self-test: status word %d after the waits, not the timeout code",
                status);
  return SCARF_OK;
}

float scarf_last_kernel_ms(void) { return t_ctx->last_kernel_ms; }

int scarf_set_tc_chunk(int harmonics) {
  if (harmonics < 0) return fail(SCARF_ERR_ARG, "chunk must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  tc_set_chunk_harmonics(harmonics);
  return SCARF_OK;
}

int scarf_set_output_overlap(int items_per_slab) {
  if (items_per_slab < 0) return fail(SCARF_ERR_ARG, "items_per_slab must be >= 0");
  std::lock_guard<std::mutex> lk(g_mu);
  t_ctx->cfg.overlap_items = items_per_slab == 1 ? kDefaultSlabItems : items_per_slab;
  return SCARF_OK;
}

int scarf_set_tc_variant(int variant) {
  if (variant != SCARF_TC_PAIR && variant != SCARF_TC_SINGLE && variant != SCARF_TC_SINGLE_TMEM_A)
    return fail(SCARF_ERR_ARG, "unknown tensor-core variant %d", variant);
  std::lock_guard<std::mutex> lk(g_mu);
  tc_set_variant(variant);
  return SCARF_OK;
}

int scarf_fim_internal_grid(int ndim, const float nc[3], const float fc[3], float dh, const float cl[3], int pad,
                            int npts[3], float off_axis[3], float flags[2]) {
  if ((ndim != 2 && ndim != 3) || !nc || !fc || !cl || !npts || !off_axis || !flags || !(dh > 0.0f))
    return fail(SCARF_ERR_ARG, "invalid FIM grid arguments");
  FimInputs in{};
  in.ndim = ndim;
  in.dh = dh;
  in.pad = pad;
  for (int c = 0; c < 3; ++c) {
    in.nc[c] = nc[c];
    in.fc[c] = fc[c];
    in.cl[c] = (c < ndim) ? cl[c] : 0.0f;
  }
  FimGrid g{};
  fim_grid(in, &g);
  for (int c = 0; c < 3; ++c) {
    npts[c] = g.npts[c];
    off_axis[c] = g.off_axis[c];
  }
  flags[0] = g.info0;
  flags[1] = g.info1;
  return SCARF_OK;
}

size_t scarf_fim_workspace_bytes(const int npts[3], int npoi) {
  if (!npts || npts[0] <= 0 || npts[1] <= 0 || npts[2] <= 0 || npoi < 0) return 0;
  FimGrid g{};
  for (int c = 0; c < 3; ++c) g.npts[c] = npts[c];
  return fim_workspace_bytes(g, npoi);
}

int scarf_set_direct_sincos(int mode) {
  if (mode != SCARF_SINCOS_FAST && mode != SCARF_SINCOS_ACCURATE)
    return fail(SCARF_ERR_ARG, "direct-sum sincos mode %d (0 accurate, 1 fast)", mode);
  std::lock_guard<std::mutex> lk(g_mu);
  direct_set_sincos(mode == SCARF_SINCOS_FAST ? 1 : 0);
  return SCARF_OK;
}

int scarf_set_tc_precision(int operand_type, int terms) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!tc_set_precision(operand_type, terms))
    return fail(SCARF_ERR_ARG, "tensor-core precision: operand type %d (0 FP16, 1 BF16), terms %d (2 or 3)",
                operand_type, terms);
  return SCARF_OK;
}

size_t scarf_field_stats_workspace_bytes(long long n) { return stats_partials_bytes(n) + 256; }

int scarf_field_stats(const float* d_field, long long n, void* d_work, size_t work_bytes, float* mean, float* var,
                      void* stream) {
  if (!d_field || n < 2 || !d_work || !mean || !var) return fail(SCARF_ERR_ARG, "invalid argument");
  if (work_bytes < scarf_field_stats_workspace_bytes(n)) return fail(SCARF_ERR_ARG, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* d_part = static_cast<double*>(d_work);
  float* d_out = reinterpret_cast<float*>(static_cast<char*>(d_work) + stats_partials_bytes(n));
  SCARF_CUDA(launch_field_stats(d_field, n, d_part, d_out, st));
  float mv[2];
  SCARF_CUDA(cudaMemcpyAsync(mv, d_out, sizeof(mv), cudaMemcpyDeviceToHost, st));
  SCARF_CUDA(cudaStreamSynchronize(st));
  *mean = mv[0];
  *var = mv[1];
  return SCARF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- autotune --
// Plan choices of the tensor-core form measured on this GPU: kernel form,
// row tile (128 / tile_j) x tile_j and column axis, per shape bucket (grid
// extents rounded up to a multiple of 16; the key also names the GPU and the
// driver). Entries live in memory and, when a cache file is set, one line
// each in that file ("key variant tile_j permute ms split").
namespace {
struct TuneState {
  std::mutex mu;
  int mode = 0;  // 0: the default plans; 1: tuned choices where a bucket has one
  std::string path;
  std::map<std::string, scarf::TcChoice> entries;
};
TuneState g_tune;

// GPU name and driver version of the current device, looked up once per
// device (a properties query costs milliseconds; plans are made per call).
std::string device_tag() {
  static std::mutex mu;
  static std::map<int, std::string> tags;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return "unknown";
  }
  std::lock_guard<std::mutex> lk(mu);
  const auto it = tags.find(dev);
  if (it != tags.end()) return it->second;
  int drv = 0;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    return "unknown";
  }
  cudaDriverGetVersion(&drv);
  std::string name = prop.name;
  for (char& c : name)
    if (c == ' ' || c == ':') c = '_';
  return tags[dev] = name + "_drv" + std::to_string(drv);
}

std::string bucket_key(int ndim, const int n[3], bool fixed_columns) {
  std::ostringstream k;
  k << device_tag() << ':' << ndim << ':';
  for (int a = 0; a < 3; ++a) k << (a ? "x" : "") << (n[a] + 15) / 16 * 16;
  k << (fixed_columns ? ":z" : ":p");
  return k.str();
}

void load_cache_locked(const std::string& path) {
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string key;
    scarf::TcChoice c{};
    if (is >> key >> c.variant >> c.tile_j >> c.permute >> c.ms) {
      if (!(is >> c.split) || c.split < 1) c.split = 1;  // lines written before the split existed
      g_tune.entries[key] = c;
    }
  }
}

void store_locked(const std::string& key, const scarf::TcChoice& c) {
  g_tune.entries[key] = c;
  if (g_tune.path.empty()) return;
  std::ofstream f(g_tune.path, std::ios::app);
  f << key << ' ' << c.variant << ' ' << c.tile_j << ' ' << c.permute << ' ' << c.ms << ' ' << std::max(1, c.split)
    << '\n';
}

// Time of one plan on the caller's data, table builds and kernel (the
// fastest of three runs after a warm-up run), or a negative value when the
// plan cannot run.
float time_plan(const scarf_srm_setup& s, const int fs[3], const int n[3], float ds, const float* d_table, int nh,
                float* d_field, void* d_work, const TcPlan& p, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
  int* d_status = reinterpret_cast<int*>(static_cast<char*>(d_work) + p.off_status);
  float best = -1.0f;
  for (int rep = 0; rep < 4; ++rep) {
    float ms = -1.0f;
    if (cudaMemsetAsync(d_status, 0, sizeof(int), st) != cudaSuccess || cudaEventRecord(e0, st) != cudaSuccess ||
        launch_tc_structured(s, fs, n, ds, d_table, nh, d_field, d_work, p, d_status, st) != cudaSuccess ||
        cudaEventRecord(e1, st) != cudaSuccess) {
      cudaGetLastError();
      return -1.0f;
    }
    int h = 1;
    if (cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess || h != 0 || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      cudaGetLastError();
      return -1.0f;
    }
    if (rep > 0 && (best < 0.0f || ms < best)) best = ms;
  }
  return best;
}
}  // namespace

namespace scarf {
bool tc_tuned_choice(int ndim, const int n[3], bool fixed_columns, TcChoice* c) {
  std::lock_guard<std::mutex> lk(g_tune.mu);
  if (g_tune.mode == 0 || g_tune.entries.empty()) return false;
  const auto it = g_tune.entries.find(bucket_key(ndim, n, fixed_columns));
  if (it == g_tune.entries.end()) return false;
  *c = it->second;
  return true;
}
}  // namespace scarf

extern "C" {

int scarf_set_tc_autotune(int mode) {
  if (mode != 0 && mode != 1) return fail(SCARF_ERR_ARG, "autotune mode must be 0 or 1");
  std::lock_guard<std::mutex> lk(g_tune.mu);
  g_tune.mode = mode;
  return SCARF_OK;
}

int scarf_set_tc_tune_cache(const char* path) {
  std::lock_guard<std::mutex> lk(g_tune.mu);
  g_tune.path = path ? path : "";
  if (!g_tune.path.empty()) load_cache_locked(g_tune.path);
  return SCARF_OK;
}

int scarf_srm_tc_autotune(const scarf_srm_setup* s, const int fs[3], const int n[3], float ds, const float* d_table,
                          int nh, int fixed_columns, void* stream, scarf_tc_tuning* out) {
  if (!s || !fs || !n || !d_table || nh <= 0 || !out) return fail(SCARF_ERR_ARG, "invalid argument");
  if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return fail(SCARF_ERR_ARG, "empty grid");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Whole stages of at most 2 048 harmonics: enough for the pipeline to
  // reach its steady state, short enough to try every candidate.
  const int nh_probe = std::min(nh, 2048);
  const int forms[3] = {SCARF_TC_SINGLE, SCARF_TC_PAIR, SCARF_TC_SINGLE_TMEM_A};
  const int tiles[5] = {1, 2, 4, 8, 16};
  std::vector<TcPlan> plans;
  std::vector<scarf::TcChoice> choices;
  int nsm = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
  }
  for (int v : forms)
    for (int tj : tiles)
      for (int perm = 0; perm < (fixed_columns ? 1 : 2); ++perm) {
        TcPlan p{};
        if (!tc_make_plan(s->ndim, n, nh_probe, &p, tj, perm != 0, v)) continue;
        if (perm == 1 && !plans.empty()) {  // the longest axis may already be z: same plan
          const TcPlan& q = plans.back();
          if (q.ax_c == p.ax_c && q.tj == p.tj && q.pair == p.pair && q.tmem_a == p.tmem_a) continue;
        }
        plans.push_back(p);
        choices.push_back(scarf::TcChoice{v, tj, perm, 0.0f, 1});
        // Fewer tiles than SMs: splitting the harmonics over 2-8 items per
        // tile fills the GPU (device fields only: scarf_execute needs the
        // final values in the kernel for its statistics and slab copies).
        const long long tiles_m = static_cast<long long>(p.bix) * p.bjx * p.bn;
        if (fixed_columns || p.pair || tiles_m >= nsm) continue;
        for (int split = 2; split <= 8 && tiles_m * split <= 2LL * nsm; split *= 2) {
          TcPlan q{};
          if (!tc_make_plan(s->ndim, n, nh_probe, &q, tj, perm != 0, v, split) || q.split != split) continue;
          plans.push_back(q);
          choices.push_back(scarf::TcChoice{v, tj, perm, 0.0f, split});
        }
      }
  size_t work = 0;
  for (const TcPlan& p : plans) work = std::max(work, p.bytes);
  const size_t npts = static_cast<size_t>(n[0]) * n[1] * n[2];
  void* d_work = nullptr;
  float* d_field = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto release = [&]() {
    scarf::device_free(d_work, work);
    scarf::device_free(d_field, sizeof(float) * npts);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  if (scarf::device_alloc(&d_work, work) != cudaSuccess ||
      scarf::device_alloc(reinterpret_cast<void**>(&d_field), sizeof(float) * npts) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    release();
    return fail(SCARF_ERR_NOMEM, "autotune: device allocation failed");
  }
  int best = -1;
  for (size_t c = 0; c < plans.size(); ++c) {
    choices[c].ms = time_plan(*s, fs, n, ds, d_table, nh_probe, d_field, d_work, plans[c], st, e0, e1);
    if (choices[c].ms > 0.0f && (best < 0 || choices[c].ms < choices[best].ms)) best = static_cast<int>(c);
  }
  release();
  if (best < 0) return fail(SCARF_ERR_CUDA, "autotune: no candidate plan ran");
  // The default plan stays unless a candidate beats it by 3 %: probe timings
  // of a few milliseconds carry about that much noise.
  TcPlan dp{};
  if (tc_make_plan(s->ndim, n, nh_probe, &dp, 0, fixed_columns == 0, SCARF_TC_SINGLE)) {
    for (size_t c = 0; c < plans.size(); ++c) {
      const TcPlan& q = plans[c];
      if (q.ax_c == dp.ax_c && q.tj == dp.tj && q.pair == dp.pair && q.tmem_a == dp.tmem_a && q.split == 1 &&
          choices[c].ms > 0.0f && choices[best].ms > 0.97f * choices[c].ms)
        best = static_cast<int>(c);
    }
  }
  const scarf::TcChoice& b = choices[best];
  {
    std::lock_guard<std::mutex> lk(g_tune.mu);
    store_locked(bucket_key(s->ndim, n, fixed_columns != 0), b);
  }
  out->variant = b.variant;
  out->tile_j = b.tile_j;
  out->permute = b.permute;
  out->ms = b.ms;
  out->split = std::max(1, b.split);
  return SCARF_OK;
}

int scarf_srm_tc_batch_autotune(const scarf_tc_field* fields, int nfields, void* stream, scarf_tc_tuning* out) {
  if (!out || !batch_fields_valid(fields, nfields)) return fail(SCARF_ERR_ARG, "invalid argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int forms[2] = {SCARF_TC_SINGLE, SCARF_TC_PAIR};
  const int tiles[5] = {1, 2, 4, 8, 16};
  std::lock_guard<std::mutex> lk(g_mu);  // the kernel form is global while a batch is planned
  const int saved = tc_get_variant();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return fail(SCARF_ERR_CUDA, "autotune: event creation failed");
  }
  scarf::TcChoice best{-1, 0, 1, 0.0f, 1}, deflt{-1, 0, 1, 0.0f, 1};
  int auto_tj = 8;  // the row tile the batch would get with tile_j = 0
  {
    auto in0 = batch_inputs(fields, nfields);
    for (auto& e : in0) e.tj = 0;
    TcBatchPlan bp0;
    if (tc_batch_plan(in0.data(), nfields, &bp0)) auto_tj = bp0.tj;
  }
  for (int v : forms) {
    tc_set_variant(v);
    for (int tj : tiles) {
      auto in = batch_inputs(fields, nfields);
      for (auto& e : in) e.tj = tj;
      TcBatchPlan bp;
      if (!tc_batch_plan(in.data(), nfields, &bp)) continue;
      void* d_work = nullptr;
      if (scarf::device_alloc(&d_work, bp.bytes) != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
      float ms = -1.0f;
      if (tc_batch_upload(in.data(), bp, d_work) == cudaSuccess) {
        const int* d_status = reinterpret_cast<const int*>(static_cast<const char*>(d_work) + bp.off_status);
        for (int rep = 0; rep < 4; ++rep) {  // a warm-up run, then the fastest of three
          int h = 1;
          float t = -1.0f;
          if (cudaEventRecord(e0, st) != cudaSuccess || tc_batch_launch(bp, d_work, st) != cudaSuccess ||
              cudaEventRecord(e1, st) != cudaSuccess ||
              cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess || h != 0 || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
            ms = -1.0f;
            break;
          }
          if (rep > 0 && (ms < 0.0f || t < ms)) ms = t;
        }
      }
      cudaGetLastError();
      scarf::device_free(d_work, bp.bytes);
      if (ms > 0.0f && (best.variant < 0 || ms < best.ms)) best = scarf::TcChoice{v, tj, 1, ms, 1};
      if (ms > 0.0f && v == SCARF_TC_SINGLE && tj == auto_tj) deflt = scarf::TcChoice{v, tj, 1, ms, 1};
    }
  }
  // As for single grids: the default (one-CTA form, automatic row tile)
  // stays unless a candidate beats it by 3 %.
  if (deflt.variant >= 0 && best.ms > 0.97f * deflt.ms) best = deflt;
  tc_set_variant(saved);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best.variant < 0) return fail(SCARF_ERR_CUDA, "autotune: no candidate batch plan ran");
  out->variant = best.variant;
  out->tile_j = best.tile_j;
  out->permute = 1;
  out->ms = best.ms;
  out->split = 1;
  return SCARF_OK;
}

}  // extern "C"
