// Tensor-core SRM sum that allocates nothing.
//
// scarf_srm_tc_structured needs a workspace for its per-axis phase tables and
// a status word, which its caller allocates. Some callers cannot allocate
// device memory when they need a field: applications whose device memory is
// entirely owned by another allocator (a framework's caching pool, or an MPI
// code that reserves the GPU's memory at start-up and allows no later
// cudaMalloc), and per-step loops where the device-wide synchronisation that
// cudaMalloc/cudaFree imply would stall the pipeline. This variant takes the
// same inputs and output and keeps its scratch in a fixed, file-scope device
// array instead.
//
// The array is kNoAllocScratchBytes (64 MiB); every GPU that loads the library
// holds it until the process exits. Calls whose tables need more are
// rejected with SCARF_ERR_ARG. All calls on a device share the array, which
// keeps the previous call's contents: every table entry is rewritten by each
// call and the status word is cleared first, but calls that overlap on the
// GPU (different streams, or host threads racing) would overwrite each
// other's tables -- serialise them.
//
// The device address of the array is looked up with cudaGetSymbolAddress the
// first time the entry point runs in each device context (with that device
// current) and cached under the context's process-unique id, so a
// cudaDeviceReset, or another driver-API context made current on the same
// device, makes the next call look the address up again instead of using a
// stale one. Each call copies its status word back and synchronises its
// stream, so it cannot be recorded into a CUDA graph.
//
// The plan (kernel form, row tile, column axis) follows the same rule as
// scarf_srm_tc_structured, tuned plans included, so both entry points run the
// same plan and scarf_srm_tc_workspace_bytes gives the scratch this one needs.
#include <cuda_runtime.h>

#include <mutex>

#include "scarf3d_b200.h"
#include "srm_kernels.h"

// 64 MiB of scratch per device, shared by every call on that device.
#define SCARF_NOALLOC_SCRATCH_BYTES (size_t(64) << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCARF_NOALLOC_SCRATCH_BYTES];

namespace scarf {

int record_error(int code, const char* msg);

namespace {

constexpr size_t kNoAllocScratchBytes = SCARF_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct ScratchSlot {
  unsigned long long ctx_id;  // process-unique id of the context the address belongs to
  void* ptr;
};
ScratchSlot g_noalloc_slot[kMaxDevices] = {};

// Device address of g_noalloc_scratch in the current context. In host code
// the symbol itself is only a host-side stand-in and must never be passed to
// a kernel. The lookup (set-up) runs once per device context: when the
// context's id cannot be read it runs on every call instead.
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  unsigned long long id = current_context_id();
  if (id != 0 && g_noalloc_slot[dev].ptr && g_noalloc_slot[dev].ctx_id == id) {
    *out = g_noalloc_slot[dev].ptr;
    return cudaSuccess;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // also makes the primary context current if none was
  if (e != cudaSuccess) return e;
  if (id == 0) id = current_context_id();
  g_noalloc_slot[dev] = ScratchSlot{id, id != 0 ? p : nullptr};
  *out = p;
  return cudaSuccess;
}

}  // namespace
}  // namespace scarf

using namespace scarf;

extern "C" size_t scarf_srm_tc_noalloc_capacity_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int scarf_srm_tc_structured_noalloc(const scarf_srm_setup* s, const int fs[3], const int n[3], float ds,
                                               const float* d_table, int nh, float* d_field, void* stream) {
  if (!s || !fs || !n || !d_table || !d_field || nh <= 0)
    return record_error(SCARF_ERR_ARG, "scarf_srm_tc_structured_noalloc: invalid argument");
  TcPlan p{};
  if (!device_field_plan(s->ndim, n, nh, &p))
    return record_error(SCARF_ERR_ARG, "scarf_srm_tc_structured_noalloc: invalid grid");
  if (p.bytes > kNoAllocScratchBytes)
    return record_error(SCARF_ERR_ARG,
                        "scarf_srm_tc_structured_noalloc: this grid and harmonic count need more scratch than "
                        "the fixed 64 MiB device array holds; use scarf_srm_tc_structured with a workspace");
  void* scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) return record_error(SCARF_ERR_CUDA, cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* d_status = reinterpret_cast<int*>(static_cast<char*>(scratch) + p.off_status);
  e = cudaMemsetAsync(d_status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch_tc_structured(*s, fs, n, ds, d_table, nh, d_field, scratch, p, d_status, st);
  int h_status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return record_error(SCARF_ERR_CUDA, cudaGetErrorString(e));
  if (h_status != 0)
    return record_error(SCARF_ERR_DEVICE, "scarf_srm_tc_structured_noalloc: a bounded wait in the kernel expired");
  return SCARF_OK;
}
