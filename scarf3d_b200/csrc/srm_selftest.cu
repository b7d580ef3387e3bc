// Self-test of the bounded waits that every pipeline kernel relies on
// (mbar_wait_bounded): the blocks of one launch wait on an mbarrier that
// nothing ever arrives on. The first block past the time limit records
// kDevTimeout in the status word; the others see the flagged status at their
// next check and return. Nothing faults or traps, so the CUDA context stays
// usable, and the host learns of the stall from the status word alone --
// the same path by which a stalled pipeline kernel reports SCARF_ERR_DEVICE.
#include "common.cuh"
#include "srm_kernels.h"

namespace scarf {
namespace {

__global__ void wait_limit_probe(int* status, unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = global_timer_ns();
  mbar_wait_bounded(&bar, 0, status);  // phase 0 never completes
  if (threadIdx.x == 0) atomicMax(waited_ns, static_cast<unsigned long long>(global_timer_ns() - t0));
}

}  // namespace

cudaError_t run_wait_limit_probe(int blocks, void* d_scratch, cudaStream_t stream, int* status,
                                 unsigned long long* waited_ns, bool* timed_out) {
  int* d_status = static_cast<int*>(d_scratch);
  unsigned long long* d_waited = reinterpret_cast<unsigned long long*>(static_cast<char*>(d_scratch) + 8);
  cudaError_t e = cudaMemsetAsync(d_scratch, 0, 16, stream);
  if (e != cudaSuccess) return e;
  wait_limit_probe<<<blocks, 64, 0, stream>>>(d_status, d_waited);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(waited_ns, d_waited, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream)) !=
      cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
  *timed_out = *status == kDevTimeout;
  return cudaSuccess;
}

}  // namespace scarf
