// Diagnostics of the device-side failure path.
//
// Every wait of the tensor-core pipelines (mbarrier phases between the TMA
// producer, the MMA issuer and the epilogue warps) is bounded: when a phase
// does not complete within the limit, the waiting thread raises the grid's
// device error word and returns instead of spinning, the kernel winds down,
// and gsht_device_status reports GSHT_ERR_TIMEOUT. gsht_check_bounded_wait
// runs that path on purpose: one thread waits, with the pipelines' own
// bounded wait, on an mbarrier that nothing arrives at. No fault, trap or
// hang is involved; the GPU context stays usable.
#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

// Error code a diagnostic wait raises (the pipelines use 1..5).
constexpr int kDiagnosticWaitCode = 100;

__global__ void k_wait_never_completes(int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_barrier_init();
  }
  __syncthreads();
  // Phase 0 needs one arrival; none comes, so the wait runs to its limit.
  if (threadIdx.x == 0) tc::mbar_wait(&bar, 0, err, kDiagnosticWaitCode);
  __syncthreads();
}

}  // namespace
}  // namespace gsht

using namespace gsht;

extern "C" gsht_status gsht_check_bounded_wait(const gsht_grid* g, void* stream) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  GSHT_CUDA(cudaSetDevice(g->device));
  k_wait_never_completes<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(g->d_err);
  GSHT_LAUNCH_CHECK("k_wait_never_completes");
  return GSHT_OK;
}
