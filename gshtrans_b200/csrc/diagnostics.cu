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

// Error code a diagnostic wait raises (the pipelines use 1..16).
constexpr int kDiagnosticWaitCode = 100;

// Per-role cycle counters of traced tensor-core launches, [form][direction]
// (form 0: BF16x3, 1: Ozaki), reset by each traced launch.
__device__ unsigned long long g_trace_counters[2][2][tc::kTrSlots];

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

std::atomic<int> g_tc_trace{0};

unsigned long long* trace_slots(int form, int dir, cudaStream_t s) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_trace_counters) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  auto* slots = static_cast<unsigned long long*>(p) + (form * 2 + dir) * tc::kTrSlots;
  if (cudaMemsetAsync(slots, 0, sizeof(unsigned long long) * tc::kTrSlots, s) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return slots;
}

}  // namespace gsht

using namespace gsht;

extern "C" gsht_status gsht_tc_trace_enable(int on) {
  g_tc_trace.store(on != 0);
  return GSHT_OK;
}

extern "C" gsht_status gsht_tc_trace_read(int form, int direction, double* out, int n) {
  if (!out || n < GSHT_TRACE_SLOTS) return fail(GSHT_ERR_BAD_ARG, "need %d output slots", GSHT_TRACE_SLOTS);
  if (form != GSHT_BF16X3 && form != GSHT_OZAKI && form != GSHT_OZAKI4)
    return fail(GSHT_ERR_BAD_ARG, "form %d has no traced kernel", form);
  if (direction != 0 && direction != 1) return fail(GSHT_ERR_BAD_ARG, "direction %d", direction);
  static_assert(GSHT_TRACE_SLOTS == tc::kTrSlots, "trace slot count");
  unsigned long long h[2][2][tc::kTrSlots];
  GSHT_CUDA(cudaMemcpyFromSymbol(h, g_trace_counters, sizeof(h)));
  const int f = form == GSHT_BF16X3 ? 0 : 1;
  for (int i = 0; i < tc::kTrSlots; i++) out[i] = (double)h[f][direction][i];
  return GSHT_OK;
}

extern "C" gsht_status gsht_check_bounded_wait(const gsht_grid* g, void* stream) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  GSHT_CUDA(cudaSetDevice(g->device));
  k_wait_never_completes<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(g->d_err);
  GSHT_LAUNCH_CHECK("k_wait_never_completes");
  return GSHT_OK;
}
