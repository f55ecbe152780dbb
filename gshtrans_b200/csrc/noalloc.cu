// gsht_inverse_noalloc: the FP64 inverse transform of one field with its
// scratch memory (per-order operand rows, their layout, and the spectral
// buffer) taken from a fixed array in the library's device memory instead of
// cudaMalloc.
//
// For callers that must not allocate device memory at the time they
// transform: code that runs while another component owns the allocator (a
// caching or arena allocator that forbids stray cudaMalloc/cudaFree), code
// on a latency-critical path where an allocation's implicit device
// synchronisation is not acceptable, and code that must not fail with an
// out-of-memory error after start-up. The caller still provides the input
// coefficients and the output field in device memory.
//
// The scratch array is a file-scope __device__ array of kNoAllocScratchBytes
// (16 MiB), which every GPU that loads this library holds until the process
// exits. Host code never dereferences the array's name (on the host it only
// stands in for the symbol); its device address is obtained once per device
// with cudaGetSymbolAddress.
#include <cstdio>
#include <mutex>

#include "gsht_internal.cuh"

namespace gsht {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device `dev`, looked up
// once per device (the first call on a device performs the lookup).
gsht_status scratch_address(int dev, void** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(GSHT_ERR_UNSUPPORTED, "device index %d too large", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return GSHT_OK;
}

// Operand layout of one call (the same per-order rows as OperandLayout),
// written by one thread into the scratch so that nothing is uploaded.
__global__ void k_noalloc_layout(int lmax, int na, int rows, int pad, long long* off,
                                 int* pitch) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  long long acc = 0;
  for (int m = 0; m <= lmax; m++) {
    const int l0 = m > na ? m : na;
    const int p = (lmax - l0 + 1 + pad - 1) / pad * pad;
    pitch[m] = p;
    off[m] = acc;
    acc += (long long)p * rows;
  }
  off[lmax + 1] = acc;
}


}  // namespace
}  // namespace gsht

using namespace gsht;

extern "C" gsht_status gsht_inverse_noalloc(const gsht_grid* g, int lmax, int n, int is_real,
                                            const void* in, void* out, void* stream) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (lmax < 1 || lmax > g->L)
    return fail(GSHT_ERR_BAD_ARG, "lmax %d outside [1, %d] (lmax 0 is not served here)", lmax, g->L);
  if (n < g->min_n || n > g->nmax)
    return fail(GSHT_ERR_BAD_ARG, "upper index %d not in the grid's range [%d, %d]", n, g->min_n, g->nmax);
  if ((n < 0 ? -n : n) > lmax) return fail(GSHT_ERR_BAD_ARG, "|n| exceeds lmax");
  if (!is_real && g->mrange != GSHT_RANGE_ALL)
    return fail(GSHT_ERR_BAD_ARG, "complex fields need MRange = All");
  GSHT_CUDA(cudaSetDevice(g->device));
  if (pointer_kind(in, g->device) != kDevicePtr || pointer_kind(out, g->device) != kDevicePtr)
    return fail(GSHT_ERR_BAD_ARG,
                "gsht_inverse_noalloc needs in and out in the memory of the grid's device (%d)",
                g->device);
  if (!aligned16(in) || !aligned16(out))
    return fail(GSHT_ERR_BAD_ARG, "device buffers must be 16-byte aligned");

  const Table* t = g->table(n);
  if (!t->t64) return fail(GSHT_ERR_UNSUPPORTED, "gsht_inverse_noalloc needs the stored FP64 table");
  const int na = n < 0 ? -n : n;
  const int Q = is_real ? 1 : 2;  // one field: rows for +m (and -m)
  // Scratch layout: [off (lmax+2) x int64][pitch (lmax+1) x int32][operand][spec].
  long long opElems = 0;
  int kpMax = 0;
  for (int m = 0; m <= lmax; m++) {
    const int l0 = m > na ? m : na;
    const int p = (int)round_up(lmax - l0 + 1, kDegreePadFp64);
    kpMax = p > kpMax ? p : kpMax;
    opElems += (long long)p * Q;
  }
  const size_t offBytes = round_up(sizeof(long long) * (lmax + 2), 256);
  const size_t pitchBytes = round_up(sizeof(int) * (lmax + 1), 256);
  const size_t opBytes = round_up(sizeof(double) * 2 * opElems, 256);
  const size_t specBytes = sizeof(double) * 2 * spec_elems(g, lmax, is_real, 1);
  const size_t need = offBytes + pitchBytes + opBytes + specBytes;
  if (need > kNoAllocScratchBytes)
    return fail(GSHT_ERR_UNSUPPORTED,
                "gsht_inverse_noalloc needs %zu bytes of scratch for lmax %d; its static "
                "scratch holds %zu bytes (use gsht_inverse)",
                need, lmax, kNoAllocScratchBytes);
  void* base = nullptr;
  gsht_status st = scratch_address(g->device, &base);
  if (st != GSHT_OK) return st;
  char* sc = static_cast<char*>(base);
  auto* dOff = reinterpret_cast<long long*>(sc);
  auto* dPitch = reinterpret_cast<int*>(sc + offBytes);
  auto* op = reinterpret_cast<double*>(sc + offBytes + pitchBytes);
  auto* spec = reinterpret_cast<double*>(sc + offBytes + pitchBytes + opBytes);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  k_noalloc_layout<<<1, 1, 0, s>>>(lmax, na, Q, kDegreePadFp64, dOff, dPitch);
  GSHT_LAUNCH_CHECK("k_noalloc_layout");
  st = legendre_inverse_fp64_layout(g, t, lmax, is_real, 1, static_cast<const double*>(in),
                                    dOff, dPitch, kpMax, op, spec, s);
  if (st != GSHT_OK) return st;
  return fft_inverse(g, lmax, is_real, 1, spec, static_cast<double*>(out), s);
}
