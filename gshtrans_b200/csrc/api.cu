// C ABI of libgsht_cuda.so (declared in include/gsht.h): grid lifetime,
// argument validation with the reference's semantics, workspace management
// and the staging of host buffers.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <unordered_map>

#include <nvtx3/nvToolsExt.h>

#include "gsht_internal.cuh"

namespace gsht {

std::atomic<unsigned long long> g_launches{0};
thread_local unsigned long long t_launches = 0;
static thread_local char t_error[512] = "";

gsht_status fail(gsht_status s, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_error, sizeof(t_error), fmt, ap);
  va_end(ap);
  return s;
}

gsht_status cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? GSHT_ERR_OOM : GSHT_ERR_CUDA,
              "%s: %s", what, cudaGetErrorString(e));
}

PtrKind pointer_kind(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return kHostPtr;
  }
  if (a.type == cudaMemoryTypeManaged) return kDevicePtr;
  if (a.type == cudaMemoryTypeDevice) return a.device == device ? kDevicePtr : kOtherDevicePtr;
  return kHostPtr;
}

namespace {

// The allocator hook (gsht_set_allocator) and the allocations it made.
struct Hook {
  gsht_alloc_fn alloc = nullptr;
  gsht_free_fn free = nullptr;
  void* ctx = nullptr;
};
std::mutex g_alloc_mu;
Hook g_hook;
std::unordered_map<void*, Hook> g_hooked;  // pointer -> the hook that made it
unsigned long long g_alloc_calls = 0, g_free_calls = 0;
size_t g_live_bytes = 0;
std::unordered_map<void*, size_t> g_live;  // pointer -> bytes, every allocation

}  // namespace

cudaError_t dev_malloc_bytes(void** p, size_t bytes) {
  *p = nullptr;
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  if (g_hook.alloc) {
    void* q = g_hook.alloc(bytes, g_hook.ctx);
    if (!q) return cudaErrorMemoryAllocation;
    g_hooked[q] = g_hook;
    *p = q;
  } else {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      return e;
    }
  }
  g_alloc_calls++;
  g_live[*p] = bytes;
  g_live_bytes += bytes;
  return cudaSuccess;
}

void dev_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  auto l = g_live.find(p);
  if (l != g_live.end()) {
    g_live_bytes -= l->second;
    g_live.erase(l);
  }
  g_free_calls++;
  auto h = g_hooked.find(p);
  if (h != g_hooked.end()) {
    const Hook hook = h->second;
    g_hooked.erase(h);
    hook.free(p, hook.ctx);
  } else {
    cudaFree(p);
  }
}

namespace {

struct ProfRecord {
  int stage;
  cudaEvent_t a, b;
  unsigned long long launches;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRecord> g_prof;
// Records whose events have completed are folded into these per-stage
// totals once more than kProfFold are pending, so that a long profiled loop
// keeps a bounded number of events.
constexpr size_t kProfFold = 1024;
double g_prof_ms[GSHT_STAGE_COUNT] = {};
long g_prof_launches[GSHT_STAGE_COUNT] = {};

// Folds every record whose end event has completed (the caller holds g_prof_mu).
void fold_completed() {
  size_t keep = 0;
  for (auto& r : g_prof) {
    if (cudaEventQuery(r.b) == cudaSuccess) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess && r.stage >= 0 &&
          r.stage < GSHT_STAGE_COUNT) {
        g_prof_ms[r.stage] += t;
        g_prof_launches[r.stage] += (long)r.launches;
      }
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    } else {
      g_prof[keep++] = r;
    }
  }
  cudaGetLastError();
  g_prof.resize(keep);
}

}  // namespace

// NVTX range names of the stages (gsht.h GSHT_STAGE_*), for profilers that
// filter or group by range (ncu --nvtx, nsys); the ranges are pushed and
// popped whether or not stage timing is enabled.
const char* const kStageRangeNames[GSHT_STAGE_COUNT] = {
    "gsht:prep_inverse", "gsht:legendre_inverse", "gsht:fft_inverse", "gsht:fft_forward",
    "gsht:prep_forward", "gsht:legendre_forward", "gsht:accumulate_forward"};

StageTimer::StageTimer(int stage, cudaStream_t s) : stage_(stage), s_(s) {
  nvtxRangePushA(stage >= 0 && stage < GSHT_STAGE_COUNT ? kStageRangeNames[stage] : "gsht:stage");
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return;  // graph capture: stage timing is for direct calls only
  }
  if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
    cudaGetLastError();
    a_ = b_ = nullptr;
    return;
  }
  cudaEventRecord(a_, s_);
  launches0_ = t_launches;
}

StageTimer::~StageTimer() {
  nvtxRangePop();
  if (!a_) return;
  cudaEventRecord(b_, s_);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.push_back({stage_, a_, b_, t_launches - launches0_});
  if (g_prof.size() > kProfFold) fold_completed();
}

namespace {

// lmax == 0 special cases of the reference (GaussLegendreGrid.h:136-140 and
// :251-260): the forward ASSIGNS out[0] = in[0] / (2 sqrt(pi)); the inverse
// writes only out[0] = in[0] * 2 sqrt(pi), leaving the other points as they
// were.
__global__ void k_lmax0(int dir, int isReal, int count, long fieldSize,
                        const double* __restrict__ in, double* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= count) return;
  const double twoSqrtPi = 3.5449077018110320546;  // 2 sqrt(pi)
  if (dir == 0) {  // forward
    const long inStride = isReal ? fieldSize : 2 * fieldSize;
    const double re = in[f * inStride];
    const double im = isReal ? 0.0 : in[f * inStride + 1];
    out[2 * f] = re / twoSqrtPi;
    out[2 * f + 1] = im / twoSqrtPi;
  } else {
    const long outStride = isReal ? fieldSize : 2 * fieldSize;
    out[f * outStride] = in[2 * f] * twoSqrtPi;
    if (!isReal) out[f * outStride + 1] = in[2 * f + 1] * twoSqrtPi;
  }
}

gsht_status ensure_workspace(gsht_grid* g, size_t bytes) {
  if (g->ws_bytes >= bytes) return GSHT_OK;
  if (g->ws) {
    GSHT_CUDA(cudaDeviceSynchronize());
    dev_free(g->ws);
    g->ws = nullptr;
    g->ws_bytes = 0;
  }
  cudaError_t e = dev_malloc(&g->ws, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(GSHT_ERR_OOM, "workspace allocation of %zu bytes failed", bytes);
  }
  g->ws_bytes = bytes;
  return GSHT_OK;
}

// Copy streams and at least `events` events for the chunked host pipeline.
gsht_status ensure_copy_streams(gsht_grid* g, int events) {
  if (!g->h2d) GSHT_CUDA(cudaStreamCreateWithFlags(&g->h2d, cudaStreamNonBlocking));
  if (!g->d2h) GSHT_CUDA(cudaStreamCreateWithFlags(&g->d2h, cudaStreamNonBlocking));
  while ((int)g->xfer_ev.size() < events) {
    cudaEvent_t e;
    GSHT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    g->xfer_ev.push_back(e);
  }
  return GSHT_OK;
}

gsht_status validate(const gsht_grid* g, int lmax, int n, int is_real,
                     int precision, int count) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (count < 1 || count > 32767) return fail(GSHT_ERR_BAD_ARG, "count %d out of range [1, 32767]", count);
  if (lmax < 0 || lmax > g->L)
    return fail(GSHT_ERR_BAD_ARG, "lmax %d outside [0, %d]", lmax, g->L);
  if (n < g->min_n || n > g->nmax)
    return fail(GSHT_ERR_BAD_ARG, "upper index %d not in the grid's range [%d, %d]", n, g->min_n, g->nmax);
  if ((n < 0 ? -n : n) > lmax)
    return fail(GSHT_ERR_BAD_ARG, "|n| = %d exceeds lmax = %d", n < 0 ? -n : n, lmax);
  if (!is_real && g->mrange != GSHT_RANGE_ALL)
    return fail(GSHT_ERR_BAD_ARG, "complex fields need MRange = All");
  if (precision != GSHT_FP64 && precision != GSHT_BF16X3 && precision != GSHT_OZAKI &&
      precision != GSHT_RECURRENCE && precision != GSHT_OZAKI4)
    return fail(GSHT_ERR_UNSUPPORTED, "precision %d not available", precision);
  if (precision == GSHT_RECURRENCE && !(g->forms & GSHT_FORM_RECURRENCE))
    return fail(GSHT_ERR_UNSUPPORTED, "the recurrence form was not built for this grid");
  if (precision == GSHT_BF16X3 && !(g->forms & GSHT_FORM_BF16X3))
    return fail(GSHT_ERR_UNSUPPORTED, "the BF16x3 table form was not built for this grid");
  if ((precision == GSHT_OZAKI || precision == GSHT_OZAKI4) && !(g->forms & GSHT_FORM_OZAKI))
    return fail(GSHT_ERR_UNSUPPORTED, "the Ozaki table form was not built for this grid");
  return GSHT_OK;
}

struct CallScope {
  gsht_grid* g;
  cudaStream_t s;
  std::lock_guard<std::mutex> lock;
  CallScope(gsht_grid* grid, cudaStream_t stream) : g(grid), s(stream), lock(grid->mu) {}
};

gsht_status run_transform(gsht_grid* g, int dir, int lmax, int n, int is_real,
                          int precision, int count, const void* in, void* out,
                          void* stream_ptr, int ntile = 128, PrivateWorkspace* pws = nullptr) {
  gsht_status st = validate(g, lmax, n, is_real, precision, count);
  if (st != GSHT_OK) return st;
  GSHT_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_ptr);
  CallScope scope(g, s);
  const Table* t = g->table(n);
  // FP64 through the l-recurrence when asked for, or when no table is stored.
  const bool rec = precision == GSHT_RECURRENCE || (precision == GSHT_FP64 && !t->t64);
  const long cs = coef_size(lmax, n, is_real);
  const long fs = (long)g->n_theta * g->n_phi;
  const size_t coefBytes = sizeof(double) * 2 * cs * (size_t)count;
  const size_t gridBytes = sizeof(double) * (is_real ? 1 : 2) * fs * (size_t)count;
  const size_t inBytes = dir == 0 ? gridBytes : coefBytes;
  const size_t outBytes = dir == 0 ? coefBytes : gridBytes;
  const PtrKind inKind = pointer_kind(in, g->device), outKind = pointer_kind(out, g->device);
  if (inKind == kOtherDevicePtr || outKind == kOtherDevicePtr)
    return fail(GSHT_ERR_BAD_ARG, "a buffer lives on another GPU than the grid (device %d)", g->device);
  const bool inDev = inKind == kDevicePtr, outDev = outKind == kDevicePtr;
  if ((inDev && !aligned16(in)) || (outDev && !aligned16(out)))
    return fail(GSHT_ERR_BAD_ARG, "device buffers must be 16-byte aligned");

  // Inside a stream capture (batch graphs) nothing may be allocated, the
  // calls are serial on one stream, and events recorded outside the capture
  // may not be waited on.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GSHT_CUDA(cudaStreamIsCapturing(s, &cap));
  const bool capturing = cap != cudaStreamCaptureStatusNone;

  // Host buffers: the fields move in chunks on two copy streams, so that the
  // upload of chunk i+1, the transform of chunk i and the download of chunk
  // i-1 overlap (PCIe carries both directions at once). At most kMaxChunks
  // chunks of at least kMinChunkBytes of transfers each.
  constexpr int kMaxChunks = 16;
  constexpr size_t kMinChunkBytes = size_t(64) << 20;
  const size_t inField = inBytes / count, outField = outBytes / count;
  int chunk = count;
  if ((!inDev || !outDev) && !capturing && lmax > 0 && count > 1) {
    const size_t moved = (inDev ? 0 : inBytes) + (outDev ? 0 : (dir == 0 ? 2 : 1) * outBytes);
    size_t nch = moved / kMinChunkBytes;
    if (nch > (size_t)kMaxChunks) nch = kMaxChunks;
    if (nch > (size_t)count) nch = count;
    if (nch > 1) chunk = (int)((count + nch - 1) / nch);
  }
  const int nChunks = (count + chunk - 1) / chunk;

  // Workspace: [spec][operand][in staging][out staging], 256-byte aligned;
  // spec and operand hold one chunk, the staging areas all fields.
  const size_t specBytes = lmax > 0 ? sizeof(double) * 2 * spec_elems(g, lmax, is_real, chunk) : 0;
  size_t opBytes = 0;
  if (lmax > 0) {
    if (precision == GSHT_BF16X3)
      opBytes = bf16_operand_bytes(g, lmax, is_real, chunk, dir);
    else if (precision == GSHT_OZAKI || precision == GSHT_OZAKI4)
      opBytes = oz_operand_bytes(g, lmax, is_real, chunk, dir, precision == GSHT_OZAKI4 ? 4 : 7);
    else if (dir == 1) {
      size_t elems = 0;
      st = fp64_operand_elems(g, t, lmax, is_real, chunk, &elems);
      if (st != GSHT_OK) return st;
      opBytes = sizeof(double) * 2 * elems;
    }
    else if (rec)
      opBytes = rec_forward_bytes(g, t, is_real, chunk);
  }
  size_t off = 0;
  auto carve = [&](size_t b) { size_t o = off; off += round_up(b, 256); return o; };
  const size_t oSpec = carve(specBytes), oOp = carve(opBytes);
  const size_t oIn = carve(inDev ? 0 : inBytes), oOut = carve(outDev ? 0 : outBytes);
  const bool priv = pws != nullptr;
  if (priv && pws->need) {  // size query only
    *pws->need = off > 0 ? off : 256;
    return GSHT_OK;
  }
  char* ws = nullptr;
  if (priv) {
    if (!pws->ptr || pws->bytes < off)
      return fail(GSHT_ERR_BAD_ARG, "private workspace of %zu bytes, %zu needed", pws->bytes, off);
    ws = static_cast<char*>(pws->ptr);
  } else {
    if (capturing && g->ws_bytes < (off > 0 ? off : 256))
      return fail(GSHT_ERR_UNSUPPORTED, "workspace must be sized by an uncaptured call first");
    st = ensure_workspace(g, off > 0 ? off : 256);
    if (st != GSHT_OK) return st;
    ws = static_cast<char*>(g->ws);
    // Calls on other streams may still use the workspace: order after them.
    if (g->ws_done && !capturing) GSHT_CUDA(cudaStreamWaitEvent(s, g->ws_done, 0));
  }

  const double* dIn = inDev ? static_cast<const double*>(in) : reinterpret_cast<double*>(ws + oIn);
  double* dOut = outDev ? static_cast<double*>(out) : reinterpret_cast<double*>(ws + oOut);

  // The transform of c fields between device buffers, on stream s.
  auto compute = [&](int c, const double* dI, double* dO) -> gsht_status {
    if (lmax == 0) {
      k_lmax0<<<(c + 127) / 128, 128, 0, s>>>(dir, is_real, c, fs, dI, dO);
      GSHT_LAUNCH_CHECK("k_lmax0");
      return GSHT_OK;
    }
    double* spec = reinterpret_cast<double*>(ws + oSpec);
    // The BF16x3 form (~1e-6) keeps its spectra in FP32 where the three-pass
    // ring FFTs run: half the bytes through the FFT, the Legendre epilogue
    // and the operand preparation, at ~3e-8 of rounding.
    const bool spec32 = precision == GSHT_BF16X3 && fft_spec32_supported(g, is_real);
    gsht_status r;
    if (dir == 0) {
      {
        StageTimer tm(GSHT_STAGE_FFT_FORWARD, s);
        r = spec32 ? fft_forward32(g, lmax, is_real, c, dI, reinterpret_cast<float*>(spec), s)
                   : fft_forward(g, lmax, is_real, c, dI, spec, s);
      }
      if (r != GSHT_OK) return r;
      if (precision == GSHT_BF16X3)
        return legendre_forward_bf16(g, t, lmax, is_real, c, spec, ws + oOp, dO, ntile, s, spec32);
      if (precision == GSHT_OZAKI || precision == GSHT_OZAKI4)
        return legendre_forward_oz(g, t, lmax, is_real, c, spec, ws + oOp, dO, s,
                                   precision == GSHT_OZAKI4 ? 4 : 7);
      if (rec) return legendre_forward_rec(g, t, lmax, is_real, c, spec, ws + oOp, dO, s);
      StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
      return legendre_forward_fp64(g, t, lmax, is_real, c, spec, dO, s);
    }
    if (precision == GSHT_BF16X3)
      r = legendre_inverse_bf16(g, t, lmax, is_real, c, dI, ws + oOp, spec, ntile, s, spec32);
    else if (precision == GSHT_OZAKI || precision == GSHT_OZAKI4)
      r = legendre_inverse_oz(g, t, lmax, is_real, c, dI, ws + oOp, spec, s,
                              precision == GSHT_OZAKI4 ? 4 : 7);
    else if (rec)
      r = legendre_inverse_rec(g, t, lmax, is_real, c, dI, reinterpret_cast<double*>(ws + oOp),
                               spec, s);
    else
      r = legendre_inverse_fp64(g, t, lmax, is_real, c, dI, reinterpret_cast<double*>(ws + oOp),
                                spec, s);
    if (r != GSHT_OK) return r;
    StageTimer tm(GSHT_STAGE_FFT_INVERSE, s);
    return spec32 ? fft_inverse32(g, lmax, is_real, c, reinterpret_cast<const float*>(spec), dO, s)
                  : fft_inverse(g, lmax, is_real, c, spec, dO, s);
  };

  if (nChunks == 1) {
    if (!inDev) GSHT_CUDA(cudaMemcpyAsync(const_cast<double*>(dIn), in, inBytes, cudaMemcpyHostToDevice, s));
    // The forward accumulates into its output, so host outputs are uploaded
    // first; the inverse leaves grid points untouched only for lmax == 0.
    if (!outDev && (dir == 0 || lmax == 0))
      GSHT_CUDA(cudaMemcpyAsync(dOut, out, outBytes, cudaMemcpyHostToDevice, s));
    st = compute(count, dIn, dOut);
    if (st != GSHT_OK) return st;
    if (!outDev) GSHT_CUDA(cudaMemcpyAsync(out, dOut, outBytes, cudaMemcpyDeviceToHost, s));
  } else {
    st = ensure_copy_streams(g, 2 * nChunks + 2);
    if (st != GSHT_OK) return st;
    cudaEvent_t* ev = g->xfer_ev.data();
    // Uploads start after the work already queued on s (which may produce
    // the host input) and after the workspace's previous users.
    GSHT_CUDA(cudaEventRecord(ev[0], s));
    GSHT_CUDA(cudaStreamWaitEvent(g->h2d, ev[0], 0));
    GSHT_CUDA(cudaStreamWaitEvent(g->d2h, ev[0], 0));
    for (int i = 0; i < nChunks && st == GSHT_OK; i++) {
      const int f0 = i * chunk, c = count - f0 < chunk ? count - f0 : chunk;
      const size_t inOff = inField * f0, outOff = outField * f0;
      const double* dI = reinterpret_cast<const double*>(reinterpret_cast<const char*>(dIn) + inOff);
      double* dO = reinterpret_cast<double*>(reinterpret_cast<char*>(dOut) + outOff);
      if (!inDev)
        GSHT_CUDA(cudaMemcpyAsync(const_cast<double*>(dI), static_cast<const char*>(in) + inOff,
                                  inField * c, cudaMemcpyHostToDevice, g->h2d));
      if (!outDev && dir == 0)
        GSHT_CUDA(cudaMemcpyAsync(dO, static_cast<const char*>(out) + outOff, outField * c,
                                  cudaMemcpyHostToDevice, g->h2d));
      GSHT_CUDA(cudaEventRecord(ev[1 + 2 * i], g->h2d));
      GSHT_CUDA(cudaStreamWaitEvent(s, ev[1 + 2 * i], 0));
      st = compute(c, dI, dO);
      if (st == GSHT_OK && !outDev) {
        GSHT_CUDA(cudaEventRecord(ev[2 + 2 * i], s));
        GSHT_CUDA(cudaStreamWaitEvent(g->d2h, ev[2 + 2 * i], 0));
        GSHT_CUDA(cudaMemcpyAsync(static_cast<char*>(out) + outOff, dO, outField * c,
                                  cudaMemcpyDeviceToHost, g->d2h));
      }
    }
    // s ends after the copies, also when a chunk failed to launch.
    GSHT_CUDA(cudaEventRecord(ev[2 * nChunks + 1], g->d2h));
    GSHT_CUDA(cudaStreamWaitEvent(s, ev[2 * nChunks + 1], 0));
    GSHT_CUDA(cudaEventRecord(ev[2 * nChunks], g->h2d));
    GSHT_CUDA(cudaStreamWaitEvent(s, ev[2 * nChunks], 0));
    if (st != GSHT_OK) {
      cudaStreamSynchronize(s);
      return st;
    }
  }
  if (!capturing && !priv) {
    if (!g->ws_done) GSHT_CUDA(cudaEventCreateWithFlags(&g->ws_done, cudaEventDisableTiming));
    GSHT_CUDA(cudaEventRecord(g->ws_done, s));
  }
  if (!inDev || !outDev) {
    GSHT_CUDA(cudaStreamSynchronize(s));
    int err = 0;
    GSHT_CUDA(cudaMemcpy(&err, g->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
      cudaMemset(g->d_err, 0, sizeof(int));
      return fail(GSHT_ERR_TIMEOUT, "a bounded device wait expired (code %d)", err);
    }
  }
  return GSHT_OK;
}

}  // namespace

gsht_status transform(gsht_grid* g, int dir, int lmax, int n, int is_real, int precision,
                      int count, const void* in, void* out, cudaStream_t s, int ntile,
                      PrivateWorkspace* pws) {
  return run_transform(g, dir, lmax, n, is_real, precision, count, in, out, s, ntile, pws);
}

}  // namespace gsht

using namespace gsht;

extern "C" {

gsht_status gsht_grid_create(int lmax, int nmax, int mrange, int nrange,
                             unsigned forms, gsht_grid** out) {
  if (!out) return fail(GSHT_ERR_BAD_ARG, "output handle pointer is NULL");
  *out = nullptr;
  if (lmax < 1) return fail(GSHT_ERR_BAD_ARG, "lmax must be >= 1 (got %d)", lmax);
  if (nmax < 0 || nmax > lmax)
    return fail(GSHT_ERR_BAD_ARG, "nmax %d outside [0, lmax]", nmax);
  if (mrange != GSHT_RANGE_ALL && mrange != GSHT_RANGE_NONNEGATIVE)
    return fail(GSHT_ERR_BAD_ARG, "mrange must be All or NonNegative");
  if (nrange < GSHT_RANGE_ALL || nrange > GSHT_RANGE_SINGLE)
    return fail(GSHT_ERR_BAD_ARG, "bad nrange %d", nrange);
  if (forms & ~15u) return fail(GSHT_ERR_BAD_ARG, "unknown form bits 0x%x", forms);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GSHT_ERR_NO_DEVICE, "no CUDA device visible");
  }
  gsht_grid* g = new (std::nothrow) gsht_grid();
  if (!g) return fail(GSHT_ERR_OOM, "host allocation failed");
  GSHT_CUDA(cudaGetDevice(&g->device));
  g->L = lmax;
  g->nmax = nmax;
  g->mrange = mrange;
  g->nrange = nrange;
  g->forms = forms == GSHT_FORM_RECURRENCE ? forms : forms | GSHT_FORM_FP64;
  g->min_n = nrange == GSHT_RANGE_ALL ? -nmax : (nrange == GSHT_RANGE_NONNEGATIVE ? 0 : nmax);
  g->n_theta = lmax + 1;
  g->n_phi = 2 * lmax;
  g->theta_pad = (int)round_up(g->n_theta, kThetaPad);
  gsht_status st = build_nodes(g);
  if (st == GSHT_OK && (dev_malloc(&g->d_err, sizeof(int)) != cudaSuccess ||
                        cudaMemset(g->d_err, 0, sizeof(int)) != cudaSuccess)) {
    cudaGetLastError();
    st = fail(GSHT_ERR_OOM, "error word allocation failed");
  }
  if (st == GSHT_OK) {
    // Twiddles exp(-2 pi i t / nPhi), t < nPhi, rounded from long double.
    std::vector<double> tw(2 * (size_t)g->n_phi);
    const long double twoPi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < g->n_phi; t++) {
      const long double a = twoPi * t / g->n_phi;
      tw[2 * t] = (double)cosl(a);
      tw[2 * t + 1] = (double)-sinl(a);
    }
    std::vector<float> tw32(tw.begin(), tw.end());
    if (dev_malloc(&g->d_twiddle, sizeof(double) * tw.size()) != cudaSuccess ||
        cudaMemcpy(g->d_twiddle, tw.data(), sizeof(double) * tw.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        dev_malloc(&g->d_twiddle32, sizeof(float) * tw32.size()) != cudaSuccess ||
        cudaMemcpy(g->d_twiddle32, tw32.data(), sizeof(float) * tw32.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      st = fail(GSHT_ERR_OOM, "twiddle table allocation failed");
    }
  }
  if (st == GSHT_OK) {
    g->tables.resize(g->nmax - g->min_n + 1);
    cudaStream_t s = nullptr;
    for (int n = g->min_n; n <= g->nmax && st == GSHT_OK; n++) {
      Table* t = &g->tables[n - g->min_n];
      t->n = n;
      if (g->forms & GSHT_FORM_FP64) {
        st = build_table(g, t, s);
        if (st == GSHT_OK) st = build_forms(g, t, s);
      }
      if (st == GSHT_OK && (g->forms & GSHT_FORM_RECURRENCE)) st = build_recurrence(g, t, s);
    }
  }
  if (st != GSHT_OK) {
    gsht_grid_destroy(g);
    return st;
  }
  *out = g;
  return GSHT_OK;
}

gsht_status gsht_grid_destroy(gsht_grid* g) {
  if (!g) return GSHT_OK;
  cudaSetDevice(g->device);
  cudaDeviceSynchronize();
  for (auto& t : g->tables) free_table(&t);
  free_layouts(g);
  dev_free(g->d_theta);
  dev_free(g->d_weight);
  dev_free(g->d_twiddle);
  dev_free(g->d_twiddle32);
  dev_free(g->d_err);
  dev_free(g->ws);
  if (g->ws_done) cudaEventDestroy(g->ws_done);
  for (cudaEvent_t e : g->xfer_ev) cudaEventDestroy(e);
  if (g->h2d) cudaStreamDestroy(g->h2d);
  if (g->d2h) cudaStreamDestroy(g->d2h);
  delete g;
  return GSHT_OK;
}

gsht_status gsht_grid_shape(const gsht_grid* g, int* lmax, int* nmax,
                            int* min_n, int* n_theta, int* n_phi) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (lmax) *lmax = g->L;
  if (nmax) *nmax = g->nmax;
  if (min_n) *min_n = g->min_n;
  if (n_theta) *n_theta = g->n_theta;
  if (n_phi) *n_phi = g->n_phi;
  return GSHT_OK;
}

gsht_status gsht_grid_nodes(const gsht_grid* g, double* colatitudes,
                            double* weights) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (colatitudes) memcpy(colatitudes, g->h_theta.data(), sizeof(double) * g->n_theta);
  if (weights) memcpy(weights, g->h_weight.data(), sizeof(double) * g->n_theta);
  return GSHT_OK;
}

gsht_status gsht_wigner_block(const gsht_grid* g, int n, int itheta,
                              double* out, long* count) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (n < g->min_n || n > g->nmax) return fail(GSHT_ERR_BAD_ARG, "upper index %d not in the grid", n);
  if (itheta < 0 || itheta >= g->n_theta) return fail(GSHT_ERR_BAD_ARG, "colatitude index %d out of range", itheta);
  const int L = g->L, na = n < 0 ? -n : n;
  const bool all = g->mrange == GSHT_RANGE_ALL;
  const long total = all ? (long)(L + 1) * (L + 1) - (long)n * n
                         : (long)(L + 1) * (L + 2) / 2 - (long)na * (na + 1) / 2;
  if (count) *count = total;
  if (!out) return GSHT_OK;
  const Table* t = g->table(n);
  if (!t->t64)
    return fail(GSHT_ERR_UNSUPPORTED, "the grid stores no table (recurrence form); use gsht_wigner_compute");
  GSHT_CUDA(cudaSetDevice(g->device));
  std::vector<double> col(t->rows), mir(t->rows);
  const size_t pitch = sizeof(double) * g->theta_pad;
  GSHT_CUDA(cudaMemcpy2D(col.data(), sizeof(double), t->t64 + itheta, pitch,
                         sizeof(double), t->rows, cudaMemcpyDeviceToHost));
  GSHT_CUDA(cudaMemcpy2D(mir.data(), sizeof(double), t->t64 + (g->n_theta - 1 - itheta),
                         pitch, sizeof(double), t->rows, cudaMemcpyDeviceToHost));
  long i = 0;
  for (int l = na; l <= L; l++) {
    for (int m = all ? -l : 0; m <= l; m++) {
      const int am = m < 0 ? -m : m;
      const int l0 = am > na ? am : na;
      const long long row = t->row_off[am] + (l - l0);
      // d^l_{-m,n}(theta_j) = (-1)^{l+n} d^l_{mn}(theta_{nTheta-1-j})
      out[i++] = m >= 0 ? col[row] : (((l + n) & 1) ? -mir[row] : mir[row]);
    }
  }
  return GSHT_OK;
}

gsht_status gsht_wigner_compute(int lmax, int mmax, int nmax, int mrange, int nrange,
                                int norm, int row_major, const double* theta, int ntheta,
                                double* out, long* count) {
  if (lmax < 0 || mmax < 0 || nmax < 0 || nmax > lmax)
    return fail(GSHT_ERR_BAD_ARG, "need 0 <= nmax <= lmax and mmax >= 0");
  if (mrange != GSHT_RANGE_ALL && mrange != GSHT_RANGE_NONNEGATIVE)
    return fail(GSHT_ERR_BAD_ARG, "mrange must be All or NonNegative");
  if (nrange < GSHT_RANGE_ALL || nrange > GSHT_RANGE_SINGLE)
    return fail(GSHT_ERR_BAD_ARG, "bad nrange %d", nrange);
  if (norm != 0 && norm != 1) return fail(GSHT_ERR_BAD_ARG, "norm must be 0 (Ortho) or 1 (FourPi)");
  if (ntheta < 1 || (!theta && out)) return fail(GSHT_ERR_BAD_ARG, "need at least one angle");
  if (out) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return fail(GSHT_ERR_NO_DEVICE, "no CUDA device visible");
    }
  }
  return wigner_compute(lmax, mmax, nmax, mrange, nrange, norm, row_major, theta, ntheta, out,
                        count);
}

long gsht_coefficient_size(int lmax, int n, int is_real) {
  if (lmax < 0 || (n < 0 ? -n : n) > lmax) return -1;
  return coef_size(lmax, n, is_real);
}

gsht_status gsht_forward(const gsht_grid* g, int lmax, int n, int is_real,
                         int precision, const void* in, void* out,
                         void* stream) {
  return run_transform(const_cast<gsht_grid*>(g), 0, lmax, n, is_real,
                       precision, 1, in, out, stream);
}

gsht_status gsht_inverse(const gsht_grid* g, int lmax, int n, int is_real,
                         int precision, const void* in, void* out,
                         void* stream) {
  return run_transform(const_cast<gsht_grid*>(g), 1, lmax, n, is_real,
                       precision, 1, in, out, stream);
}

// ---- Stages of a transform sharded over ranks (include/gsht.h) ----

gsht_status gsht_spectra_layout(const gsht_grid* g, int lmax, int is_real, int count,
                                long* elems, int* pitch) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  if (lmax < 1 || lmax > g->L) return fail(GSHT_ERR_BAD_ARG, "lmax %d outside [1, %d]", lmax, g->L);
  if (count < 1) return fail(GSHT_ERR_BAD_ARG, "count %d < 1", count);
  if (elems) *elems = (long)spec_elems(g, lmax, is_real, count);
  if (pitch) *pitch = g->theta_pad;
  return GSHT_OK;
}

namespace {

// Common checks of the stage entry points: FP64 table form, device buffers
// of the grid's device, a range inside [0, limit).
gsht_status stage_check(const gsht_grid* g, int lmax, int n, int is_real, int count, int begin,
                        int end, int limit, const void* a, const void* b) {
  gsht_status st = validate(g, lmax, n, is_real, GSHT_FP64, count);
  if (st != GSHT_OK) return st;
  if (lmax < 1) return fail(GSHT_ERR_BAD_ARG, "the stages need lmax >= 1");
  if (begin < 0 || end > limit || begin > end)
    return fail(GSHT_ERR_BAD_ARG, "range [%d, %d) outside [0, %d)", begin, end, limit);
  if (!a || !b) return fail(GSHT_ERR_BAD_ARG, "NULL buffer");
  if (pointer_kind(a, g->device) != kDevicePtr || pointer_kind(b, g->device) != kDevicePtr)
    return fail(GSHT_ERR_BAD_ARG, "the stages take device buffers of the grid's device (%d)",
                g->device);
  if (!aligned16(a) || !aligned16(b))
    return fail(GSHT_ERR_BAD_ARG, "device buffers must be 16-byte aligned");
  return GSHT_OK;
}

}  // namespace

gsht_status gsht_forward_rings(const gsht_grid* g, int lmax, int is_real, int count,
                               int ring_begin, int ring_end, const void* grid_values,
                               void* spectra, void* stream) {
  const int n = g ? g->min_n : 0;
  gsht_status st = stage_check(g, lmax, n, is_real, count, ring_begin, ring_end,
                               g ? g->n_theta : 0, grid_values, spectra);
  if (st != GSHT_OK) return st;
  GSHT_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  StageTimer tm(GSHT_STAGE_FFT_FORWARD, s);
  return fft_forward(g, lmax, is_real, count, static_cast<const double*>(grid_values),
                     static_cast<double*>(spectra), s, RingRange{ring_begin, ring_end});
}

gsht_status gsht_inverse_rings(const gsht_grid* g, int lmax, int is_real, int count,
                               int ring_begin, int ring_end, const void* spectra,
                               void* grid_values, void* stream) {
  const int n = g ? g->min_n : 0;
  gsht_status st = stage_check(g, lmax, n, is_real, count, ring_begin, ring_end,
                               g ? g->n_theta : 0, spectra, grid_values);
  if (st != GSHT_OK) return st;
  GSHT_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  StageTimer tm(GSHT_STAGE_FFT_INVERSE, s);
  return fft_inverse(g, lmax, is_real, count, static_cast<const double*>(spectra),
                     static_cast<double*>(grid_values), s, RingRange{ring_begin, ring_end});
}

gsht_status gsht_forward_orders(const gsht_grid* g, int lmax, int n, int is_real, int count,
                                int m_begin, int m_end, const void* spectra, void* coef_out,
                                void* stream) {
  gsht_status st = stage_check(g, lmax, n, is_real, count, m_begin, m_end, lmax + 1, spectra,
                               coef_out);
  if (st != GSHT_OK) return st;
  const Table* t = g->table(n);
  if (!t->t64) return fail(GSHT_ERR_UNSUPPORTED, "the order stages need the stored FP64 table");
  GSHT_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
  return legendre_forward_fp64(g, t, lmax, is_real, count, static_cast<const double*>(spectra),
                               static_cast<double*>(coef_out), s, m_begin, m_end);
}

gsht_status gsht_inverse_orders(const gsht_grid* g, int lmax, int n, int is_real, int count,
                                int m_begin, int m_end, const void* coef_in, void* spectra,
                                void* stream) {
  gsht_status st = stage_check(g, lmax, n, is_real, count, m_begin, m_end, lmax + 1, coef_in,
                               spectra);
  if (st != GSHT_OK) return st;
  const Table* t = g->table(n);
  if (!t->t64) return fail(GSHT_ERR_UNSUPPORTED, "the order stages need the stored FP64 table");
  GSHT_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  gsht_grid* gm = const_cast<gsht_grid*>(g);
  CallScope scope(gm, s);
  size_t elems = 0;
  st = fp64_operand_elems(g, t, lmax, is_real, count, &elems);
  if (st != GSHT_OK) return st;
  st = ensure_workspace(gm, sizeof(double) * 2 * elems + 256);
  if (st != GSHT_OK) return st;
  if (g->ws_done) GSHT_CUDA(cudaStreamWaitEvent(s, g->ws_done, 0));
  st = legendre_inverse_fp64(g, t, lmax, is_real, count, static_cast<const double*>(coef_in),
                             static_cast<double*>(g->ws), static_cast<double*>(spectra), s,
                             m_begin, m_end);
  if (st != GSHT_OK) return st;
  if (!gm->ws_done) GSHT_CUDA(cudaEventCreateWithFlags(&gm->ws_done, cudaEventDisableTiming));
  GSHT_CUDA(cudaEventRecord(gm->ws_done, s));
  return GSHT_OK;
}

gsht_status gsht_forward_batch(const gsht_grid* g, int lmax, int n,
                               int is_real, int precision, int count,
                               const void* in, void* out, void* stream) {
  return run_transform(const_cast<gsht_grid*>(g), 0, lmax, n, is_real,
                       precision, count, in, out, stream);
}

gsht_status gsht_inverse_batch(const gsht_grid* g, int lmax, int n,
                               int is_real, int precision, int count,
                               const void* in, void* out, void* stream) {
  return run_transform(const_cast<gsht_grid*>(g), 1, lmax, n, is_real,
                       precision, count, in, out, stream);
}

gsht_status gsht_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_prof.clear();
  for (int i = 0; i < GSHT_STAGE_COUNT; i++) {
    g_prof_ms[i] = 0.0;
    g_prof_launches[i] = 0;
  }
  g_prof_on = on != 0;
  return GSHT_OK;
}

gsht_status gsht_profile_read(double* ms, long* launches, int nstages) {
  if (nstages < 0) return fail(GSHT_ERR_BAD_ARG, "negative stage count");
  for (int i = 0; i < nstages; i++) {
    if (ms) ms[i] = 0.0;
    if (launches) launches[i] = 0;
  }
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (int i = 0; i < nstages && i < GSHT_STAGE_COUNT; i++) {
    if (ms) ms[i] = g_prof_ms[i];
    if (launches) launches[i] = g_prof_launches[i];
  }
  for (auto& r : g_prof) {
    GSHT_CUDA(cudaEventSynchronize(r.b));
    float t = 0.f;
    GSHT_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.stage < nstages) {
      if (ms) ms[r.stage] += t;
      if (launches) launches[r.stage] += (long)r.launches;
    }
  }
  return GSHT_OK;
}

gsht_status gsht_device_status(const gsht_grid* g) {
  if (!g) return fail(GSHT_ERR_BAD_ARG, "grid is NULL");
  GSHT_CUDA(cudaSetDevice(g->device));
  GSHT_CUDA(cudaDeviceSynchronize());
  int err = 0;
  GSHT_CUDA(cudaMemcpy(&err, g->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    GSHT_CUDA(cudaMemset(g->d_err, 0, sizeof(int)));
    return fail(GSHT_ERR_TIMEOUT, "a bounded device wait expired (code %d)", err);
  }
  return GSHT_OK;
}

const char* gsht_last_error(void) { return t_error; }

unsigned long long gsht_launch_count(void) { return g_launches.load(); }

gsht_status gsht_set_allocator(gsht_alloc_fn alloc, gsht_free_fn free_fn, void* ctx) {
  if ((alloc == nullptr) != (free_fn == nullptr))
    return fail(GSHT_ERR_BAD_ARG, "give both an allocation and a release function, or neither");
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  g_hook.alloc = alloc;
  g_hook.free = free_fn;
  g_hook.ctx = ctx;
  return GSHT_OK;
}

gsht_status gsht_alloc_stats(unsigned long long* allocations, unsigned long long* releases,
                             size_t* live_bytes) {
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  if (allocations) *allocations = g_alloc_calls;
  if (releases) *releases = g_free_calls;
  if (live_bytes) *live_bytes = g_live_bytes;
  return GSHT_OK;
}

}  // extern "C"
