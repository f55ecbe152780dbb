// Internal declarations shared by the CUDA translation units of
// libgsht_cuda.so. Nothing here is part of the C ABI (include/gsht.h).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "gsht.h"

namespace gsht {

// ---------------------------------------------------------------------------
// Errors and launch accounting
// ---------------------------------------------------------------------------
gsht_status fail(gsht_status s, const char* fmt, ...);
gsht_status cuda_fail(cudaError_t e, const char* what);
extern std::atomic<unsigned long long> g_launches;
// Launches made by this thread (stage launch counts: exact for the calls of
// one thread, whichever other threads launch meanwhile).
extern thread_local unsigned long long t_launches;

// Per-role trace of the tensor-core Legendre kernels (diagnostics.cu): when
// set, launches take the traced kernel copies, whose counters trace_slots
// (form 0 BF16x3, 1 Ozaki; dir 0 inverse, 1 forward) clears on stream s and
// returns (NULL on failure).
extern std::atomic<int> g_tc_trace;
unsigned long long* trace_slots(int form, int dir, cudaStream_t s);

#define GSHT_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return gsht::cuda_fail(e_, #call); \
  } while (0)

// Marks one kernel launch and checks the launch status.
#define GSHT_LAUNCH_CHECK(name)                                    \
  do {                                                             \
    gsht::g_launches.fetch_add(1, std::memory_order_relaxed);      \
    gsht::t_launches++;                                            \
    cudaError_t e_ = cudaGetLastError();                           \
    if (e_ != cudaSuccess) return gsht::cuda_fail(e_, name);       \
  } while (0)

inline long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// Where a caller's buffer lives, seen from `device`: host memory, memory the
// device uses in place (its own, or managed), or another GPU's memory
// (rejected by the entry points: the kernels would read it over a peer
// mapping that need not exist).
enum PtrKind { kHostPtr = 0, kDevicePtr = 1, kOtherDevicePtr = 2 };
PtrKind pointer_kind(const void* p, int device);
// Device buffers are read and written as 16-byte complex elements (and by
// bulk copies, which need 16-byte addresses): misaligned ones are refused.
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Every device allocation of the library goes through these: the hook of
// gsht_set_allocator when one is set, else cudaMalloc / cudaFree. A pointer
// is released by the allocator that made it, even if the hook has changed
// since. A failed hook allocation reads as cudaErrorMemoryAllocation.
cudaError_t dev_malloc_bytes(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}
void dev_free(void* p);

// Device scratch of one call, released (dev_free) when it leaves scope, so
// that every early return of the call gives it back.
template <typename T>
struct ScopedDev {
  T* p = nullptr;
  ScopedDev() = default;
  ScopedDev(const ScopedDev&) = delete;
  ScopedDev& operator=(const ScopedDev&) = delete;
  ~ScopedDev() { dev_free(p); }
};

// Brackets one stage of a transform call with CUDA events while stage
// profiling is enabled (gsht_profile_enable); otherwise does nothing.
class StageTimer {
 public:
  StageTimer(int stage, cudaStream_t s);
  ~StageTimer();
  StageTimer(const StageTimer&) = delete;
  StageTimer& operator=(const StageTimer&) = delete;

 private:
  int stage_;
  cudaStream_t s_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
  unsigned long long launches0_ = 0;
};

// ---------------------------------------------------------------------------
// Layout constants
// ---------------------------------------------------------------------------
// Row pitch (in elements) of every table and spectral buffer along the
// colatitude axis: nTheta rounded up to kThetaPad.
constexpr int kThetaPad = 16;
// Padding of the degree axis of field-side operands (K of the inverse GEMM).
constexpr int kDegreePadFp64 = 16;
constexpr int kDegreePadTc = 128;
// Ozaki slice count of the table (7 bits per slice).
constexpr int kTableSlices = 7;
// Extra zero rows allocated after every table so that tile over-reads stay
// inside the allocation.
constexpr int kTablePadRows = 256;

// Per upper index n: Wigner table for orders m = 0..L, degrees
// l = l0(m)..L with l0(m) = max(m, |n|), colatitudes j = 0..nThetaPad-1.
// Row (m, l) lives at row_off[m] + (l - l0(m)); element (row, j) at
// row * thetaPad + j. Negative orders follow from
// d^l_{-m,n}(pi - theta) = (-1)^{l+n} d^l_{mn}(theta) on the symmetric
// Gauss-Legendre colatitudes.
struct Table {
  int n = 0;
  long long rows = 0;                 // sum over m of K_m = L - l0(m) + 1
  std::vector<long long> row_off;     // host, size L+2
  long long* d_row_off = nullptr;     // device copy
  double* t64 = nullptr;              // FP64 values
  __nv_bfloat16* tbf = nullptr;       // 3 planes (hi, mid, lo), same layout
  int8_t* ti8 = nullptr;              // kTableSlices planes, same layout
  int* i8_exp = nullptr;              // (L+1) x thetaPad column exponents
  // FP64 values of the last colatitude column (theta_{nTheta-1}), one per
  // row, when the Ozaki form is stored and nTheta = 128 k + 1: that
  // colatitude would fill a 128-row inverse tile of its own, so the operand
  // preparation contracts it instead (legendre_oz.cu).
  double* tail64 = nullptr;
  // Recurrence form (no stored values): start values d^{l0(m)}_{mn}(theta_j)
  // = rec_f * 2^rec_e, [m][thetaPad], and per row the coefficients (a', b')
  // of the rescaled recurrence e_k = (a' cos(theta) - b') e_{k-1} - e_{k-2}
  // and the factor rec_sc with d_k * norm_k = rec_sc * e_k (grid.cu).
  double* rec_f = nullptr;
  int* rec_e = nullptr;
  double2* rec_ab = nullptr;
  double* rec_sc = nullptr;
};

// Per-order layout of field-side operand rows for one (lmax, |n|, rows,
// padding): order m owns `rows` rows of pitch[m] = round_up(lmax - l0(m) + 1,
// pad) elements starting at off[m]. Built once per key and cached on the grid.
struct OperandLayout {
  int lmax = 0, na = 0, rows = 0, pad = 0;
  std::vector<long long> off;  // host, size lmax + 2 (off[lmax+1] = total)
  std::vector<int> pitch;      // host, size lmax + 1
  long long* d_off = nullptr;
  int* d_pitch = nullptr;
  long long total = 0;
  int pitch_max = 0;
};

// Work list of a persistent tensor-core launch: tiles (m, mtile, ntile, nk)
// in order of decreasing m-block work, cached on the grid per key.
struct TileList {
  int dir = 0, lmax = 0, na = 0, rows = 0, ntile = 0, kstep = 0, tail = 0;
  int4* d_tiles = nullptr;
  int count = 0;
};

}  // namespace gsht

// The opaque handle of the C ABI.
struct gsht_grid {
  int L = 0;           // grid degree (MaxDegree)
  int nmax = 0;        // MaxUpperIndex
  int min_n = 0;       // MinUpperIndex
  int mrange = 0;      // GSHT_RANGE_ALL / NONNEGATIVE
  int nrange = 0;
  unsigned forms = 0;  // GSHT_FORM_* built
  int device = 0;
  int n_theta = 0, n_phi = 0, theta_pad = 0;

  std::vector<double> h_theta, h_weight;  // host copies of the nodes
  double* d_theta = nullptr;              // device nodes
  double* d_weight = nullptr;
  double* d_twiddle = nullptr;            // FFT twiddles exp(-2 pi i t / nPhi), t < nPhi
  float* d_twiddle32 = nullptr;           // the same rounded to FP32 (FP32-spectrum FFTs)
  int* d_err = nullptr;                   // device error word (bounded-wait timeouts)

  std::vector<gsht::Table> tables;        // index n - min_n

  // Workspace shared by the transform calls on this grid.
  std::mutex mu;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  cudaEvent_t ws_done = nullptr;  // recorded after the last call's kernels
  // Copy streams and events of the chunked host-buffer pipeline (guarded by mu).
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> xfer_ev;
  // Cached operand layouts (guarded by mu).
  mutable std::vector<gsht::OperandLayout*> layouts;
  mutable std::vector<gsht::TileList*> tile_lists;

  const gsht::Table* table(int n) const {
    if (n < min_n || n > nmax) return nullptr;
    return &tables[n - min_n];
  }
};

namespace gsht {

// Table build (grid.cu).
gsht_status build_nodes(gsht_grid* g);
gsht_status build_table(gsht_grid* g, Table* t, cudaStream_t s);
gsht_status build_forms(gsht_grid* g, Table* t, cudaStream_t s);
gsht_status build_recurrence(gsht_grid* g, Table* t, cudaStream_t s);
void free_table(Table* t);
gsht_status wigner_compute(int lmax, int mmax, int nmax, int mrange, int nrange, int norm,
                           int row_major, const double* theta, int ntheta, double* out,
                           long* count);

// Colatitudes [jBegin, jEnd) a ring-FFT launch transforms: the whole grid,
// or one rank's slab of a transform sharded over colatitudes (rings outside
// the range are not written). jEnd < 0 stands for the whole grid. fields:
// when set (a device array), field f's grid is fields[f] rather than the
// f-th of the launch's contiguous grids (batch plans: the callers' buffers).
struct RingRange {
  int jBegin = 0, jEnd = -1;
  double* const* fields = nullptr;
  __host__ __device__ bool has(int j) const { return j >= jBegin && j < jEnd; }
  // Start of field f's grid, given the contiguous grids at base with
  // fieldDoubles doubles each.
  __host__ __device__ double* grid(double* base, int f, size_t fieldDoubles) const {
    return fields ? fields[f] : base + (size_t)f * fieldDoubles;
  }
  __host__ __device__ const double* grid(const double* base, int f, size_t fieldDoubles) const {
    return fields ? fields[f] : base + (size_t)f * fieldDoubles;
  }
};
inline RingRange resolve(RingRange r, int nTheta) {
  if (r.jEnd < 0 || r.jEnd > nTheta) r.jEnd = nTheta;
  if (r.jBegin < 0) r.jBegin = 0;
  return r;
}

// FFT stage (fft.cu). spec: spectral buffer [m][sgn][f][j] complex.
gsht_status fft_inverse(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* spec, double* out, cudaStream_t s, RingRange rr = {});
gsht_status fft_forward(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* in, double* spec, cudaStream_t s, RingRange rr = {});
// FP32 spectra (BF16x3 form): the -m rows are stored at their own
// colatitudes (no mirror). Ring lengths 256..4096 (powers of two) only.
bool fft_spec32_supported(const gsht_grid* g, int is_real);
gsht_status fft_inverse32(const gsht_grid* g, int lmax, int is_real, int count, const float* spec,
                          double* out, cudaStream_t s, double* const* fields = nullptr);
gsht_status fft_forward32(const gsht_grid* g, int lmax, int is_real, int count, const double* in,
                          float* spec, cudaStream_t s, double* const* fields = nullptr);

// Legendre stage, FP64 (legendre_fp64.cu).
gsht_status fp64_operand_elems(const gsht_grid* g, const Table* t, int lmax, int is_real,
                               int count, size_t* elems);
// [mBegin, mEnd): the orders contracted (a rank's share of a transform
// sharded over orders); mEnd < 0 stands for all orders 0..lmax.
gsht_status legendre_inverse_fp64(const gsht_grid* g, const Table* t, int lmax,
                                  int is_real, int count, const double* coef,
                                  double* operand, double* spec,
                                  cudaStream_t s, int mBegin = 0, int mEnd = -1);
// Packed coefficients -> FP64 operand rows op[m][q][k] (the inverse's A).
gsht_status prep_inverse_fp64(const gsht_grid* g, const Table* t, int lmax, int is_real,
                              int count, const double* coef, double* operand,
                              const OperandLayout** layout, cudaStream_t s, int mBegin = 0,
                              int mEnd = -1);
gsht_status legendre_forward_fp64(const gsht_grid* g, const Table* t, int lmax,
                                  int is_real, int count, const double* spec,
                                  double* coef, cudaStream_t s, int mBegin = 0, int mEnd = -1);
gsht_status legendre_inverse_fp64_layout(const gsht_grid* g, const Table* t, int lmax,
                                         int is_real, int count, const double* coef,
                                         const long long* dOff, const int* dPitch, int kpMax,
                                         double* operand, double* spec, cudaStream_t s);

// BF16x3 stages for batch plans (legendre_tc.cu): the operand preparation of
// each direction on its own, and one persistent Legendre launch over the
// tiles of several groups (each with its grid, table, operand rows and
// spectra; every group's tensor maps and arguments in device memory).
gsht_status bf16_prep_inverse(const gsht_grid* g, const Table* t, int lmax, int is_real,
                              int count, const double* coef, void* operand, cudaStream_t s,
                              const double* const* fieldPtrs = nullptr);
gsht_status bf16_prep_forward(const gsht_grid* g, int lmax, int is_real, int count,
                              const double* spec, void* operand, cudaStream_t s, bool spec32);
struct Bf16MultiGroup {
  const gsht_grid* g = nullptr;
  const Table* t = nullptr;
  int lmax = 0, isReal = 0, count = 0;
  void* operand = nullptr;   // prepared operand rows of the direction
  double* spec = nullptr;    // spectra (inverse output) / result rows (forward output)
  bool spec32 = false;       // inverse: FP32 spectra
};
struct Bf16Multi {
  void* d_groups = nullptr;  // per-group tensor maps and arguments
  void* d_tiles = nullptr;   // tiles (group << 16 | m, M tile, N tile, K blocks)
  int numTiles = 0, dir = 0, ntile = 0, bk = 0, device = 0;
  int* err = nullptr;        // device error word the launch reports through
};
gsht_status bf16_multi_build(int dir, const Bf16MultiGroup* groups, int ngroups, int ntile,
                             Bf16Multi* out);
gsht_status bf16_multi_launch(const Bf16Multi& multi, cudaStream_t s);
void bf16_multi_free(Bf16Multi* multi);

// Legendre stage, BF16x3 on tcgen05 (legendre_tc.cu). dir 0 = forward
// (operand rows over colatitudes), 1 = inverse (rows over degrees).
size_t bf16_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir);
// A workspace owned by the caller of transform() instead of the grid's (so
// that transforms on one grid can run concurrently on several streams). With
// `need` set, transform() only stores the bytes it would use there.
struct PrivateWorkspace {
  void* ptr = nullptr;
  size_t bytes = 0;
  size_t* need = nullptr;
};
// One batched transform (the body of gsht_forward_batch / gsht_inverse_batch)
// with an explicit BF16x3 tile width; dir 0 forward, 1 inverse.
gsht_status transform(gsht_grid* g, int dir, int lmax, int n, int is_real, int precision,
                      int count, const void* in, void* out, cudaStream_t s, int ntile,
                      PrivateWorkspace* pws = nullptr);
// spec32: the spectra are FP32 with unmirrored -m rows (fft_inverse32 /
// fft_forward32); the buffer is still sized for FP64 spectra.
gsht_status legendre_inverse_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, const double* coef, void* operand, double* spec,
                                  int ntile, cudaStream_t s, bool spec32 = false);
// The spectra buffer is reused for the kernel's result rows.
gsht_status legendre_forward_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, double* spec, void* operand, double* coef,
                                  int ntile, cudaStream_t s, bool spec32 = false);

// Legendre stage, Ozaki INT8 slices on tcgen05 (legendre_oz.cu). slices: 7
// (the FP64-class form) or 4 (the ~1e-7 form, first 4 table slices).
size_t oz_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir,
                        int slices = kTableSlices);
gsht_status legendre_inverse_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, const double* coef, void* operand, double* spec,
                                cudaStream_t s, int slices = kTableSlices);
// The spectra buffer is reused for the kernel's result rows.
gsht_status legendre_forward_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, double* spec, void* operand, double* coef,
                                cudaStream_t s, int slices = kTableSlices);
// Legendre stage, FP64 with the Wigner values generated by the l-recurrence
// inside the contraction (legendre_rec.cu); no stored table.
size_t rec_forward_bytes(const gsht_grid* g, const Table* t, int is_real, int count);
gsht_status legendre_inverse_rec(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                 int count, const double* coef, double* operand, double* spec,
                                 cudaStream_t s);
// spec is overwritten with the result rows; partial holds rec_forward_bytes.
gsht_status legendre_forward_rec(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                 int count, double* spec, void* partial, double* coef,
                                 cudaStream_t s);

// Adds order-major result rows R[m][q][l - l0] (pitch `pitch`; complex
// FP64, or FP32 with rows32) into the packed coefficients of `count` fields
// (forward accumulate semantics): coef + f * coefSize, or fieldPtrs[f] when
// fieldPtrs (a device array) is set.
gsht_status accumulate_forward(int L, int lmax, int n, int na, int count, int Q, int is_real,
                               long coefSize, int pitch, const double* rows, double* coef,
                               cudaStream_t s, bool rows32 = false,
                               double* const* fieldPtrs = nullptr);

// Cached operand layout (legendre_fp64.cu); the caller holds g->mu.
const OperandLayout* operand_layout(const gsht_grid* g, int lmax, int na,
                                    int rows, int pad, gsht_status* st);
void free_layouts(gsht_grid* g);
// Cached tile list for a persistent tensor-core launch (legendre_tc.cu).
// dir 0 = inverse (M = colatitudes), 1 = forward (M = degrees); rows = field
// rows R; ntile = field rows per tile; the caller holds g->mu.
// tail: colatitudes at the end left out of the tiles: of the inverse's M
// tiles (their spectra are written by another kernel) or the forward's K
// steps (their products are added in the epilogue).
const TileList* tile_list(const gsht_grid* g, int dir, int lmax, int na, int rows,
                          int ntile, int kstep, gsht_status* st, int tail = 0);

// Spectral buffer element count: (lmax+1) x sgn x count x thetaPad complex.
inline size_t spec_elems(const gsht_grid* g, int lmax, int is_real, int count) {
  const int sgn = is_real ? 1 : 2;
  return (size_t)(lmax + 1) * sgn * count * g->theta_pad;
}

inline long coef_size(int lmax, int n, int is_real) {
  const long na = n < 0 ? -n : n;
  if (is_real) return (long)(lmax + 1) * (lmax + 2) / 2 - na * (na + 1) / 2;
  return (long)(lmax + 1) * (lmax + 1) - (long)n * n;
}

}  // namespace gsht
