/*
 * gsht.h — C ABI of libgsht_cuda.so, the B200 (sm_100a) implementation of the
 * Gauss-Legendre generalized-spherical-harmonic transforms of GSHTrans.
 *
 * Plain C: opaque handles, plain pointers and sizes, status codes. Each entry
 * point names the reference interface it replaces (paths relative to the
 * GSHTrans source tree). The C++ drop-in headers (GSHTrans/Core in this
 * repository) and any FFI binding call only these functions.
 *
 * Conventions shared with the reference:
 *   - grid: nTheta = L+1 Gauss-Legendre colatitudes theta_j = acos(-x_j)
 *     ascending from the north pole, nPhi = 2L longitudes phi_k = k*pi/L;
 *     field values are ring-major (theta outer, phi inner), real or complex
 *     (interleaved re/im doubles) — CanonicalComponentField.h:122-124.
 *   - coefficients: complex (interleaved re/im doubles) in GSHIndices<All>
 *     order for complex fields (index l^2 - n^2 + l + m) and
 *     GSHIndices<NonNegative> order for real fields (index
 *     l(l+1)/2 - |n|(|n|+1)/2 + m) — Indexing.h:104-131,143-146.
 *   - forward ACCUMULATES into its output (c += ...), and for complex fields
 *     with lmax == L sets c_{L,L} = 0 — GaussLegendreGrid.h:186-215.
 *   - FFTs are unnormalised with FFTW's sign conventions.
 *
 * Pointers may be host or device memory (detected per call). With device
 * pointers a call only enqueues work on `stream` (NULL = legacy default
 * stream); with any host pointer the call copies through the grid's
 * workspace and returns after the results are in host memory. Device
 * pointers must be 16-byte aligned (GSHT_ERR_BAD_ARG otherwise).
 * Calls that share one grid handle share its workspace: they are ordered on
 * the GPU (each call waits for the previous one), whichever streams they use.
 */
#ifndef GSHT_H
#define GSHT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gsht_status {
  GSHT_OK = 0,
  GSHT_ERR_BAD_ARG = 1,     /* the reference asserts instead: GaussLegendreGrid.h:41-44,126-134,240-248 */
  GSHT_ERR_OOM = 2,         /* device or host allocation failed */
  GSHT_ERR_CUDA = 3,        /* a CUDA runtime/driver call failed */
  GSHT_ERR_TIMEOUT = 4,     /* a bounded device-side wait expired */
  GSHT_ERR_UNSUPPORTED = 5, /* form not built for this grid, or unsupported shape */
  GSHT_ERR_NO_DEVICE = 6    /* no CUDA device visible */
} gsht_status;

/* Index ranges — Concepts.h:24-27 (All, NonNegative, Single). */
enum { GSHT_RANGE_ALL = 0, GSHT_RANGE_NONNEGATIVE = 1, GSHT_RANGE_SINGLE = 2 };

/* Legendre-stage precision of a transform call. */
enum {
  GSHT_FP64 = 0,   /* FP64 tensor-core (DMMA) contraction: the drop-in path   */
  GSHT_BF16X3 = 1, /* hi/mid/lo BF16 split products, FP32 accumulation       */
  GSHT_OZAKI = 2,  /* Ozaki INT8 slices, exact INT32 accumulation, FP64 sum   */
  GSHT_RECURRENCE = 3, /* FP64 with d^l_mn(theta) generated by the l-recurrence
                          inside the contraction kernels (no stored table); the
                          path GSHT_FP64 takes on grids built without FP64 table */
  GSHT_OZAKI4 = 4     /* Ozaki INT8 with 4 slices (products i + j <= 3): ~1e-7,
                          for the same tier as BF16X3; uses the first 4 planes of
                          the GSHT_FORM_OZAKI table */
};

/* Table forms built by gsht_grid_create (bit mask). GSHT_FORM_RECURRENCE
 * alone builds no table at all: only the recurrence's start values and
 * coefficients (about (L+1)^2 x 28 B per upper index instead of
 * (L+1)^2 (L+1) x 4 B); transforms then run in FP64 through the recurrence,
 * and the BF16x3 / Ozaki forms and gsht_wigner_block are unavailable. No
 * counterpart in the reference, whose grid always stores the table
 * (GaussLegendreGrid.h:52-53). */
enum { GSHT_FORM_FP64 = 1, GSHT_FORM_BF16X3 = 2, GSHT_FORM_OZAKI = 4, GSHT_FORM_RECURRENCE = 8 };

typedef struct gsht_grid gsht_grid;

/* Replaces GaussLegendreGrid<double, MRange, NRange>(lMax, nMax, flag)
 * (GaussLegendreGrid.h:38-73) and the Wigner table it builds
 * (Wigner<double, Ortho, MRange, NRange, Multiple, ColumnMajor>,
 * Wigner.h:116-137): computes the Gauss-Legendre nodes and the Wigner tables
 * for every upper index in the NRange (GridBase.h:17-33) on the GPU.
 * mrange: GSHT_RANGE_ALL or GSHT_RANGE_NONNEGATIVE; nrange: any range;
 * forms: GSHT_FORM_* mask (the FP64 table is built unless forms is exactly
 * GSHT_FORM_RECURRENCE). */
gsht_status gsht_grid_create(int lmax, int nmax, int mrange, int nrange,
                             unsigned forms, gsht_grid** grid);

/* Releases the grid, its tables and its workspace. */
gsht_status gsht_grid_destroy(gsht_grid* grid);

/* MaxDegree / MaxUpperIndex / MinUpperIndex / NumberOfCoLatitudes /
 * NumberOfLongitudes (GaussLegendreGrid.h:86-87, GridBase.h:17-45). Any
 * output pointer may be NULL. */
gsht_status gsht_grid_shape(const gsht_grid* grid, int* lmax, int* nmax,
                            int* min_n, int* n_theta, int* n_phi);

/* CoLatitudes() and CoLatitudeWeights() (GaussLegendreGrid.h:89-92) into
 * host arrays of n_theta doubles (either may be NULL). */
gsht_status gsht_grid_nodes(const gsht_grid* grid, double* colatitudes,
                            double* weights);

/* Wigner::operator[](n, iTheta) (Wigner.h:241-244): copies the table block
 * d^l_{mn}(theta_iTheta), l = |n|..L, in the reference's block layout
 * (GSHIndices<MRange>(L, L, n), Indexing.h:104-131) into host memory. If
 * out is NULL only *count is set. */
gsht_status gsht_wigner_block(const gsht_grid* grid, int n, int itheta,
                              double* out, long* count);

/* Wigner<double, Norm, MRange, NRange, AngleRange, Storage>(lMax, mMax, nMax,
 * theta) (Wigner.h:99-159, 289-486) for arbitrary angles: d^l_{mn}(theta_k)
 * for every upper index of the NRange (All: -nMax..nMax, NonNegative:
 * 0..nMax, Single: nMax), computed on the GPU (same recurrence and start
 * values as the grid tables) and written to host memory in the reference's
 * storage: one block GSHIndices<MRange>(lMax, mMax, n) per (n, angle), n
 * outer (ColumnMajor, row_major = 0) or angle outer (RowMajor). norm: 0
 * Ortho, 1 FourPi. With out == NULL only *count (the total length) is set. */
gsht_status gsht_wigner_compute(int lmax, int mmax, int nmax, int mrange, int nrange,
                                int norm, int row_major, const double* theta, int ntheta,
                                double* out, long* count);

/* Coefficient count for (lmax, n): GridBase.h:79-85 (Real/ComplexCoefficientSize). */
long gsht_coefficient_size(int lmax, int n, int is_real);

/* ForwardTransformation(lMax, n, in, out) (GaussLegendreGrid.h:108-217):
 * grid values -> coefficients, accumulated into out. */
gsht_status gsht_forward(const gsht_grid* grid, int lmax, int n, int is_real,
                         int precision, const void* in, void* out,
                         void* stream);

/* InverseTransformation(lMax, n, in, out) (GaussLegendreGrid.h:222-321):
 * coefficients -> grid values (out overwritten). */
gsht_status gsht_inverse(const gsht_grid* grid, int lmax, int n, int is_real,
                         int precision, const void* in, void* out,
                         void* stream);

/* Batched forms: `count` fields of the same (lmax, n, is_real), stored back
 * to back (field i at in + i * field_size, out + i * coefficient_size; sizes
 * in elements of the respective type). One call runs each stage once for the
 * whole batch, sharing the Wigner table across the fields. */
gsht_status gsht_forward_batch(const gsht_grid* grid, int lmax, int n,
                               int is_real, int precision, int count,
                               const void* in, void* out, void* stream);
gsht_status gsht_inverse_batch(const gsht_grid* grid, int lmax, int n,
                               int is_real, int precision, int count,
                               const void* in, void* out, void* stream);

/* Stages of one transform split over several GPUs (ranks): the ring FFTs
 * shard over colatitudes, the Legendre sums over orders, and the spectra
 * cross between the two by an all-to-all exchange that the caller runs
 * (gshtrans_b200.sharded does it over torch.distributed). No counterpart in
 * the reference, whose transforms loop serially over the rings
 * (GaussLegendreGrid.h:163, :281). FP64 with the stored table; all buffers
 * are device memory of the grid's device; work is enqueued on `stream`.
 *
 * The spectra buffer (gsht_spectra_layout: `elems` complex doubles, column
 * pitch `pitch`) is [m][sgn][field][pitch] for m = 0..lmax, sgn = 0 (+m) and,
 * for complex fields, 1 (-m): column j of a +m row holds ring j, column
 * nTheta-1-j of a -m row holds ring j (the colatitude mirror); columns
 * [nTheta, pitch) must hold zeros when gsht_forward_orders reads it.
 *
 * gsht_forward_rings: ring FFTs of rings [ring_begin, ring_end) of `count`
 * fields (full-size grids, other rings not read), weighted by the Gauss
 * weights and 2 pi / nPhi (GaussLegendreGrid.h:165-178), into their spectra
 * columns. gsht_forward_orders: the forward Legendre sums of orders
 * [m_begin, m_end) from complete spectra columns, ADDED into the packed
 * coefficients like ForwardTransformation (GaussLegendreGrid.h:183-207; the
 * c_{L,L} = 0 rule is the caller's once the shares are summed).
 * gsht_inverse_orders: the inverse sums of orders [m_begin, m_end) into the
 * spectra rows of those orders, every column (GaussLegendreGrid.h:284-312).
 * gsht_inverse_rings: backward FFTs of rings [ring_begin, ring_end) from
 * complete spectra rows into those grid rings (GaussLegendreGrid.h:314-319). */
gsht_status gsht_spectra_layout(const gsht_grid* grid, int lmax, int is_real, int count,
                                long* elems, int* pitch);
gsht_status gsht_forward_rings(const gsht_grid* grid, int lmax, int is_real, int count,
                               int ring_begin, int ring_end, const void* grid_values,
                               void* spectra, void* stream);
gsht_status gsht_forward_orders(const gsht_grid* grid, int lmax, int n, int is_real, int count,
                                int m_begin, int m_end, const void* spectra, void* coef_out,
                                void* stream);
gsht_status gsht_inverse_orders(const gsht_grid* grid, int lmax, int n, int is_real, int count,
                                int m_begin, int m_end, const void* coef_in, void* spectra,
                                void* stream);
gsht_status gsht_inverse_rings(const gsht_grid* grid, int lmax, int is_real, int count,
                               int ring_begin, int ring_end, const void* spectra,
                               void* grid_values, void* stream);

/* Allocation-free FP64 inverse transform of ONE field. No counterpart in the
 * reference: it serves callers that must not allocate device memory while
 * they transform (an owning arena or caching allocator, a latency-critical
 * loop, or a component that must not meet out-of-memory after start-up).
 * `in` (coefficients) and `out` (grid values) must be device pointers; the
 * scratch comes from a fixed 16 MiB array in the library's device memory,
 * which every GPU that loads the library holds until the process exits.
 * Sizes whose scratch would exceed it are rejected with GSHT_ERR_UNSUPPORTED
 * and a message giving the bytes needed (a complex field on a grid of its
 * own degree fits up to lmax ~ 580, a real one up to ~ 800); lmax >= 1.
 * The first call on a device looks up the array's device address, so make
 * that first call before any stream capture. All calls share the one array
 * and it keeps the last call's contents: calls that overlap on the GPU (on
 * different streams, or different threads) race and corrupt each other;
 * order them. CUDA loads the library's device module lazily, so the first
 * call on a device is also when the 16 MiB are reserved there: make it at
 * start-up (a failure then reads GSHT_ERR_OOM). The cached address goes
 * stale after cudaDeviceReset. Results equal gsht_inverse with GSHT_FP64. */
gsht_status gsht_inverse_noalloc(const gsht_grid* grid, int lmax, int n, int is_real,
                                 const void* in, void* out, void* stream);

/* Fused pointwise field expressions. Replaces the materialising assignment
 * of CanonicalComponentField expressions (CanonicalComponentFieldBase.h
 * :201-339) over the lazy nodes of CanonicalComponentFieldBinary.h:100-305
 * (+ - * /), CanonicalComponentFieldUnary.h:103-354 (conj, real, imag, unary
 * minus) and the scalar forms of CanonicalComponentFieldOverloads.h:66-146.
 * `program` is the expression in postfix order over a value stack; LOAD
 * pushes input[arg] at the current point (a real input as x + 0i), CONST
 * pushes re + i im, the binary operations pop b then a and push a op b.
 * `count` fields are evaluated, field k of every buffer starting at
 * k * field_stride elements; inputs and output hold complex (interleaved)
 * or real doubles; a real output keeps the real part. Runs as one kernel on
 * `stream`: each point reads its inputs once and writes its value once. With
 * device buffers the call only enqueues; host buffers are staged through a
 * library workspace and the call returns with the result in host memory.
 * Limits: 64 operations, 16 inputs, a stack 8 values deep.
 * The first call with a given program (on a device) compiles it into a
 * kernel of its own with NVRTC (loaded at run time, libnvrtc.so.12), cached
 * for later calls; where NVRTC is unavailable or compilation fails, an
 * interpreting kernel evaluates the program instead (GSHT_FIELD_JIT=0 forces
 * it). gsht_field_jit_stats reports how many programs were compiled and how
 * many could not be (NULL arguments are skipped). */
enum {
  GSHT_OP_LOAD = 0, GSHT_OP_CONST = 1, GSHT_OP_ADD = 2, GSHT_OP_SUB = 3,
  GSHT_OP_MUL = 4, GSHT_OP_DIV = 5, GSHT_OP_NEG = 6, GSHT_OP_CONJ = 7,
  GSHT_OP_REAL = 8, GSHT_OP_IMAG = 9
};
typedef struct gsht_expr_op {
  int op;
  int arg;
  double re;
  double im;
} gsht_expr_op;
gsht_status gsht_field_eval(const gsht_expr_op* program, int nops,
                            const void* const* inputs, const int* input_is_real,
                            int ninputs, void* out, int out_is_real, long npoints,
                            int count, long field_stride, void* stream);
gsht_status gsht_field_jit_stats(int* compiled, int* failed);

/* Batched transforms of many fields of uneven size in one CUDA graph. No
 * counterpart in the reference (its transforms take one field per call,
 * GaussLegendreGrid.h:108-321; callers loop). Each field has its own degree
 * and Gauss-Legendre grid (nTheta = lmax + 1, nPhi = 2 lmax), upper index and
 * kind; its buffers are device memory in the layouts of gsht_forward /
 * gsht_inverse: coef_in (packed coefficients the inverse reads), grid (the
 * inverse writes, the forward reads), coef_out (the forward ADDS into, like
 * ForwardTransformation). gsht_plan_batch groups the fields by (lmax, n,
 * kind), builds one grid per distinct lmax (tables shared by every field of
 * that degree), autotunes the BF16x3 tensor-core tile width per group when
 * `autotune` is set, and captures one CUDA graph per mode; the buffers'
 * addresses are fixed at planning, their contents are read at each
 * execution. A plan is not thread-safe. */
typedef struct gsht_field_desc {
  int lmax;
  int n;
  int is_real;
  const void* coef_in;
  void* grid;
  void* coef_out;
} gsht_field_desc;
typedef struct gsht_batch gsht_batch;
enum {
  GSHT_BATCH_FORWARD = 0,    /* grids -> coef_out += coefficients */
  GSHT_BATCH_INVERSE = 1,    /* coef_in -> grids */
  GSHT_BATCH_ROUND_TRIP = 2  /* inverse, then forward of the grids just made */
};
gsht_status gsht_plan_batch(const gsht_field_desc* fields, int count, int precision,
                            int autotune, gsht_batch** out);
gsht_status gsht_batch_execute(gsht_batch* batch, int mode, void* stream);
/* Number of (lmax, n, kind) groups, of grids, and of graph nodes per mode. */
gsht_status gsht_batch_info(const gsht_batch* batch, int* groups, int* grids,
                            long* graph_nodes /* [3] or NULL */);
gsht_status gsht_batch_group(const gsht_batch* batch, int index, int* lmax, int* n,
                             int* is_real, int* count, int* ntile);
/* Number of streams the plan's graphs spread the groups over (each group
 * has its own workspace; with `autotune` the count is the fastest of 1, 2,
 * 4, 8, 16 for the round trip). Groups are listed largest first. */
gsht_status gsht_batch_schedule(const gsht_batch* batch, int* streams);
gsht_status gsht_batch_destroy(gsht_batch* batch);

/* Stage timing. No counterpart in the reference (which has no tracing):
 * while enabled, every stage of a transform call is bracketed by CUDA events
 * recorded on the call's stream; gsht_profile_read synchronises those events
 * and returns, per stage, the summed device milliseconds and the number of
 * kernel launches (counted per calling thread, so exact for each thread's
 * own calls; a stage's time brackets whatever else runs on its stream
 * meanwhile). Completed records are folded into per-stage totals, so long
 * profiled loops hold a bounded number of events. Enabling clears earlier
 * records. */
enum {
  GSHT_STAGE_PREP_INVERSE = 0,     /* coefficients -> per-order operand rows   */
  GSHT_STAGE_LEGENDRE_INVERSE = 1, /* order-wise contraction, inverse          */
  GSHT_STAGE_FFT_INVERSE = 2,      /* ring FFTs, inverse                       */
  GSHT_STAGE_FFT_FORWARD = 3,      /* ring FFTs, forward                       */
  GSHT_STAGE_PREP_FORWARD = 4,     /* spectra -> per-order operand rows        */
  GSHT_STAGE_LEGENDRE_FORWARD = 5, /* order-wise contraction, forward          */
  GSHT_STAGE_ACCUMULATE_FORWARD = 6, /* forward result rows added into the packed
                                        coefficients (tensor-core and recurrence
                                        forms)                                  */
  GSHT_STAGE_COUNT = 7
};
gsht_status gsht_profile_enable(int on);
gsht_status gsht_profile_read(double* ms, long* launches, int nstages);

/* Synchronises the grid's device and reports GSHT_ERR_TIMEOUT if a kernel
 * gave up a bounded wait since the last check (the word is then cleared).
 * No counterpart in the reference, which has no device code. Calls with
 * host buffers perform this check themselves. */
gsht_status gsht_device_status(const gsht_grid* grid);

/* Runs the failure path of the bounded device waits on purpose: one thread
 * of a one-block kernel waits, with the wait the tensor-core pipelines use,
 * on an mbarrier phase that nothing completes; after the wait limit (about
 * half a second) it raises the grid's device error word (code 100) and the
 * kernel returns. A following gsht_device_status reports GSHT_ERR_TIMEOUT
 * and clears the word; the context stays usable. No counterpart in the
 * reference (it has no device code); for checking that a caller's error
 * handling sees device-side timeouts. Enqueued on `stream`. */
gsht_status gsht_check_bounded_wait(const gsht_grid* grid, void* stream);

/* Per-role cycle trace of the tensor-core Legendre kernels. No counterpart
 * in the reference (it has no device code). While enabled (a process-wide
 * switch), the Legendre stage of BF16x3 and Ozaki transforms launches traced
 * copies of its kernels (the BF16x3 one-CTA kernel only at its 128-row tile
 * width): same results, and every thread that waits in the pipeline times its
 * waits with clock64. gsht_tc_trace_read synchronises the calling thread's
 * current device and returns the counters of the last traced launch of one
 * form (GSHT_BF16X3, or GSHT_OZAKI / GSHT_OZAKI4, which share them) and
 * direction (0 inverse, 1 forward) as GSHT_TRACE_SLOTS doubles, in SM clock
 * cycles summed over the CTAs (the epilogue slots also over its warps):
 *   [0] producer thread, kernel start to its end  [1] of which waiting for a
 *   free stage  [2] MMA issuing thread, start to end  [3] of which waiting for
 *   a loaded stage  [4] of which waiting for the epilogue to free the
 *   accumulators  [5] epilogue warps, start to end  [6] of which waiting for
 *   finished accumulators  [7] CTAs  [8] CTAs that issued MMAs (in the
 *   CTA-pair kernels only the first CTA of a pair issues).
 * A diagnostic: the traced kernels add a few instructions per wait. */
#define GSHT_TRACE_SLOTS 9
gsht_status gsht_tc_trace_enable(int on);
gsht_status gsht_tc_trace_read(int form, int direction, double* out, int n);

/* Device-memory allocator hook. No counterpart in the reference (its tables
 * live in host std::vector storage, Wigner.h:126-128). Every device
 * allocation of the library (grid tables and nodes, workspaces, batch plans,
 * staging buffers) is made by alloc(bytes, ctx) and released by free_fn(ptr,
 * ctx) of the hook that made it, even if the hook has been changed since. A
 * NULL from alloc makes the call that needed the memory return GSHT_ERR_OOM
 * after releasing what it had taken. For callers whose device memory belongs
 * to a pool (a caching allocator, an arena). Both NULL restores cudaMalloc /
 * cudaFree. Change it only while no other thread is inside the library; the
 * hook is called with the library's allocation lock held, so it must not
 * call back into the library. */
typedef void* (*gsht_alloc_fn)(size_t bytes, void* ctx);
typedef void (*gsht_free_fn)(void* ptr, void* ctx);
gsht_status gsht_set_allocator(gsht_alloc_fn alloc, gsht_free_fn free_fn, void* ctx);

/* Device allocations and releases the library has made in this process, and
 * the bytes it holds now (any of the pointers may be NULL). */
gsht_status gsht_alloc_stats(unsigned long long* allocations, unsigned long long* releases,
                             size_t* live_bytes);

/* Message describing the last non-OK status returned on this thread. */
const char* gsht_last_error(void);

/* Number of kernels this library has launched in this process (used to
 * count device work inside timed regions). */
unsigned long long gsht_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* GSHT_H */
