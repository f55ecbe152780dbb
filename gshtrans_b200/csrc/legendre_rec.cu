// Legendre stage in FP64 with the Wigner values generated inside the
// contraction by the l-recurrence (no stored table).
//
// The stored-table kernels read d^l_mn(theta_j) from HBM: 34.7 GB per
// transform at lmax 2048 for one upper index, which bounds a single-field
// transform by HBM bandwidth and a grid's memory by the table. Here each
// thread runs the recurrence of the table build (grid.cu: Wigner.h:347-472
// with exponent-extended start values) for its colatitudes and contracts
// every value as it is produced, so the work is FP64 arithmetic on the CUDA
// cores and the grid holds only the start values and the per-row recurrence
// coefficients ((L+1)^2/2 x 24 B).
//
// The chains carry e_k = d_k / s_k, for which the recurrence reads
// e_k = (a'_k cos - b'_k) e_{k-1} - e_{k-2} (two FMAs per step); the factor
// sc_k = norm_k s_k goes onto the other operand (grid.cu, k_rec_coefficients).
//
//   inverse  spec[m][q][j] = sum_k (A[m][q][k] sc_k) e_k(theta_j)
//            (A: the FP64 operand rows of legendre_fp64.cu; +m and the
//            mirrored -m rows share d through d^l_{-m,n}(pi - theta) =
//            (-1)^{l+n} d^l_{mn}(theta))
//   forward  R[m][q][k] = sc_k sum_j e_k(theta_j) spec[m][q][j], then
//            accumulate_forward adds R into the packed coefficients.
//
// Values still in exponent-extended form (below 2^-612, near the poles at
// high degree) are contracted as zero; the table stores them scaled back,
// where they are equally negligible against O(2^-52) rounding of the sums.
// Warps whose chains are all in double range (nearly all) run the steps
// without the exponent checks.
#include "gsht_internal.cuh"

namespace gsht {
namespace {

struct RecArgs {
  int lmax, na, Q, nTheta, thetaPad;
  const long long* rowOff;  // table row offset per m (grid degree layout)
  const long long* opOff;   // inverse operand offset per m
  const int* opPitch;       // inverse operand pitch per m
  const double* theta;
  const double* startF;     // [m][thetaPad] start value mantissas
  const int* startE;        // [m][thetaPad] start value exponents
  const double2* ab;        // per row: (a', b')
  const double* sc;         // per row: norm_k s_k
  const double2* A;         // inverse: operand; forward: spec [m][Q][thetaPad]
  double2* out;             // inverse: spec; forward: partial sums [blk][Q][rows]
  long long rows;           // table rows (forward partial plane)
};

// Exponent-extended chain state of one colatitude: e = p1 * 2^E.
struct Chain {
  double cs, p1, p2;
  int E;
};

// Initial state e_{-1} = 0, e_{-2} = -d_0, so that step 0 ((a', b') =
// (0, -1)) yields d_0 and every step is the same update.
__device__ __forceinline__ Chain chain_start(const RecArgs& p, int m, int j) {
  Chain c;
  c.cs = cos(p.theta[j]);
  int ef = 0;
  const size_t o = (size_t)m * p.thetaPad + j;
  const double f0 = frexp(p.startF[o], &ef);  // [0.5, 1)
  const int e0 = p.startE[o] + ef;
  c.E = (f0 != 0.0 && e0 < -900) ? -512 * ((-900 - e0 + 511) / 512) : 0;
  c.p1 = 0.0;
  c.p2 = -ldexp(f0, e0 - c.E);
  return c;
}

// One step; kChecked also moves the chain out of the extended range and
// returns 0 for values still scaled.
template <bool kChecked>
__device__ __forceinline__ double chain_step(Chain& c, double a, double b) {
  const double p = fma(fma(a, c.cs, -b), c.p1, -c.p2);
  c.p2 = c.p1;
  c.p1 = p;
  if constexpr (kChecked) {
    if (c.E < 0 && fabs(c.p1) >= 0x1p-100) {
      c.p1 = ldexp(c.p1, -512);
      c.p2 = ldexp(c.p2, -512);
      c.E += 512;
    }
    return c.E == 0 ? c.p1 : 0.0;
  }
  return p;
}

// Colatitudes per thread (inverse): 1 ran 8% slower, 4 (98 registers) 43%
// slower at lmax 2048.
constexpr int kInvT = 2;
// Blocks per SM asked of the compiler for one or two rows: 4 (64 registers)
// ran the lmax 2048 inverse in 2.67 ms against 3.10 ms at 98 registers.
constexpr int kInvMinBlocks = 4;

// Inverse: block (colatitude block of 256 x kInvT, order m, row group of kQ).
// The block's operand rows (times sc_k) and recurrence coefficients are
// staged in shared memory 256 degrees at a time and read as broadcasts; each
// thread carries kInvT independent chains.
template <int kQ, bool kChecked>
__device__ __forceinline__ void rec_inv_steps(int kn, const double2* sAB,
                                              const double2 (*sA)[256], Chain (&ch)[kInvT],
                                              double2 (&acc)[kInvT][kQ]) {
#pragma unroll 4
  for (int i = 0; i < kn; i++) {
    const double2 ab = sAB[i];
    double v[kInvT];
#pragma unroll
    for (int t = 0; t < kInvT; t++) v[t] = chain_step<kChecked>(ch[t], ab.x, ab.y);
#pragma unroll
    for (int q = 0; q < kQ; q++) {
      const double2 a = sA[q][i];
#pragma unroll
      for (int t = 0; t < kInvT; t++) {
        acc[t][q].x = fma(a.x, v[t], acc[t][q].x);
        acc[t][q].y = fma(a.y, v[t], acc[t][q].y);
      }
    }
  }
}

template <int kQ>
__global__ void __launch_bounds__(256, kQ <= 2 ? kInvMinBlocks : 1) k_legendre_rec_inv(RecArgs p) {
  __shared__ double2 sAB[256];
  __shared__ double2 sA[kQ][256];
  const int m = blockIdx.y, q0 = blockIdx.z * kQ;
  const int l0 = m > p.na ? m : p.na;
  const int K = p.lmax - l0 + 1;
  const int kp = p.opPitch[m];
  const int tid = threadIdx.x;
  const size_t row0 = (size_t)p.rowOff[m];
  const double2* A = p.A + p.opOff[m] + (size_t)q0 * kp;
  Chain ch[kInvT];
  int j[kInvT];
  bool mine = false;
#pragma unroll
  for (int t = 0; t < kInvT; t++) {
    j[t] = (blockIdx.x * kInvT + t) * 256 + tid;
    mine |= j[t] < p.nTheta;
    ch[t] = chain_start(p, m, j[t] < p.nTheta ? j[t] : 0);
  }
  // Warps with no colatitude inside the grid (the last block's tail) only
  // help with the staging.
  const bool warpActive = __any_sync(0xffffffffu, mine);
  double2 acc[kInvT][kQ];
#pragma unroll
  for (int t = 0; t < kInvT; t++)
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[t][q] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < K; k0 += 256) {
    __syncthreads();
    const int k = k0 + tid;
    double f = 0.0;
    if (k < K) {
      sAB[tid] = p.ab[row0 + k];
      f = p.sc[row0 + k];
    }
#pragma unroll
    for (int q = 0; q < kQ; q++) {
      double2 a = make_double2(0.0, 0.0);
      if (q0 + q < p.Q && k < K) a = A[(size_t)q * kp + k];
      sA[q][tid] = make_double2(a.x * f, a.y * f);
    }
    __syncthreads();
    if (!warpActive) continue;
    const int kn = K - k0 < 256 ? K - k0 : 256;
    bool scaled = false;
#pragma unroll
    for (int t = 0; t < kInvT; t++) scaled |= ch[t].E < 0;
    if (__any_sync(0xffffffffu, scaled))
      rec_inv_steps<kQ, true>(kn, sAB, sA, ch, acc);
    else
      rec_inv_steps<kQ, false>(kn, sAB, sA, ch, acc);
  }
#pragma unroll
  for (int t = 0; t < kInvT; t++) {
    if (j[t] >= p.nTheta) continue;
#pragma unroll
    for (int q = 0; q < kQ; q++)
      if (q0 + q < p.Q) p.out[((size_t)m * p.Q + q0 + q) * p.thetaPad + j[t]] = acc[t][q];
  }
}

// Sum over the warp of V values per lane with log2(V) exchange steps that
// halve the values each lane holds, then plain butterfly steps: 5 + V/2 - 1
// shuffles instead of 5 V. Afterwards lane l holds the sum of value
// l >> (5 - log2 V) in x[0].
template <int V>
__device__ __forceinline__ void warp_sum_spread(double (&x)[V], int lane) {
  int width = 16;
#pragma unroll
  for (int n = V; n > 1; n >>= 1) {
    const bool upper = (lane & width) != 0;
#pragma unroll
    for (int i = 0; i < n / 2; i++) {
      const double send = upper ? x[i] : x[i + n / 2];
      const double keep = upper ? x[i + n / 2] : x[i];
      x[i] = keep + __shfl_xor_sync(0xffffffffu, send, width);
    }
    width >>= 1;
  }
#pragma unroll
  for (; width >= 1; width >>= 1) x[0] += __shfl_xor_sync(0xffffffffu, x[0], width);
}

constexpr int kFwdChunk = 32;  // degrees per shared-memory reduction round

// Colatitudes per thread and degrees per warp reduction (G x 2 kQ = 8
// values). A sweep at lmax 2048 (one complex field) chose these: 4
// colatitudes per thread or 16-value reductions need 80-128 registers and
// ran 17-78% slower at the lower occupancy; one colatitude per thread 34-56%
// slower.
template <int kQ>
__host__ __device__ constexpr int fwd_t() { return 2; }
template <int kQ>
__host__ __device__ constexpr int fwd_g() { return kQ >= 4 ? 1 : 4 / kQ; }

template <int kQ, bool kChecked>
__device__ __forceinline__ void rec_fwd_steps(int kn, int warp, int lane, const double2* sAB,
                                              double (*red)[kFwdChunk][2 * kQ],
                                              Chain (&ch)[fwd_t<kQ>()],
                                              const double2 (&F)[fwd_t<kQ>()][kQ]) {
  constexpr int T = fwd_t<kQ>(), V = 2 * kQ, G = fwd_g<kQ>(), W = G * V;
  for (int i0 = 0; i0 < kn; i0 += G) {
    double x[W];
#pragma unroll
    for (int g = 0; g < G; g++) {
      const double2 ab = sAB[i0 + g];
      double v[T];
#pragma unroll
      for (int t = 0; t < T; t++) v[t] = chain_step<kChecked>(ch[t], ab.x, ab.y);
#pragma unroll
      for (int q = 0; q < kQ; q++) {
        double sr = v[0] * F[0][q].x, si = v[0] * F[0][q].y;
#pragma unroll
        for (int t = 1; t < T; t++) {
          sr = fma(v[t], F[t][q].x, sr);
          si = fma(v[t], F[t][q].y, si);
        }
        x[g * V + 2 * q] = sr;
        x[g * V + 2 * q + 1] = si;
      }
    }
    warp_sum_spread<W>(x, lane);
    if ((lane & (32 / W - 1)) == 0) {
      const int idx = lane / (32 / W);
      red[warp][i0 + idx / V][idx % V] = x[0];
    }
  }
}

// Forward: block (colatitude block of 256 x T, order m, row group of kQ).
// Each thread holds its colatitudes' spectra in registers and runs their
// chains; per degree the products are summed over the thread's colatitudes,
// over the warp (warp_sum_spread, G degrees at a time) and, every kFwdChunk
// degrees, over the block's warps, giving one partial sum per (block, row,
// degree).
template <int kQ>
__global__ void __launch_bounds__(256) k_legendre_rec_fwd(RecArgs p) {
  constexpr int T = fwd_t<kQ>();
  constexpr int V = 2 * kQ;
  __shared__ double2 sAB[kFwdChunk];
  __shared__ double red[8][kFwdChunk][V];
  __shared__ bool activeW[8];
  const int m = blockIdx.y, q0 = blockIdx.z * kQ;
  const int l0 = m > p.na ? m : p.na;
  const int K = p.lmax - l0 + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t row0 = (size_t)p.rowOff[m];
  Chain ch[T];
  double2 F[T][kQ];
  bool mine = false;
#pragma unroll
  for (int t = 0; t < T; t++) {
    const int j = (blockIdx.x * T + t) * 256 + tid;
    const bool ok = j < p.nTheta;
    mine |= ok;
    ch[t] = chain_start(p, m, ok ? j : 0);
#pragma unroll
    for (int q = 0; q < kQ; q++)
      F[t][q] = (ok && q0 + q < p.Q) ? p.A[((size_t)m * p.Q + q0 + q) * p.thetaPad + j]
                                     : make_double2(0.0, 0.0);
  }
  // Warps with no colatitude inside the grid (the last block's tail) skip
  // the chains and are left out of the block sums.
  const bool warpActive = __any_sync(0xffffffffu, mine);
  if (lane == 0) activeW[warp] = warpActive;
  double* part = reinterpret_cast<double*>(p.out);
  for (int k0 = 0; k0 < K; k0 += kFwdChunk) {
    __syncthreads();
    // Degrees past K get (a', b') = (0, 0): their chain steps only swap
    // bounded values, and their sums are never read.
    if (tid < kFwdChunk) sAB[tid] = k0 + tid < K ? p.ab[row0 + k0 + tid] : make_double2(0.0, 0.0);
    __syncthreads();
    const int kn = K - k0 < kFwdChunk ? K - k0 : kFwdChunk;
    if (warpActive) {
      bool scaled = false;
#pragma unroll
      for (int t = 0; t < T; t++) scaled |= ch[t].E < 0;
      if (__any_sync(0xffffffffu, scaled))
        rec_fwd_steps<kQ, true>(kn, warp, lane, sAB, red, ch, F);
      else
        rec_fwd_steps<kQ, false>(kn, warp, lane, sAB, red, ch, F);
    }
    __syncthreads();
    for (int u = tid; u < kn * V; u += 256) {
      const int i = u / V, c = u - i * V, q = c >> 1;
      if (q0 + q >= p.Q) continue;
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 8; w++)
        if (activeW[w]) s += red[w][i][c];
      const size_t plane = (size_t)blockIdx.x * p.Q + q0 + q;
      part[2 * (plane * p.rows + row0 + k0 + i) + (c & 1)] = s;
    }
  }
}

// Forward finish: R[m][q][k] = sc_k * sum over colatitude blocks, written
// order-major with pitch thetaPad (into the spectra buffer) for
// accumulate_forward.
__global__ void k_rec_forward_sum(int lmax, int na, int Q, int nblk, int thetaPad,
                                  long long rows, const long long* __restrict__ rowOff,
                                  const double* __restrict__ sc,
                                  const double2* __restrict__ part, double2* __restrict__ out) {
  const int m = blockIdx.y, q = blockIdx.z;
  const int l0 = m > na ? m : na;
  const int K = lmax - l0 + 1;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const size_t r = (size_t)rowOff[m] + k;
  double2 s = make_double2(0.0, 0.0);
  for (int b = 0; b < nblk; b++) {
    const double2 v = part[((size_t)b * Q + q) * rows + r];
    s.x += v.x;
    s.y += v.y;
  }
  const double f = sc[r];
  out[((size_t)m * Q + q) * thetaPad + k] = make_double2(s.x * f, s.y * f);
}

int fwd_kq(int Q) { return Q <= 1 ? 1 : (Q <= 2 ? 2 : 4); }

int fwd_blocks(int nTheta, int kq) {
  const int per = 256 * (kq == 1 ? fwd_t<1>() : (kq == 2 ? fwd_t<2>() : fwd_t<4>()));
  return (nTheta + per - 1) / per;
}

RecArgs rec_args(const gsht_grid* g, const Table* t, int lmax, int Q) {
  RecArgs a{};
  a.lmax = lmax;
  a.na = t->n < 0 ? -t->n : t->n;
  a.Q = Q;
  a.nTheta = g->n_theta;
  a.thetaPad = g->theta_pad;
  a.rowOff = t->d_row_off;
  a.theta = g->d_theta;
  a.startF = t->rec_f;
  a.startE = t->rec_e;
  a.ab = t->rec_ab;
  a.sc = t->rec_sc;
  a.rows = t->rows;
  return a;
}

}  // namespace

size_t rec_forward_bytes(const gsht_grid* g, const Table* t, int is_real, int count) {
  const int Q = (is_real ? 1 : 2) * count;
  return sizeof(double2) * (size_t)fwd_blocks(g->n_theta, fwd_kq(Q)) * Q * (size_t)t->rows;
}

gsht_status legendre_inverse_rec(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                 int count, const double* coef, double* operand, double* spec,
                                 cudaStream_t s) {
  if (!t->rec_f) return fail(GSHT_ERR_UNSUPPORTED, "the recurrence form was not built for this grid");
  const int Q = (is_real ? 1 : 2) * count;
  const OperandLayout* lay = nullptr;
  gsht_status st = prep_inverse_fp64(g, t, lmax, is_real, count, coef, operand, &lay, s);
  if (st != GSHT_OK) return st;
  RecArgs a = rec_args(g, t, lmax, Q);
  a.opOff = lay->d_off;
  a.opPitch = lay->d_pitch;
  a.A = reinterpret_cast<const double2*>(operand);
  a.out = reinterpret_cast<double2*>(spec);
  StageTimer tm(GSHT_STAGE_LEGENDRE_INVERSE, s);
  const int kq = Q <= 1 ? 1 : (Q <= 2 ? 2 : (Q <= 4 ? 4 : 8));
  dim3 grid((g->n_theta + 256 * kInvT - 1) / (256 * kInvT), lmax + 1, (Q + kq - 1) / kq);
  if (kq == 1) k_legendre_rec_inv<1><<<grid, 256, 0, s>>>(a);
  else if (kq == 2) k_legendre_rec_inv<2><<<grid, 256, 0, s>>>(a);
  else if (kq == 4) k_legendre_rec_inv<4><<<grid, 256, 0, s>>>(a);
  else k_legendre_rec_inv<8><<<grid, 256, 0, s>>>(a);
  GSHT_LAUNCH_CHECK("k_legendre_rec_inv");
  return GSHT_OK;
}

gsht_status legendre_forward_rec(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                 int count, double* spec, void* partial, double* coef,
                                 cudaStream_t s) {
  if (!t->rec_f) return fail(GSHT_ERR_UNSUPPORTED, "the recurrence form was not built for this grid");
  const int Q = (is_real ? 1 : 2) * count;
  const int na = t->n < 0 ? -t->n : t->n;
  const int kq = fwd_kq(Q);
  const int nblk = fwd_blocks(g->n_theta, kq);
  RecArgs a = rec_args(g, t, lmax, Q);
  a.A = reinterpret_cast<const double2*>(spec);
  a.out = static_cast<double2*>(partial);
  {
    StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
    dim3 grid(nblk, lmax + 1, (Q + kq - 1) / kq);
    if (kq == 1) k_legendre_rec_fwd<1><<<grid, 256, 0, s>>>(a);
    else if (kq == 2) k_legendre_rec_fwd<2><<<grid, 256, 0, s>>>(a);
    else k_legendre_rec_fwd<4><<<grid, 256, 0, s>>>(a);
    GSHT_LAUNCH_CHECK("k_legendre_rec_fwd");
    const int kMax = lmax - na + 1;
    dim3 sg((kMax + 127) / 128, lmax + 1, Q);
    k_rec_forward_sum<<<sg, 128, 0, s>>>(lmax, na, Q, nblk, g->theta_pad, t->rows, t->d_row_off,
                                         t->rec_sc, static_cast<const double2*>(partial),
                                         reinterpret_cast<double2*>(spec));
    GSHT_LAUNCH_CHECK("k_rec_forward_sum");
  }
  return accumulate_forward(g->L, lmax, t->n, na, count, Q, is_real,
                            coef_size(lmax, t->n, is_real), g->theta_pad, spec, coef, s);
}

}  // namespace gsht
