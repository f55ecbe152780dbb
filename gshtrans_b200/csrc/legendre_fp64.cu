// Legendre stage in FP64: per order m, a dense contraction of the batch's
// coefficients (rows: field x {+m, -m}) against the Wigner table block
// d^l_{mn}(theta_j), on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64).
//
// Replaces the theta-loop accumulations of GaussLegendreGrid.h:176-207
// (forward: c_lm += sum_j d^l_mn(theta_j) F_j(m) w_j 2pi/nPhi) and :284-312
// (inverse: F_j(m) = sum_l c_lm d^l_mn(theta_j)), reorganised so that the
// table block of |m| is read once for the whole batch and for both signs of m
// (negative orders use d^l_{-m,n}(pi-theta) = (-1)^{l+n} d^l_{mn}(theta); the
// spectral buffer stores -m at mirrored colatitudes).
#include <cstdio>

#include "gsht_internal.cuh"

namespace gsht {
namespace {

constexpr int BMC = 32;   // complex rows per block tile
constexpr int BN = 128;   // columns per block tile
constexpr int BK = 16;    // reduction depth per stage
constexpr int STAGES = 3;
constexpr int PA = 20;    // A smem pitch (double2 units): conflict-free fragments
constexpr int PB_KN = 132;  // B smem pitch for [k][n] tiles (doubles)
constexpr int PB_NK = 20;   // B smem pitch for [n][k] tiles (doubles)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)),
               "l"(src), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

struct Fp64Args {
  int L, lmax, n, na, count, sgnCount, Q;  // Q = complex rows = sgnCount * count
  int nTheta, thetaPad, isReal;
  const long long* rowOff;   // table row offset per m
  const long long* opOff;    // operand offset per m (complex elements)
  const int* opPitch;        // operand row pitch per m (Kp_m)
  const double* table;
  const double2* A;          // inverse: operand [m][q][Kp_m]; forward: spec [m][q][thetaPad]
  double2* out;              // inverse: spec; forward: packed coefficients
  long coefSize;
  int mBegin, mCount;        // orders mBegin .. mBegin + mCount - 1 (a rank's share)
};

// kDir = 0: inverse (K = degree, N = colatitude; B tile [k][n] from the
// table rows). kDir = 1: forward (K = colatitude, N = degree; B tile [n][k]).
template <int kDir>
constexpr int kBTile = kDir == 0 ? BK * PB_KN : BN * PB_NK;

template <int kDir>
constexpr size_t fp64_smem_bytes() {
  return sizeof(double2) * STAGES * BMC * PA + sizeof(double) * STAGES * kBTile<kDir>;
}

template <int kDir>
__global__ void __launch_bounds__(256, 2) k_legendre_fp64(Fp64Args p) {
  extern __shared__ __align__(16) unsigned char fp64_smem[];
  auto As = reinterpret_cast<double2(*)[BMC * PA]>(fp64_smem);
  auto Bs = reinterpret_cast<double(*)[kBTile<kDir>]>(
      fp64_smem + sizeof(double2) * STAGES * BMC * PA);

  const int m = blockIdx.z + p.mBegin;
  const int l0 = m > p.na ? m : p.na;
  const int Keff = p.lmax - l0 + 1;            // degrees l0..lmax
  const int q0 = blockIdx.y * BMC;
  const int n0 = blockIdx.x * BN;
  const int ncols = kDir == 0 ? p.nTheta : Keff;
  if (n0 >= ncols) return;
  const int kTotal = kDir == 0 ? p.opPitch[m] : p.thetaPad;
  const long long tRow0 = p.rowOff[m];
  const double* T = p.table;
  const int tp = p.thetaPad;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wq = (warp >> 2) * 16;   // warp row offset (complex rows)
  const int wn = (warp & 3) * 32;    // warp column offset

  // A rows: inverse -> operand rows of length Kp_m; forward -> spec rows.
  const double2* Abase;
  long long aPitch;
  if (kDir == 0) {
    Abase = p.A + p.opOff[m];
    aPitch = p.opPitch[m];
  } else {
    Abase = p.A + (size_t)m * p.Q * tp;
    aPitch = tp;
  }

  auto load_stage = [&](int stage, int k0) {
    // A: BMC rows x BK double2 = 512 chunks of 16 B.
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int idx = tid + c * 256;
      const int r = idx >> 4, kk = idx & 15;
      const int q = q0 + r;
      const bool ok = q < p.Q;
      const double2* src = Abase + (size_t)(ok ? q : 0) * aPitch + k0 + kk;
      cp_async16(&As[stage][r * PA + kk], src, ok);
    }
    if (kDir == 0) {
      // B: BK table rows x BN colatitudes, 16 B chunks = 2 doubles.
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int idx = tid + c * 256;
        const int kr = idx >> 6, jj = (idx & 63) * 2;
        const double* src = T + (size_t)(tRow0 + k0 + kr) * tp + n0 + jj;
        cp_async16(&Bs[stage][kr * PB_KN + jj], src, true);
      }
    } else {
      // B: BN table rows (degrees) x BK colatitudes.
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int idx = tid + c * 256;
        const int nr = idx >> 3, kk = (idx & 7) * 2;
        const double* src = T + (size_t)(tRow0 + n0 + nr) * tp + k0 + kk;
        cp_async16(&Bs[stage][nr * PB_NK + kk], src, true);
      }
    }
  };

  double acc[2][2][4][2];  // [row group][re/im][col group][2]
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c][0] = acc[a][b][c][1] = 0.0;

  const int nk = kTotal / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nk) load_stage(s, s * BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int next = kt + STAGES - 1;
    if (next < nk) load_stage(next % STAGES, next * BK);
    cp_async_commit();
    const int st = kt % STAGES;
    const double2* as = As[st];
    const double* bs = Bs[st];
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      const int ka = k4 + (lane & 3);
      double2 af[2];
#pragma unroll
      for (int rg = 0; rg < 2; rg++) af[rg] = as[(wq + rg * 8 + (lane >> 2)) * PA + ka];
      double bf[4];
#pragma unroll
      for (int cg = 0; cg < 4; cg++) {
        const int nn = wn + cg * 8 + (lane >> 2);
        bf[cg] = kDir == 0 ? bs[ka * PB_KN + nn] : bs[nn * PB_NK + ka];
      }
#pragma unroll
      for (int rg = 0; rg < 2; rg++)
#pragma unroll
        for (int cg = 0; cg < 4; cg++) {
          dmma(acc[rg][0][cg][0], acc[rg][0][cg][1], af[rg].x, bf[cg]);
          dmma(acc[rg][1][cg][0], acc[rg][1][cg][1], af[rg].y, bf[cg]);
        }
    }
  }
  cp_async_wait<0>();

  // Epilogue: thread holds rows q = q0 + wq + rg*8 + lane/4 and columns
  // n = n0 + wn + cg*8 + 2*(lane%4) + {0,1}, with re and im together.
#pragma unroll
  for (int rg = 0; rg < 2; rg++) {
    const int q = q0 + wq + rg * 8 + (lane >> 2);
    if (q >= p.Q) continue;
    const int sgn = q / p.count, f = q - sgn * p.count;
#pragma unroll
    for (int cg = 0; cg < 4; cg++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int col = n0 + wn + cg * 8 + 2 * (lane & 3) + h;
        if (col >= ncols) continue;
        double2 v = make_double2(acc[rg][0][cg][h], acc[rg][1][cg][h]);
        if (kDir == 0) {
          p.out[((size_t)m * p.Q + q) * tp + col] = v;
        } else {
          if (sgn == 1 && m == 0) continue;
          const int l = l0 + col;
          if (sgn == 1 && ((l + p.n) & 1)) v = make_double2(-v.x, -v.y);
          long idx;
          if (p.isReal) {
            idx = (long)l * (l + 1) / 2 - (long)p.na * (p.na + 1) / 2 + m;
          } else {
            const int ms = sgn ? -m : m;
            idx = (long)l * l - (long)p.n * p.n + l + ms;
          }
          double2* o = p.out + (size_t)f * p.coefSize + idx;
          if (!p.isReal && sgn == 0 && m == p.L && l == p.L && p.lmax == p.L) {
            *o = make_double2(0.0, 0.0);  // GaussLegendreGrid.h:209-215
          } else {
            double2 c = *o;
            *o = make_double2(c.x + v.x, c.y + v.y);
          }
        }
      }
    }
  }
}

// Narrow batches (at most kStreamRows complex rows: one or two complex
// fields, up to four real ones): the contraction is a table-streaming GEMV,
// bound by HBM, so the table is read once with plain coalesced FP64 loads and
// FMAs on the CUDA cores instead of DMMA tiles whose rows would be mostly
// empty. Inverse: one thread per colatitude, the block's operand rows staged
// in shared memory 256 degrees at a time. Forward: one warp per 2 degree
// rows (each staged spectrum value feeds both), lanes across colatitudes, the
// spectra staged 32 KB (1024 colatitudes for one complex field) at a time,
// then a warp reduction. Chunk size and rows per warp were chosen by a sweep
// at lmax 2048: 256-colatitude chunks or 4 rows per warp ran 8-40% slower,
// reading the spectra from L1 instead of staging them 20% slower.
constexpr int kStreamRows = 4;

template <int kQ>
__global__ void __launch_bounds__(256) k_legendre_fp64_stream_inv(Fp64Args p) {
  __shared__ double2 As[kQ][256];
  const int m = blockIdx.y + p.mBegin;
  const int l0 = m > p.na ? m : p.na;
  const int K = p.lmax - l0 + 1;
  const int kp = p.opPitch[m];
  const int tid = threadIdx.x;
  const int j = blockIdx.x * 256 + tid;
  const int tp = p.thetaPad;
  const double2* A = p.A + p.opOff[m];
  const double* T = p.table + (size_t)p.rowOff[m] * tp + (j < tp ? j : 0);
  double2 acc[kQ];
#pragma unroll
  for (int q = 0; q < kQ; q++) acc[q] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < K; k0 += 256) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kQ; q++)
      As[q][tid] = (q < p.Q && k0 + tid < kp) ? A[(size_t)q * kp + k0 + tid] : make_double2(0.0, 0.0);
    __syncthreads();
    const int kn = K - k0 < 256 ? K - k0 : 256;
    if (j < p.nTheta) {
#pragma unroll 16
      for (int kk = 0; kk < kn; kk++) {
        const double t = __ldg(T + (size_t)(k0 + kk) * tp);
#pragma unroll
        for (int q = 0; q < kQ; q++) {
          acc[q].x = fma(t, As[q][kk].x, acc[q].x);
          acc[q].y = fma(t, As[q][kk].y, acc[q].y);
        }
      }
    }
  }
  if (j < p.nTheta) {
#pragma unroll
    for (int q = 0; q < kQ; q++)
      if (q < p.Q) p.out[((size_t)m * p.Q + q) * tp + j] = acc[q];
  }
}


constexpr int kFwdRowsPerWarp = 2;

template <int kQ>
__global__ void __launch_bounds__(256) k_legendre_fp64_stream_fwd(Fp64Args p) {
  constexpr int kChunk = 2048 / kQ;  // 32 KB of spectra per block
  __shared__ double2 Fs[kQ][kChunk];
  constexpr int kRowsPerWarp = kFwdRowsPerWarp;
  const int m = blockIdx.y + p.mBegin;
  const int l0 = m > p.na ? m : p.na;
  const int K = p.lmax - l0 + 1;
  const int kBlock = blockIdx.x * 8 * kRowsPerWarp;
  if (kBlock >= K) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tp = p.thetaPad;
  const int k0 = kBlock + warp * kRowsPerWarp;
  const double2* F = p.A + (size_t)m * p.Q * tp;
  double2 acc[kRowsPerWarp][kQ];
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; r++)
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[r][q] = make_double2(0.0, 0.0);
  // The warp's rows past the end re-read its last valid row (never stored),
  // so the rows' loads are issued together without a branch.
  const bool active = k0 < K;
  const double* T[kRowsPerWarp];
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; r++)
    T[r] = p.table + (size_t)(p.rowOff[m] + (k0 + r < K ? k0 + r : K - 1)) * tp;
  for (int j0 = 0; j0 < tp; j0 += kChunk) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kQ; q++)
      for (int u = tid; u < kChunk; u += 256)
        Fs[q][u] = (q < p.Q && j0 + u < tp) ? F[(size_t)q * tp + j0 + u] : make_double2(0.0, 0.0);
    __syncthreads();
    if (!active) continue;
    const int jn = tp - j0 < kChunk ? tp - j0 : kChunk;
#pragma unroll 4
    for (int jj = lane; jj < jn; jj += 32) {
      double t[kRowsPerWarp];
#pragma unroll
      for (int r = 0; r < kRowsPerWarp; r++) t[r] = __ldg(T[r] + j0 + jj);
#pragma unroll
      for (int q = 0; q < kQ; q++) {
        const double2 f = Fs[q][jj];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; r++) {
          acc[r][q].x = fma(t[r], f.x, acc[r][q].x);
          acc[r][q].y = fma(t[r], f.y, acc[r][q].y);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; r++)
#pragma unroll
    for (int q = 0; q < kQ; q++)
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        acc[r][q].x += __shfl_xor_sync(0xffffffffu, acc[r][q].x, o);
        acc[r][q].y += __shfl_xor_sync(0xffffffffu, acc[r][q].y, o);
      }
  if (lane != 0) return;
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; r++) {
    const int k = k0 + r;
    if (k >= K) break;
    const int l = l0 + k;
#pragma unroll
    for (int q = 0; q < kQ; q++) {
      if (q >= p.Q) break;
      const int sgn = q / p.count, f = q - sgn * p.count;
      if (sgn == 1 && m == 0) continue;
      double2 v = acc[r][q];
      if (sgn == 1 && ((l + p.n) & 1)) v = make_double2(-v.x, -v.y);
      const long idx = p.isReal ? (long)l * (l + 1) / 2 - (long)p.na * (p.na + 1) / 2 + m
                                : (long)l * l - (long)p.n * p.n + l + (sgn ? -m : m);
      double2* o = p.out + (size_t)f * p.coefSize + idx;
      if (!p.isReal && sgn == 0 && m == p.L && l == p.L && p.lmax == p.L) {
        *o = make_double2(0.0, 0.0);  // GaussLegendreGrid.h:209-215
      } else {
        const double2 c = *o;
        *o = make_double2(c.x + v.x, c.y + v.y);
      }
    }
  }
}

// Launches the inverse contraction: the streaming kernel for narrow batches,
// the DMMA tiles otherwise.
gsht_status launch_inverse_fp64(const gsht_grid* g, const Fp64Args& a, cudaStream_t s) {
  if (a.Q <= kStreamRows) {
    dim3 grid((g->n_theta + 255) / 256, a.mCount);
    if (a.Q <= 1) k_legendre_fp64_stream_inv<1><<<grid, 256, 0, s>>>(a);
    else if (a.Q <= 2) k_legendre_fp64_stream_inv<2><<<grid, 256, 0, s>>>(a);
    else k_legendre_fp64_stream_inv<4><<<grid, 256, 0, s>>>(a);
    GSHT_LAUNCH_CHECK("k_legendre_fp64_stream_inv");
    return GSHT_OK;
  }
  dim3 grid((g->n_theta + BN - 1) / BN, (a.Q + BMC - 1) / BMC, a.mCount);
  GSHT_CUDA(cudaFuncSetAttribute(k_legendre_fp64<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fp64_smem_bytes<0>()));
  k_legendre_fp64<0><<<grid, 256, fp64_smem_bytes<0>(), s>>>(a);
  GSHT_LAUNCH_CHECK("k_legendre_fp64<inverse>");
  return GSHT_OK;
}

// Packed coefficients -> per-order operand rows (inverse A operand):
// op[m][q = sgn*count + f][k] = c_{l0+k, +/-m} * ((-1)^{l+n} for -m), zero
// for l > lmax and in the padding.
__global__ void k_prep_inverse_fp64(int lmax, int n, int na, int count,
                                    int sgnCount, int isReal, long coefSize,
                                    const double2* __restrict__ coef,
                                    const long long* __restrict__ opOff,
                                    const int* __restrict__ opPitch,
                                    double2* __restrict__ op, int mBegin) {
  const int m = blockIdx.y + mBegin;
  const int q = blockIdx.z;
  const int sgn = q / count, f = q - sgn * count;
  const int l0 = m > na ? m : na;
  const int kp = opPitch[m];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kp) return;
  const int l = l0 + k;
  double2 v = make_double2(0.0, 0.0);
  if (l <= lmax && !(sgn == 1 && m == 0)) {
    long idx;
    if (isReal) {
      idx = (long)l * (l + 1) / 2 - (long)na * (na + 1) / 2 + m;
    } else {
      idx = (long)l * l - (long)n * n + l + (sgn ? -m : m);
    }
    v = coef[(size_t)f * coefSize + idx];
    if (sgn == 1 && ((l + n) & 1)) v = make_double2(-v.x, -v.y);
  }
  op[opOff[m] + (size_t)q * kp + k] = v;
}

}  // namespace

const OperandLayout* operand_layout(const gsht_grid* g, int lmax, int na,
                                    int rows, int pad, gsht_status* st) {
  *st = GSHT_OK;
  for (auto* o : g->layouts)
    if (o->lmax == lmax && o->na == na && o->rows == rows && o->pad == pad) return o;
  auto* o = new OperandLayout();
  o->lmax = lmax; o->na = na; o->rows = rows; o->pad = pad;
  o->off.resize(lmax + 2);
  o->pitch.resize(lmax + 1);
  long long acc = 0;
  for (int m = 0; m <= lmax; m++) {
    const int l0 = m > na ? m : na;
    o->pitch[m] = (int)round_up(lmax - l0 + 1, pad);
    o->pitch_max = o->pitch[m] > o->pitch_max ? o->pitch[m] : o->pitch_max;
    o->off[m] = acc;
    acc += (long long)o->pitch[m] * rows;
  }
  o->off[lmax + 1] = acc;
  o->total = acc;
  if (dev_malloc(&o->d_off, sizeof(long long) * o->off.size()) != cudaSuccess ||
      dev_malloc(&o->d_pitch, sizeof(int) * o->pitch.size()) != cudaSuccess ||
      cudaMemcpy(o->d_off, o->off.data(), sizeof(long long) * o->off.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(o->d_pitch, o->pitch.data(), sizeof(int) * o->pitch.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    dev_free(o->d_off);
    dev_free(o->d_pitch);
    delete o;
    *st = fail(GSHT_ERR_OOM, "operand layout allocation failed");
    return nullptr;
  }
  g->layouts.push_back(o);
  return o;
}

void free_layouts(gsht_grid* g) {
  for (auto* o : g->layouts) {
    dev_free(o->d_off);
    dev_free(o->d_pitch);
    delete o;
  }
  g->layouts.clear();
  for (auto* t : g->tile_lists) {
    dev_free(t->d_tiles);
    delete t;
  }
  g->tile_lists.clear();
}

gsht_status fp64_operand_elems(const gsht_grid* g, const Table* t, int lmax, int is_real,
                               int count, size_t* elems) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count;
  gsht_status st;
  const OperandLayout* o = operand_layout(g, lmax, na, Q, kDegreePadFp64, &st);
  *elems = o ? (size_t)o->total : 0;
  return st;
}

gsht_status prep_inverse_fp64(const gsht_grid* g, const Table* t, int lmax, int is_real,
                              int count, const double* coef, double* operand,
                              const OperandLayout** layout, cudaStream_t s, int mBegin,
                              int mEnd) {
  if (mEnd < 0 || mEnd > lmax + 1) mEnd = lmax + 1;
  const int na = t->n < 0 ? -t->n : t->n;
  const int sgnCount = is_real ? 1 : 2;
  const int Q = sgnCount * count;
  gsht_status st;
  const OperandLayout* lay = operand_layout(g, lmax, na, Q, kDegreePadFp64, &st);
  if (!lay) return st;
  *layout = lay;
  StageTimer tm(GSHT_STAGE_PREP_INVERSE, s);
  if (mBegin >= mEnd) return GSHT_OK;
  dim3 pg((lay->pitch_max + 127) / 128, mEnd - mBegin, Q);
  k_prep_inverse_fp64<<<pg, 128, 0, s>>>(lmax, t->n, na, count, sgnCount, is_real,
                                         coef_size(lmax, t->n, is_real),
                                         reinterpret_cast<const double2*>(coef), lay->d_off,
                                         lay->d_pitch, reinterpret_cast<double2*>(operand),
                                         mBegin);
  GSHT_LAUNCH_CHECK("k_prep_inverse_fp64");
  return GSHT_OK;
}

gsht_status legendre_inverse_fp64(const gsht_grid* g, const Table* t, int lmax,
                                  int is_real, int count, const double* coef,
                                  double* operand, double* spec,
                                  cudaStream_t s, int mBegin, int mEnd) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int sgnCount = is_real ? 1 : 2;
  const int Q = sgnCount * count;
  if (mEnd < 0 || mEnd > lmax + 1) mEnd = lmax + 1;
  if (mBegin >= mEnd) return GSHT_OK;
  const OperandLayout* lay = nullptr;
  gsht_status st =
      prep_inverse_fp64(g, t, lmax, is_real, count, coef, operand, &lay, s, mBegin, mEnd);
  if (st != GSHT_OK) return st;
  Fp64Args a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count;
  a.sgnCount = sgnCount; a.Q = Q; a.nTheta = g->n_theta; a.thetaPad = g->theta_pad;
  a.isReal = is_real; a.rowOff = t->d_row_off; a.opOff = lay->d_off; a.opPitch = lay->d_pitch;
  a.table = t->t64; a.A = reinterpret_cast<double2*>(operand);
  a.out = reinterpret_cast<double2*>(spec);
  a.coefSize = coef_size(lmax, t->n, is_real);
  a.mBegin = mBegin;
  a.mCount = mEnd - mBegin;
  StageTimer tm(GSHT_STAGE_LEGENDRE_INVERSE, s);
  return launch_inverse_fp64(g, a, s);
}

gsht_status legendre_forward_fp64(const gsht_grid* g, const Table* t, int lmax,
                                  int is_real, int count, const double* spec,
                                  double* coef, cudaStream_t s, int mBegin, int mEnd) {
  if (mEnd < 0 || mEnd > lmax + 1) mEnd = lmax + 1;
  if (mBegin >= mEnd) return GSHT_OK;
  const int na = t->n < 0 ? -t->n : t->n;
  const int sgnCount = is_real ? 1 : 2;
  const int Q = sgnCount * count;
  Fp64Args a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count;
  a.sgnCount = sgnCount; a.Q = Q; a.nTheta = g->n_theta; a.thetaPad = g->theta_pad;
  a.isReal = is_real; a.rowOff = t->d_row_off; a.opOff = nullptr; a.opPitch = nullptr;
  a.table = t->t64; a.A = reinterpret_cast<const double2*>(spec);
  a.out = reinterpret_cast<double2*>(coef);
  a.coefSize = coef_size(lmax, t->n, is_real);
  a.mBegin = mBegin;
  a.mCount = mEnd - mBegin;
  const int kMax = lmax - na + 1;
  if (Q <= kStreamRows) {
    dim3 sg((kMax + 8 * kFwdRowsPerWarp - 1) / (8 * kFwdRowsPerWarp), a.mCount);
    if (Q <= 1) k_legendre_fp64_stream_fwd<1><<<sg, 256, 0, s>>>(a);
    else if (Q <= 2) k_legendre_fp64_stream_fwd<2><<<sg, 256, 0, s>>>(a);
    else k_legendre_fp64_stream_fwd<4><<<sg, 256, 0, s>>>(a);
    GSHT_LAUNCH_CHECK("k_legendre_fp64_stream_fwd");
    return GSHT_OK;
  }
  dim3 grid((kMax + BN - 1) / BN, (Q + BMC - 1) / BMC, a.mCount);
  GSHT_CUDA(cudaFuncSetAttribute(k_legendre_fp64<1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fp64_smem_bytes<1>()));
  k_legendre_fp64<1><<<grid, 256, fp64_smem_bytes<1>(), s>>>(a);
  GSHT_LAUNCH_CHECK("k_legendre_fp64<forward>");
  return GSHT_OK;
}

}  // namespace gsht

namespace gsht {

// The inverse contraction of legendre_inverse_fp64 with an operand layout the
// caller already placed in device memory (off/pitch as in OperandLayout) and
// without stage timers: launches only the two kernels, allocates nothing.
gsht_status legendre_inverse_fp64_layout(const gsht_grid* g, const Table* t, int lmax,
                                         int is_real, int count, const double* coef,
                                         const long long* dOff, const int* dPitch, int kpMax,
                                         double* operand, double* spec, cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int sgnCount = is_real ? 1 : 2;
  const int Q = sgnCount * count;
  double2* op = reinterpret_cast<double2*>(operand);
  const long cs = coef_size(lmax, t->n, is_real);
  dim3 pg((kpMax + 127) / 128, lmax + 1, Q);
  k_prep_inverse_fp64<<<pg, 128, 0, s>>>(lmax, t->n, na, count, sgnCount, is_real, cs,
                                         reinterpret_cast<const double2*>(coef), dOff, dPitch,
                                         op, 0);
  GSHT_LAUNCH_CHECK("k_prep_inverse_fp64");
  Fp64Args a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count;
  a.sgnCount = sgnCount; a.Q = Q; a.nTheta = g->n_theta; a.thetaPad = g->theta_pad;
  a.isReal = is_real; a.rowOff = t->d_row_off; a.opOff = dOff; a.opPitch = dPitch;
  a.table = t->t64; a.A = op; a.out = reinterpret_cast<double2*>(spec);
  a.coefSize = cs;
  a.mBegin = 0;
  a.mCount = lmax + 1;
  return launch_inverse_fp64(g, a, s);
}

}  // namespace gsht
