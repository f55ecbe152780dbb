// Legendre stage in the Ozaki form: INT8 slices on the tcgen05 tensor cores
// (kind::i8) with exact INT32 accumulation in TMEM and an FP64 recombination
// epilogue.
//
// Same contraction and operand roles as legendre_tc.cu (GaussLegendreGrid.h
// :176-207 forward, :284-312 inverse). Each operand x is written as
// x = 2^e sum_{s=0..6} S_s 2^{-7(s+1)} with S_s in [-127, 127] and one
// power-of-two scale per table column (m, theta_j) and per field row; the
// 28 slice products S^A_i S^B_j with i + j <= 6 are accumulated exactly in
// INT32, one TMEM accumulator per diagonal d = i + j (7 x 64 columns), and
// combined in FP64 as sum_d 2^{-7(d+2)} acc_d times the two scales. Dropped
// products are below 2^-56 of the operands' scales.
//
// Table scale folding: in the inverse the table scale belongs to an output
// row (colatitude) and is applied in the epilogue; in the forward it runs
// along the contraction and is folded into the field-side rows before they
// are sliced.
#include <cstdio>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

using namespace tc;

constexpr int kBM = 128;  // tile rows (TMEM lanes)
constexpr int kN = 64;    // field rows per tile
constexpr int kBK = 64;   // K (bytes) per stage
constexpr int kS = kTableSlices;            // 7 slices per operand
constexpr int kNDiag = kS;                  // diagonals d = 0..6
constexpr int kTileA = kBM * kBK;           // 8 KB per slice
constexpr int kTileB = kN * kBK;            // 4 KB per slice
constexpr int kStageBytes = kS * (kTileA + kTileB);  // 84 KB
constexpr int kStages = 2;
constexpr int kTmemCols = 512;
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024 + 256;

struct OzArgs {
  int L, lmax, n, na, count, Q, R, nTheta, thetaPad, isReal;
  const long long* rowOff;
  const int* tabExp;  // [m][thetaPad] table column exponents
  const int* rowExp;  // [m * R + r] field row exponents
  double2* out;
  long coefSize;
  int* err;
};

template <int kDir>
__global__ void __launch_bounds__(192, 1)
    k_legendre_oz(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB, OzArgs p) {
  extern __shared__ __align__(1024) unsigned char oz_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(oz_smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accBar = empty + kStages;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(accBar + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mtile = blockIdx.x, ntile = blockIdx.y, m = blockIdx.z;
  const int l0 = m > p.na ? m : p.na;
  const int Keff = p.lmax - l0 + 1;
  const int rowsM = kDir == 0 ? p.nTheta : Keff;
  if (mtile * kBM >= rowsM) return;
  __shared__ int skip;
  if (threadIdx.x == 0) skip = *reinterpret_cast<volatile int*>(p.err);
  __syncthreads();
  if (skip) return;
  const int nk = kDir == 0 ? (Keff + kBK - 1) / kBK : (p.thetaPad + kBK - 1) / kBK;
  const long long tRow = p.rowOff[m];
  const int bRow = m * p.R + ntile * kN;

  if (warp == 0 && lane == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accBar, 1);
    fence_barrier_init();
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
  }
  if (warp == 1) tmem_alloc(tmemSlot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmemSlot;

  if (warp == 0) {
    if (lane == 0) {
      for (int kc = 0; kc < nk; kc++) {
        const int s = kc % kStages;
        if (kc >= kStages && !mbar_wait(&empty[s], ((kc / kStages) - 1) & 1, p.err, 11)) break;
        unsigned char* st = smem + s * kStageBytes;
        mbar_arrive_expect_tx(&full[s], kStageBytes);
        for (int a = 0; a < kS; a++) {
          if (kDir == 0) {
            // MN-major: 128 colatitudes (one 128 B row) x 64 degree rows.
            tma_load_3d(st + a * kTileA, &mapA, &full[s], mtile * kBM, (int)(tRow + kc * kBK), a);
          } else {
            tma_load_3d(st + a * kTileA, &mapA, &full[s], kc * kBK, (int)(tRow + mtile * kBM), a);
          }
        }
        for (int b = 0; b < kS; b++)
          tma_load_3d(st + kS * kTileA + b * kTileB, &mapB, &full[s], kc * kBK, bRow, b);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t id = idesc(2, 1, kDir == 0 ? 1 : 0, 0, kN, kBM);
      for (int kc = 0; kc < nk; kc++) {
        const int s = kc % kStages;
        if (!mbar_wait(&full[s], (kc / kStages) & 1, p.err, 12)) break;
        tc_fence_after();
        const uint32_t st = smem_u32(smem + s * kStageBytes);
#pragma unroll
        for (int i = 0; i < kS; i++) {
#pragma unroll
          for (int j = 0; i + j < kS; j++) {
            const uint32_t aBase = st + i * kTileA;
            const uint32_t bBase = st + kS * kTileA + j * kTileB;
            const uint32_t d = tmem + (uint32_t)((i + j) * kN);
#pragma unroll
            for (int k32 = 0; k32 < kBK / 32; k32++) {
              const uint64_t ad = kDir == 0 ? sdesc_sw128(aBase + k32 * 4096, 8192, 1024)
                                            : sdesc_sw64(aBase + k32 * 32, 16, 512);
              const uint64_t bd = sdesc_sw64(bBase + k32 * 32, 16, 512);
              mma_i8(d, ad, bd, id, (kc | i | k32) != 0);
            }
          }
        }
        mma_commit(&empty[s]);
      }
      mma_commit(accBar);
    }
  } else {
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const bool ready = mbar_wait(accBar, 0, p.err, 13);
    tc_fence_after();
    if (ready) {
      const int tileRow = mtile * kBM + row;
      const bool live = tileRow < rowsM;
      const int eA = (kDir == 0 && live) ? p.tabExp[(size_t)m * p.thetaPad + tileRow] : 0;
#pragma unroll 1
      for (int c = 0; c < kN / 16; c++) {
        double acc[16];
#pragma unroll
        for (int i = 0; i < 16; i++) acc[i] = 0.0;
#pragma unroll 1
        for (int d = 0; d < kNDiag; d++) {
          uint32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + d * kN + c * 16, v);
          tmem_wait_ld();
          const double w = ldexp(1.0, -7 * (d + 2));
#pragma unroll
          for (int i = 0; i < 16; i++) acc[i] = fma((double)(int)v[i], w, acc[i]);
        }
        if (!live) continue;
        const int r0 = ntile * kN + c * 16;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int q = r0 / 2 + i;
          if (q >= p.Q) break;
          const int ere = p.rowExp[(size_t)m * p.R + 2 * q];
          const int eim = p.rowExp[(size_t)m * p.R + 2 * q + 1];
          double2 val = make_double2(ldexp(acc[2 * i], eA + ere), ldexp(acc[2 * i + 1], eA + eim));
          if (kDir == 0) {
            p.out[((size_t)m * p.Q + q) * p.thetaPad + tileRow] = val;
          } else {
            const int sgn = q / p.count, f = q - sgn * p.count;
            if (sgn == 1 && m == 0) continue;
            const int l = l0 + tileRow;
            if (sgn == 1 && ((l + p.n) & 1)) val = make_double2(-val.x, -val.y);
            long idx;
            if (p.isReal) {
              idx = (long)l * (l + 1) / 2 - (long)p.na * (p.na + 1) / 2 + m;
            } else {
              idx = (long)l * l - (long)p.n * p.n + l + (sgn ? -m : m);
            }
            double2* o = p.out + (size_t)f * p.coefSize + idx;
            if (!p.isReal && sgn == 0 && m == p.L && l == p.L && p.lmax == p.L) {
              *o = make_double2(0.0, 0.0);
            } else {
              const double2 c0 = *o;
              *o = make_double2(c0.x + val.x, c0.y + val.y);
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// Field-side slicing: one warp per (m, complex row q) handles the re and im
// real rows 2q, 2q+1: row maxima -> exponents -> 7 truncation slices.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ void write_slices(double y, int8_t* dst, size_t plane) {
#pragma unroll
  for (int s = 0; s < kS; s++) {
    y *= 128.0;
    const double q = trunc(y);
    y -= q;
    dst[s * plane] = (int8_t)q;
  }
}

// Inverse: packed coefficients -> slices over degrees, K pitch `pitch`.
__global__ void k_prep_inverse_oz(int lmax, int n, int na, int count, int Q, int R, int isReal,
                                  long coefSize, int pitch, size_t plane,
                                  const double2* __restrict__ coef, int8_t* __restrict__ op,
                                  int* __restrict__ rowExp) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (wid >= (lmax + 1) * Q) return;
  const int m = wid / Q, q = wid - m * Q;
  const int sgn = q / count, f = q - sgn * count;
  const int l0 = m > na ? m : na;
  const int keff = lmax - l0 + 1;
  const int kp = (keff + kBK - 1) / kBK * kBK;
  auto value = [&](int k) {
    double2 v = make_double2(0.0, 0.0);
    const int l = l0 + k;
    if (k < keff && !(sgn == 1 && m == 0)) {
      const long idx = isReal ? (long)l * (l + 1) / 2 - (long)na * (na + 1) / 2 + m
                              : (long)l * l - (long)n * n + l + (sgn ? -m : m);
      v = coef[(size_t)f * coefSize + idx];
      if (sgn == 1 && ((l + n) & 1)) v = make_double2(-v.x, -v.y);
    }
    return v;
  };
  double mre = 0.0, mim = 0.0;
  for (int k = lane; k < keff; k += 32) {
    const double2 v = value(k);
    mre = fmax(mre, fabs(v.x));
    mim = fmax(mim, fabs(v.y));
  }
  mre = warp_max(mre);
  mim = warp_max(mim);
  int ere = 0, eim = 0;
  if (mre > 0.0) frexp(mre, &ere);
  if (mim > 0.0) frexp(mim, &eim);
  const size_t r0 = ((size_t)m * R + 2 * q) * pitch;
  if (lane == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  for (int k = lane; k < kp; k += 32) {
    const double2 v = value(k);
    write_slices(ldexp(v.x, -ere), op + r0 + k, plane);
    write_slices(ldexp(v.y, -eim), op + r0 + pitch + k, plane);
  }
}

// Forward: weighted spectra times the table column scales -> slices over
// colatitudes (pitch thetaPad).
__global__ void k_prep_forward_oz(int lmax, int Q, int R, int thetaPad, size_t plane,
                                  const double2* __restrict__ spec,
                                  const int* __restrict__ tabExp, int8_t* __restrict__ op,
                                  int* __restrict__ rowExp) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (wid >= (lmax + 1) * Q) return;
  const int m = wid / Q, q = wid - m * Q;
  const double2* row = spec + ((size_t)m * Q + q) * thetaPad;
  const int* te = tabExp + (size_t)m * thetaPad;
  double mre = 0.0, mim = 0.0;
  for (int j = lane; j < thetaPad; j += 32) {
    const double2 v = row[j];
    mre = fmax(mre, fabs(ldexp(v.x, te[j])));
    mim = fmax(mim, fabs(ldexp(v.y, te[j])));
  }
  mre = warp_max(mre);
  mim = warp_max(mim);
  int ere = 0, eim = 0;
  if (mre > 0.0) frexp(mre, &ere);
  if (mim > 0.0) frexp(mim, &eim);
  if (lane == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  const size_t r0 = ((size_t)m * R + 2 * q) * thetaPad;
  for (int j = lane; j < thetaPad; j += 32) {
    const double2 v = row[j];
    write_slices(ldexp(v.x, te[j] - ere), op + r0 + j, plane);
    write_slices(ldexp(v.y, te[j] - eim), op + r0 + thetaPad + j, plane);
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
    else
      cudaGetLastError();
  }
  return fn;
}

// 3-D byte tensor [planes][rows][inner] with a [1][boxRows][boxInner] box.
gsht_status make_map_i8(CUtensorMap* map, const void* base, uint64_t inner, uint64_t rows,
                        uint64_t planes, uint64_t rowPitch, uint64_t planeBytes,
                        uint32_t boxInner, uint32_t boxRows, CUtensorMapSwizzle sw) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {inner, rows, planes};
  cuuint64_t strides[2] = {rowPitch, planeBytes};
  cuuint32_t box[3] = {boxInner, boxRows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return GSHT_OK;
}

template <int kDir>
gsht_status launch_oz(const OzArgs& a, const CUtensorMap& mapA, const CUtensorMap& mapB,
                      int gridX, cudaStream_t s) {
  auto kern = k_legendre_oz<kDir>;
  GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemBytes));
  dim3 grid(gridX, (a.R + kN - 1) / kN, a.lmax + 1);
  kern<<<grid, 192, kSmemBytes, s>>>(mapA, mapB, a);
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_oz<inverse>" : "k_legendre_oz<forward>");
  return GSHT_OK;
}

}  // namespace

size_t oz_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir) {
  const int R = 2 * (is_real ? 1 : 2) * count;
  const long long pitch = dir == 0 ? g->theta_pad : round_up(lmax + 1, kBK);
  return (size_t)kS * (lmax + 1) * R * pitch + sizeof(int) * (size_t)(lmax + 1) * R + 256;
}

gsht_status legendre_inverse_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, const double* coef, void* operand, double* spec,
                                cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int pitch = (int)round_up(lmax + 1, kBK);
  const size_t plane = (size_t)(lmax + 1) * R * pitch;
  auto* op = static_cast<int8_t*>(operand);
  int* rowExp = reinterpret_cast<int*>(static_cast<char*>(operand) + round_up(kS * plane, 256));
  {
    StageTimer tm(GSHT_STAGE_PREP_INVERSE, s);
    const long long warps = (long long)(lmax + 1) * Q;
    k_prep_inverse_oz<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
        lmax, t->n, na, count, Q, R, is_real, coef_size(lmax, t->n, is_real), pitch, plane,
        reinterpret_cast<const double2*>(coef), op, rowExp);
    GSHT_LAUNCH_CHECK("k_prep_inverse_oz");
  }
  CUtensorMap mapA, mapB;
  const size_t tplane = (size_t)(t->rows + kTablePadRows) * g->theta_pad;
  gsht_status st = make_map_i8(&mapA, t->ti8, g->theta_pad, t->rows + kTablePadRows, kS,
                               g->theta_pad, tplane, 128, 64, CU_TENSOR_MAP_SWIZZLE_128B);
  if (st != GSHT_OK) return st;
  st = make_map_i8(&mapB, op, pitch, (uint64_t)(lmax + 1) * R, kS, pitch, plane, 64, kN,
                   CU_TENSOR_MAP_SWIZZLE_64B);
  if (st != GSHT_OK) return st;
  OzArgs a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count; a.Q = Q; a.R = R;
  a.nTheta = g->n_theta; a.thetaPad = g->theta_pad; a.isReal = is_real;
  a.rowOff = t->d_row_off; a.tabExp = t->i8_exp; a.rowExp = rowExp;
  a.out = reinterpret_cast<double2*>(spec);
  a.coefSize = coef_size(lmax, t->n, is_real); a.err = g->d_err;
  StageTimer tm(GSHT_STAGE_LEGENDRE_INVERSE, s);
  return launch_oz<0>(a, mapA, mapB, (g->n_theta + kBM - 1) / kBM, s);
}

gsht_status legendre_forward_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, const double* spec, void* operand, double* coef,
                                cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int tp = g->theta_pad;
  const size_t plane = (size_t)(lmax + 1) * R * tp;
  auto* op = static_cast<int8_t*>(operand);
  int* rowExp = reinterpret_cast<int*>(static_cast<char*>(operand) + round_up(kS * plane, 256));
  {
    StageTimer tm(GSHT_STAGE_PREP_FORWARD, s);
    const long long warps = (long long)(lmax + 1) * Q;
    k_prep_forward_oz<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
        lmax, Q, R, tp, plane, reinterpret_cast<const double2*>(spec), t->i8_exp, op, rowExp);
    GSHT_LAUNCH_CHECK("k_prep_forward_oz");
  }
  CUtensorMap mapA, mapB;
  const size_t tplane = (size_t)(t->rows + kTablePadRows) * tp;
  gsht_status st = make_map_i8(&mapA, t->ti8, tp, t->rows + kTablePadRows, kS, tp, tplane, 64,
                               kBM, CU_TENSOR_MAP_SWIZZLE_64B);
  if (st != GSHT_OK) return st;
  st = make_map_i8(&mapB, op, tp, (uint64_t)(lmax + 1) * R, kS, tp, plane, 64, kN,
                   CU_TENSOR_MAP_SWIZZLE_64B);
  if (st != GSHT_OK) return st;
  OzArgs a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count; a.Q = Q; a.R = R;
  a.nTheta = g->n_theta; a.thetaPad = tp; a.isReal = is_real;
  a.rowOff = t->d_row_off; a.tabExp = t->i8_exp; a.rowExp = rowExp;
  a.out = reinterpret_cast<double2*>(coef);
  a.coefSize = coef_size(lmax, t->n, is_real); a.err = g->d_err;
  const int kMax = lmax - na + 1;
  StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
  return launch_oz<1>(a, mapA, mapB, (kMax + kBM - 1) / kBM, s);
}

}  // namespace gsht
