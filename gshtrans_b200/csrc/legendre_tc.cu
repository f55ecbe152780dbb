// Legendre stage on the 5th-generation tensor cores (tcgen05, TMEM, TMA).
//
// Replaces the same theta-loop accumulations as legendre_fp64.cu
// (GaussLegendreGrid.h:176-207 forward, :284-312 inverse) with per-order
// GEMM tiles:
//   inverse  D[theta][r] = sum_k T[row_m + k][theta] * B[r][k]   (A MN-major)
//   forward  D[k][r]     = sum_j T[row_m + k][j]     * B[r][j]   (A K-major)
// The table T is operand A (M = 128 colatitudes or degrees per tile), the
// batch's field rows (r = 2 q + re/im, q = sign x field) are operand B
// (N = 128). In the BF16x3 form both operands are split into hi/mid/lo BF16
// planes and six split products (hi.hi, hi.mid, mid.hi, hi.lo, lo.hi,
// mid.mid) accumulate in FP32 in TMEM.
//
// Warp roles (192 threads): warp 0 issues TMA loads, warp 1 owns TMEM and
// issues MMAs from one lane, warps 2-5 drain TMEM in the epilogue. Every
// mbarrier wait is bounded (tc_common.cuh) and reports a timeout through
// the grid's device error word instead of hanging.
#include <cstdio>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

using namespace tc;

constexpr int kBM = 128;       // tile rows (TMEM lanes)
constexpr int kBK = 64;        // K per stage: 64 x 2 B = one 128 B swizzle row
constexpr int kTileA = kBM * kBK * 2;  // bytes per A split tile (16 KB)

struct TcArgs {
  int L, lmax, n, na, count, Q, R, nTheta, thetaPad, isReal;
  const long long* rowOff;
  double2* out;
  long coefSize;
  int* err;
};

// TMEM accumulators per tile: products of very different magnitude would
// otherwise share one FP32 accumulator whose every update truncates; hi.hi
// goes to up to kBigAcc accumulators by K block and the other five products to
// a separate one, all summed in FP64 in the epilogue (4 x 128 = 512 columns).
constexpr int kBigAcc = 3;
constexpr int kAccumulators = kBigAcc + 1;

// Products of the BF16x3 form: (A split, B split).
__host__ __device__ constexpr int prodA(int p) { return p == 0 ? 0 : p == 1 ? 0 : p == 2 ? 1 : p == 3 ? 0 : p == 4 ? 2 : 1; }
__host__ __device__ constexpr int prodB(int p) { return p == 0 ? 0 : p == 1 ? 1 : p == 2 ? 0 : p == 3 ? 2 : p == 4 ? 0 : 1; }

template <int kNA, int kNB, int kN, int kStages>
constexpr size_t tc_smem_bytes() {
  return (size_t)kStages * (kNA * kTileA + kNB * kN * kBK * 2) + 1024 + 256;
}

template <int kDir, int kNA, int kNB, int kNP, int kN, int kStages>
__global__ void __launch_bounds__(192, 1)
    k_legendre_tc(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB, TcArgs p) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  // 1024-byte alignment for the swizzled tiles.
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int kTileB = kN * kBK * 2;
  constexpr int kStageBytes = kNA * kTileA + kNB * kTileB;
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
  if (threadIdx.x == 0) skip = *reinterpret_cast<volatile int*>(p.err);  // an earlier block timed out
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
  if (warp == 1) tmem_alloc(tmemSlot, kAccumulators * kN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmemSlot;

  if (warp == 0) {
    if (lane == 0) {
      for (int kc = 0; kc < nk; kc++) {
        const int s = kc % kStages;
        if (kc >= kStages && !mbar_wait(&empty[s], ((kc / kStages) - 1) & 1, p.err, 1)) break;
        unsigned char* st = smem + s * kStageBytes;
        mbar_arrive_expect_tx(&full[s], kStageBytes);
        for (int a = 0; a < kNA; a++) {
          unsigned char* dst = st + a * kTileA;
          if (kDir == 0) {
            // MN-major: two 64-colatitude halves of 64 degree rows each.
            tma_load_3d(dst, &mapA, &full[s], mtile * kBM, (int)(tRow + kc * kBK), a);
            tma_load_3d(dst + kTileA / 2, &mapA, &full[s], mtile * kBM + 64, (int)(tRow + kc * kBK), a);
          } else {
            tma_load_3d(dst, &mapA, &full[s], kc * kBK, (int)(tRow + mtile * kBM), a);
          }
        }
        for (int b = 0; b < kNB; b++)
          tma_load_3d(st + kNA * kTileA + b * kTileB, &mapB, &full[s], kc * kBK, bRow, b);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t id = idesc(1, 1, kDir == 0 ? 1 : 0, 0, kN, kBM);
      // hi.hi products go to one of nbig accumulators by K block; the five
      // smaller products share accumulator 0 (see kAccumulators).
      const int nbig = nk < kBigAcc ? nk : kBigAcc;
      bool ok = true;
      for (int kc = 0; kc < nk && ok; kc++) {
        const int s = kc % kStages;
        if (!mbar_wait(&full[s], (kc / kStages) & 1, p.err, 2)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int big = 1 + (kc * nbig) / nk;
        const int bigFirst = ((big - 1) * nk + nbig - 1) / nbig;
        const uint32_t st = smem_u32(smem + s * kStageBytes);
#pragma unroll
        for (int pr = 0; pr < kNP; pr++) {
          const uint32_t aBase = st + prodA(pr) * kTileA;
          const uint32_t bBase = st + kNA * kTileA + prodB(pr) * kTileB;
          const uint32_t d = tmem + (uint32_t)((pr == 0 ? big : 0) * kN);
#pragma unroll
          for (int k16 = 0; k16 < kBK / 16; k16++) {
            const uint64_t ad = kDir == 0 ? sdesc_sw128(aBase + k16 * 2048, kTileA / 2, 1024)
                                          : sdesc_sw128(aBase + k16 * 32, 16, 1024);
            const uint64_t bd = sdesc_sw128(bBase + k16 * 32, 16, 1024);
            const bool first = pr == 0 ? (kc == bigFirst && k16 == 0)
                                       : (kc == 0 && k16 == 0 && pr == 1);
            mma_f16(d, ad, bd, id, first ? 0u : 1u);
          }
        }
        mma_commit(&empty[s]);
      }
      mma_commit(accBar);
    }
  } else {
    // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31.
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const bool ready = mbar_wait(accBar, 0, p.err, 3);
    tc_fence_after();
    if (ready) {
      const int tileRow = mtile * kBM + row;
      const int nbig = nk < kBigAcc ? nk : kBigAcc;
#pragma unroll 1
      for (int c = 0; c < kN / 16; c++) {
        double acc[16];
#pragma unroll
        for (int i = 0; i < 16; i++) acc[i] = 0.0;
#pragma unroll 1
        for (int a = 0; a <= nbig; a++) {
          uint32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + a * kN + c * 16, v);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; i++) acc[i] += (double)__uint_as_float(v[i]);
        }
        const int q0 = (ntile * kN + c * 16) / 2;
        if (tileRow >= rowsM) continue;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int q = q0 + i;
          if (q >= p.Q) break;
          double2 val = make_double2(acc[2 * i], acc[2 * i + 1]);
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
    tmem_dealloc(tmem, kAccumulators * kN);
  }
}

// ---------------------------------------------------------------------------
// Field-side operands: BF16 hi/mid/lo planes of the real rows r = 2q + part.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void split3(double x, __nv_bfloat16& h, __nv_bfloat16& md,
                                       __nv_bfloat16& lo) {
  h = __double2bfloat16(x);
  const double r1 = x - (double)__bfloat162float(h);
  md = __double2bfloat16(r1);
  lo = __double2bfloat16(r1 - (double)__bfloat162float(md));
}

// Inverse: packed coefficients -> B[split][m*R + 2q + part][k], k < Kp_m.
__global__ void k_prep_inverse_bf16(int lmax, int n, int na, int count, int Q, int R,
                                    int isReal, long coefSize, int pitch, size_t plane,
                                    const double2* __restrict__ coef,
                                    __nv_bfloat16* __restrict__ op) {
  const int m = blockIdx.y, q = blockIdx.z;
  const int sgn = q / count, f = q - sgn * count;
  const int l0 = m > na ? m : na;
  const int kp = (lmax - l0 + 1 + kBK - 1) / kBK * kBK;
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
  const size_t r0 = ((size_t)m * R + 2 * q) * pitch + k;
  __nv_bfloat16 h, md, lo;
  split3(v.x, h, md, lo);
  op[r0] = h;
  op[plane + r0] = md;
  op[2 * plane + r0] = lo;
  split3(v.y, h, md, lo);
  op[r0 + pitch] = h;
  op[plane + r0 + pitch] = md;
  op[2 * plane + r0 + pitch] = lo;
}

// Forward: weighted spectra (FP64) -> B[split][m*R + 2q + part][j].
__global__ void k_prep_forward_bf16(int lmax, int Q, int R, int thetaPad, size_t plane,
                                    const double2* __restrict__ spec,
                                    __nv_bfloat16* __restrict__ op) {
  const int m = blockIdx.y;
  const int q = blockIdx.z;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= thetaPad) return;
  const double2 v = spec[((size_t)m * Q + q) * thetaPad + j];
  const size_t r0 = ((size_t)m * R + 2 * q) * thetaPad + j;
  __nv_bfloat16 h, md, lo;
  split3(v.x, h, md, lo);
  op[r0] = h;
  op[plane + r0] = md;
  op[2 * plane + r0] = lo;
  split3(v.y, h, md, lo);
  op[r0 + thetaPad] = h;
  op[plane + r0 + thetaPad] = md;
  op[2 * plane + r0 + thetaPad] = lo;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
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

// 3-D BF16 tensor [planes][rows][inner] with a [1][boxRows][64] box, 128 B swizzle.
gsht_status make_map_bf16(CUtensorMap* map, const void* base, uint64_t inner, uint64_t rows,
                          uint64_t planes, uint64_t rowPitchElems, uint64_t planeElems,
                          uint32_t boxInner, uint32_t boxRows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {inner, rows, planes};
  cuuint64_t strides[2] = {rowPitchElems * 2, planeElems * 2};
  cuuint32_t box[3] = {boxInner, boxRows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return GSHT_OK;
}

constexpr int kNsplit = 3, kNprod = 6, kNTile = 128, kStagesBf = 2;

template <int kDir>
gsht_status launch_bf16(const gsht_grid* g, const Table* t, const TcArgs& a,
                        const CUtensorMap& mapA, const CUtensorMap& mapB, int gridX,
                        cudaStream_t s) {
  auto kern = k_legendre_tc<kDir, kNsplit, kNsplit, kNprod, kNTile, kStagesBf>;
  const size_t sm = tc_smem_bytes<kNsplit, kNsplit, kNTile, kStagesBf>();
  GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(gridX, (a.R + kNTile - 1) / kNTile, a.lmax + 1);
  kern<<<grid, 192, sm, s>>>(mapA, mapB, a);
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_tc<inverse,bf16x3>" : "k_legendre_tc<forward,bf16x3>");
  return GSHT_OK;
}

}  // namespace

size_t bf16_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir) {
  const int R = 2 * (is_real ? 1 : 2) * count;
  const long long pitch = dir == 0 ? g->theta_pad : round_up(lmax + 1, kBK);
  return sizeof(__nv_bfloat16) * kNsplit * (size_t)(lmax + 1) * R * pitch;
}

gsht_status legendre_inverse_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, const double* coef, void* operand, double* spec,
                                  cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int pitch = (int)round_up(lmax + 1, kBK);
  const size_t plane = (size_t)(lmax + 1) * R * pitch;
  auto* op = static_cast<__nv_bfloat16*>(operand);
  {
    StageTimer tm(GSHT_STAGE_PREP_INVERSE, s);
    dim3 pg((pitch + 127) / 128, lmax + 1, Q);
    k_prep_inverse_bf16<<<pg, 128, 0, s>>>(lmax, t->n, na, count, Q, R, is_real,
                                           coef_size(lmax, t->n, is_real), pitch, plane,
                                           reinterpret_cast<const double2*>(coef), op);
    GSHT_LAUNCH_CHECK("k_prep_inverse_bf16");
  }
  CUtensorMap mapA, mapB;
  const size_t tplane = (size_t)(t->rows + kTablePadRows) * g->theta_pad;
  gsht_status st = make_map_bf16(&mapA, t->tbf, g->theta_pad, t->rows + kTablePadRows, 3,
                                 g->theta_pad, tplane, 64, 64);
  if (st != GSHT_OK) return st;
  st = make_map_bf16(&mapB, op, pitch, (uint64_t)(lmax + 1) * R, 3, pitch, plane, 64, kNTile);
  if (st != GSHT_OK) return st;
  TcArgs a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count; a.Q = Q; a.R = R;
  a.nTheta = g->n_theta; a.thetaPad = g->theta_pad; a.isReal = is_real;
  a.rowOff = t->d_row_off; a.out = reinterpret_cast<double2*>(spec);
  a.coefSize = coef_size(lmax, t->n, is_real); a.err = g->d_err;
  StageTimer tm(GSHT_STAGE_LEGENDRE_INVERSE, s);
  return launch_bf16<0>(g, t, a, mapA, mapB, (g->n_theta + kBM - 1) / kBM, s);
}

gsht_status legendre_forward_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, const double* spec, void* operand, double* coef,
                                  cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int tp = g->theta_pad;
  const size_t plane = (size_t)(lmax + 1) * R * tp;
  auto* op = static_cast<__nv_bfloat16*>(operand);
  {
    StageTimer tm(GSHT_STAGE_PREP_FORWARD, s);
    dim3 pg((tp + 127) / 128, lmax + 1, Q);
    k_prep_forward_bf16<<<pg, 128, 0, s>>>(lmax, Q, R, tp, plane,
                                           reinterpret_cast<const double2*>(spec), op);
    GSHT_LAUNCH_CHECK("k_prep_forward_bf16");
  }
  CUtensorMap mapA, mapB;
  const size_t tplane = (size_t)(t->rows + kTablePadRows) * tp;
  gsht_status st = make_map_bf16(&mapA, t->tbf, tp, t->rows + kTablePadRows, 3, tp, tplane, 64,
                                 kBM);
  if (st != GSHT_OK) return st;
  st = make_map_bf16(&mapB, op, tp, (uint64_t)(lmax + 1) * R, 3, tp, plane, 64, kNTile);
  if (st != GSHT_OK) return st;
  TcArgs a{};
  a.L = g->L; a.lmax = lmax; a.n = t->n; a.na = na; a.count = count; a.Q = Q; a.R = R;
  a.nTheta = g->n_theta; a.thetaPad = tp; a.isReal = is_real;
  a.rowOff = t->d_row_off; a.out = reinterpret_cast<double2*>(coef);
  a.coefSize = coef_size(lmax, t->n, is_real); a.err = g->d_err;
  const int kMax = lmax - na + 1;
  StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
  return launch_bf16<1>(g, t, a, mapA, mapB, (kMax + kBM - 1) / kBM, s);
}

}  // namespace gsht
