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
// products are below 2^-56 of the operands' scales. The products of one A
// slice with consecutive B slices are issued as one MMA of N up to 256 (10
// MMAs per K step instead of 28), which cuts the shared-memory operand reads
// that bound the kernel by 43%.
//
// The 4-slice form (GSHT_OZAKI4, ~1e-7) keeps the first four table slices
// and the products i + j <= 3: 10 products in 4 MMAs per K step on 128-row
// field tiles, 4 diagonal accumulators x 128 columns.
//
// Table scale folding: in the inverse the table scale belongs to an output
// row (colatitude) and is applied in the epilogue; in the forward it runs
// along the contraction and is folded into the field-side rows before they
// are sliced.
#include <cstdio>
#include <type_traits>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

using namespace tc;

constexpr int kBM = 128;  // tile rows (TMEM lanes)
constexpr int kBK = 64;   // K (bytes) per stage
constexpr int kTmemCols = 512;

// Per-form configuration: kS slices per operand (7: the FP64-class form; 4:
// the ~1e-7 form, products i + j <= 3) and kN field rows per tile. One TMEM
// accumulator of kN columns per diagonal d = i + j.
template <int kS_, int kN_>
struct OzCfg {
  static constexpr int kNDiag = kS_;
  static constexpr int kTileA = kBM * kBK;  // 8 KB per slice
  static constexpr int kTileB = kN_ * kBK;  // 4 or 8 KB per slice
  static constexpr int kStageBytes = kS_ * (kTileA + kTileB);
  static constexpr int kStages = kS_ == 7 ? 2 : 3;
  static constexpr int kMaxMerge = 256 / kN_;  // B slices per MMA (N <= 256)
  static constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024 + 256;
  static_assert(kNDiag * kN_ <= kTmemCols, "diagonal accumulators exceed the TMEM allocation");
  static_assert(kSmemBytes <= 227 * 1024, "stages exceed shared memory");
};

struct OzArgs {
  int L, lmax, n, na, count, Q, R, nTheta, thetaPad, isReal;
  const long long* rowOff;
  const int* tabExp;  // [m][thetaPad] table column exponents
  const int* rowExp;  // [m * R + r] field row exponents
  double2* out;
  long coefSize;
  int* err;
  unsigned long long* trace;  // kTrSlots counters of a traced launch
  // Forward with a tail colatitude left out of the K steps: the FP64 table
  // column (rows from rowOff[m]) and the saved spectra [m Q + q], whose
  // product the epilogue adds to each result.
  const double* tail64;
  const double2* tailVals;
};

// Four warps per TMEM lane quarter, 16 columns each: the MMA warp waits for
// the drain of all 7 diagonals before the next tile, and 16 warps drain it
// in half the time of 8 (inverse 3.62 -> 3.36 ms at lmax 1024, 64 fields).
constexpr int kEpiWarps = 16;
constexpr int kThreads = 32 * (2 + kEpiWarps);

// Exact INT32 -> FP64 on the FP64 pipe: the double with high word 0x43300000
// and low word v + 2^31 is 2^52 + v + 2^31. Same value as a conversion
// instruction, without its lower-throughput pipe (the epilogue converts 7 x
// 32 accumulators per thread per tile).
__device__ __forceinline__ double i32_to_f64(uint32_t v) {
  return __hiloint2double(0x43300000, (int)(v ^ 0x80000000u)) - 4503601774854144.0;
}

// Persistent kernel over the tile list (see legendre_tc.cu for the protocol):
// the epilogue sums the 7 diagonal accumulators of its 32 columns in FP64,
// releases TMEM, then writes.
template <int kDir, int kS, int kN, bool kTrace>
__global__ void __launch_bounds__(kThreads, 1)
    k_legendre_oz(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB, OzArgs p,
                  const int4* __restrict__ tiles, int numTiles) {
  using C = OzCfg<kS, kN>;
  constexpr int kNDiag = C::kNDiag, kTileA = C::kTileA, kTileB = C::kTileB;
  constexpr int kStageBytes = C::kStageBytes, kStages = C::kStages, kMaxMerge = C::kMaxMerge;
  extern __shared__ __align__(1024) unsigned char oz_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(oz_smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int kCols = kN / (kEpiWarps / 4);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accFull = empty + kStages;
  uint64_t* accEmpty = accFull + 1;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(accEmpty + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ int skip;
  if (threadIdx.x == 0) skip = *reinterpret_cast<volatile int*>(p.err);
  __syncthreads();
  if (skip || blockIdx.x >= numTiles) return;
  long long trStart = 0, trW1 = 0, trW2 = 0;  // trace: start, first and second wait
  if constexpr (kTrace) trStart = clock64();

  if (warp == 0 && lane == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accFull, 1);
    mbar_init(accEmpty, kEpiWarps);
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
      int it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < numTiles && ok; t += gridDim.x) {
        const int4 tl = tiles[t];
        const long long tRow = p.rowOff[tl.x];
        const int bRow = tl.x * p.R + tl.z * kN;
        for (int kc = 0; kc < tl.w; kc++, it++) {
          const int s = it % kStages;
          if (it >= kStages && !timed_wait<kTrace>(trW1, &empty[s], ((it / kStages) - 1) & 1, p.err, 11)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * kStageBytes;
          mbar_arrive_expect_tx(&full[s], kStageBytes);
          for (int a = 0; a < kS; a++) {
            if (kDir == 0) {
              // MN-major: 128 colatitudes (one 128 B row) x 64 degree rows.
              tma_load_3d(st + a * kTileA, &mapA, &full[s], tl.y * kBM, (int)(tRow + kc * kBK), a);
            } else {
              tma_load_3d(st + a * kTileA, &mapA, &full[s], kc * kBK, (int)(tRow + tl.y * kBM), a);
            }
          }
          for (int b = 0; b < kS; b++)
            tma_load_3d(st + kS * kTileA + b * kTileB, &mapB, &full[s], kc * kBK, bRow, b);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {

      int it = 0, tc = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < numTiles && ok; t += gridDim.x, tc++) {
        const int4 tl = tiles[t];
        const int nk = tl.w;
        // K steps of 32 past the last degree (inverse) or colatitude
        // (forward) multiply zero padding and are not issued.
        const int kLim = kDir == 0 ? p.lmax - (tl.x > p.na ? tl.x : p.na) + 1 : p.nTheta;
        if (tc > 0 && !timed_wait<kTrace>(trW2, accEmpty, (tc - 1) & 1, p.err, 14)) break;
        tc_fence_after();
        for (int kc = 0; kc < nk; kc++, it++) {
          const int s = it % kStages;
          if (!timed_wait<kTrace>(trW1, &full[s], (it / kStages) & 1, p.err, 12)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + s * kStageBytes);
          // A slice i meets B slices j = 0..6-i, whose products belong to
          // diagonals i..6: the B slices lie back to back in shared memory
          // (one 64-row operand each, same 512 B row-group stride) and the
          // diagonal accumulators back to back in TMEM, so one MMA of N =
          // 64 x (number of slices) covers up to four of them. 10 MMAs per
          // K step instead of 28: A is read from shared memory 10 times.
          // The last K block may end inside the padding: its K steps past
          // kLim are skipped (a separate copy of the loop, so that the full
          // blocks keep the branch-free one).
          auto issue = [&](auto whole) {
#pragma unroll
          for (int i = 0; i < kS; i++) {
#pragma unroll
            for (int j0 = 0; i + j0 < kS; j0 += kMaxMerge) {
              const int nb = (kS - i - j0) < kMaxMerge ? (kS - i - j0) : kMaxMerge;
              const uint32_t idn = idesc(2, 1, kDir == 0 ? 1 : 0, 0, nb * kN, kBM);
              const uint32_t aBase = st + i * kTileA;
              const uint32_t bBase = st + kS * kTileA + j0 * kTileB;
              const uint32_t d = tmem + (uint32_t)((i + j0) * kN);
#pragma unroll
              for (int k32 = 0; k32 < kBK / 32; k32++) {
                if constexpr (!decltype(whole)::value)
                  if (k32 > 0 && kc * kBK + k32 * 32 >= kLim) break;
                const uint64_t ad = kDir == 0 ? sdesc_sw128(aBase + k32 * 4096, 8192, 1024)
                                              : sdesc_sw64(aBase + k32 * 32, 16, 512);
                const uint64_t bd = sdesc_sw64(bBase + k32 * 32, 16, 512);
                mma_i8(d, ad, bd, idn, (kc | i | k32) != 0);
              }
            }
          }
          };
          if ((kc + 1) * kBK <= kLim) issue(std::true_type{});
          else issue(std::false_type{});
          mma_commit(&empty[s]);
        }
        mma_commit(accFull);
      }
    }
  } else {
    const int quarter = warp & 3;
    const int group = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;
    int tc = 0;
    for (int t = blockIdx.x; t < numTiles; t += gridDim.x, tc++) {
      const int4 tl = tiles[t];
      const int m = tl.x;
      if (!timed_wait<kTrace>(trW1, accFull, tc & 1, p.err, 13)) break;
      tc_fence_after();
      double acc[kCols];
#pragma unroll
      for (int i = 0; i < kCols; i++) acc[i] = 0.0;
      static_assert(kCols % 16 == 0, "16-column TMEM loads");
#pragma unroll
      for (int d = 0; d < kNDiag; d++) {
        const double w = ldexp(1.0, -7 * (d + 2));
        const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + d * kN + group * kCols;
        uint32_t v[kCols];
#pragma unroll
        for (int c = 0; c < kCols / 16; c++)
          tmem_ld16(ta + 16 * c, *reinterpret_cast<uint32_t(*)[16]>(v + 16 * c));
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < kCols; i++) acc[i] = fma(i32_to_f64(v[i]), w, acc[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(accEmpty);
      const int l0 = m > p.na ? m : p.na;
      const int keff = p.lmax - l0 + 1;
      const int tileRow = tl.y * kBM + row;
      const int rowsM = kDir == 0 ? p.nTheta : keff;
      if (tileRow >= rowsM) continue;
      const int eA = kDir == 0 ? p.tabExp[(size_t)m * p.thetaPad + tileRow] : 0;
      const int q0 = (tl.z * kN + group * kCols) / 2;
      // Both directions write order-major rows [m][q][row] (row = colatitude
      // for the inverse, degree offset l - l0 for the forward, whose rows
      // k_accumulate_forward then adds into the packed coefficients).
#pragma unroll
      for (int i = 0; i < kCols / 2; i++) {
        const int q = q0 + i;
        if (q >= p.Q) break;
        const int ere = p.rowExp[(size_t)m * p.R + 2 * q];
        const int eim = p.rowExp[(size_t)m * p.R + 2 * q + 1];
        double2 o = make_double2(ldexp(acc[2 * i], eA + ere), ldexp(acc[2 * i + 1], eA + eim));
        if (kDir == 1 && p.tailVals) {
          const double d = p.tail64[p.rowOff[m] + tileRow];
          const double2 sv = p.tailVals[(size_t)m * p.Q + q];
          o = make_double2(fma(d, sv.x, o.x), fma(d, sv.y, o.y));
        }
        p.out[((size_t)m * p.Q + q) * p.thetaPad + tileRow] = o;
      }
    }
  }
  if constexpr (kTrace)
    if (lane == 0) trace_role(p.trace, warp, true, trStart, trW1, trW2);
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


// frexp exponent of x (|x| = f 2^e, f in [0.5, 1)) read from its bits;
// kNoExp for zero. Subnormals included.
constexpr int kNoExp = -100000;
__device__ __forceinline__ int exp_of(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  const int eb = (int)((b >> 52) & 0x7FF);
  if (eb != 0) return eb - 1022;
  const unsigned long long mant = b & ((1ull << 52) - 1);
  return mant == 0 ? kNoExp : -1010 - __clzll((long long)mant);
}

// floor(|x| 2^(sc + 49)) for |x| 2^sc < 1, from the bits of x: the 49 bits
// of y = x 2^sc that seven 7-bit slices keep, exactly (no rounding, so the
// same digits as truncating y * 128 seven times).
__device__ __forceinline__ unsigned long long digits49(double x, int sc) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  const int eb = (int)((b >> 52) & 0x7FF);
  unsigned long long m = b & ((1ull << 52) - 1);
  int e = 1;
  if (eb != 0) {
    m |= 1ull << 52;
    e = eb;
  }
  const int sh = 1026 - e - sc;  // |x| 2^(sc+49) = m 2^(e + sc - 1026)
  return sh >= 64 ? 0ull : (sh <= 0 ? 0ull : m >> sh);
}

// Four values y_t = x_t 2^{sc_t} (|y_t| < 1) -> kS slice quads, s-th quad
// to dst + s * plane (4-byte aligned): y = sum_s S_s 2^{-7(s+1)} with signed
// 7-bit truncation digits S_s, taken from the integer floor(|y| 2^49).
template <int kS>
__device__ __forceinline__ void write_slices4(const double (&x)[4], const int (&sc)[4],
                                              int8_t* dst, size_t plane) {
  unsigned long long Y[4];
  bool neg[4];
#pragma unroll
  for (int t = 0; t < 4; t++) {
    Y[t] = digits49(x[t], sc[t]);
    neg[t] = x[t] < 0.0;
  }
#pragma unroll
  for (int s = 0; s < kS; s++) {
    unsigned int w = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
      int d = (int)((Y[t] >> (42 - 7 * s)) & 127u);
      if (neg[t]) d = -d;
      w |= ((unsigned int)d & 0xFFu) << (8 * t);
    }
    *reinterpret_cast<unsigned int*>(dst + s * plane) = w;
  }
}

__device__ __forceinline__ int warp_max_int(int v) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Inverse: packed coefficients -> slices over degrees, K pitch `pitch` (a
// multiple of 64). One warp per row (m, q): the row maxima give the two
// exponents, then each lane writes four consecutive degrees as 4-byte slice
// quads.
// Six 256-thread blocks per SM (40 registers): the strided coefficient
// gathers need warps in flight more than registers (1.01 -> 0.85 ms at lmax
// 1024, 64 fields, against 76 registers and three blocks).
template <int kS>
__global__ void __launch_bounds__(256, 6) k_prep_inverse_oz(int lmax, int n, int na, int count, int Q, int R, int isReal,
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
  // Row exponents: the frexp exponent of each row's largest magnitude (0
  // for an all-zero row), from the exponent bits.
  int ere = kNoExp, eim = kNoExp;
  for (int k = lane; k < keff; k += 32) {
    const double2 v = value(k);
    ere = max(ere, exp_of(v.x));
    eim = max(eim, exp_of(v.y));
  }
  ere = warp_max_int(ere);
  eim = warp_max_int(eim);
  if (ere == kNoExp) ere = 0;
  if (eim == kNoExp) eim = 0;
  const size_t r0 = ((size_t)m * R + 2 * q) * pitch;
  if (lane == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  const int sre[4] = {-ere, -ere, -ere, -ere}, sim[4] = {-eim, -eim, -eim, -eim};
  for (int k4 = 4 * lane; k4 < kp; k4 += 128) {
    double re[4], im[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const double2 v = value(k4 + t);
      re[t] = v.x;
      im[t] = v.y;
    }
    write_slices4<kS>(re, sre, op + r0 + k4, plane);
    write_slices4<kS>(im, sim, op + r0 + pitch + k4, plane);
  }
}

// Forward: weighted spectra times the table column scales -> slices over
// colatitudes (pitch thetaPad, a multiple of 16). One warp per row (m, q),
// four consecutive colatitudes per lane: a first pass finds the row maxima,
// the second (reading the row again, now from L2) writes 4-byte slice quads.
template <int kS>
__global__ void k_prep_forward_oz(int lmax, int Q, int R, int thetaPad, size_t plane,
                                  const double2* __restrict__ spec,
                                  const int* __restrict__ tabExp, int8_t* __restrict__ op,
                                  int* __restrict__ rowExp) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (wid >= (lmax + 1) * Q) return;
  const int m = wid / Q, q = wid - m * Q;
  const double2* row = spec + ((size_t)m * Q + q) * thetaPad;
  const int4* te4 = reinterpret_cast<const int4*>(tabExp + (size_t)m * thetaPad);
  const int nq = thetaPad / 4;
  // Row exponents of the column-scaled values x 2^{e_j}: the largest
  // exp(x) + e_j (0 for an all-zero row).
  int ere = kNoExp, eim = kNoExp;
  for (int j4 = lane; j4 < nq; j4 += 32) {
    const int4 e = te4[j4];
    const int ev[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const double2 v = row[4 * j4 + t];
      const int xr = exp_of(v.x), xi = exp_of(v.y);
      if (xr != kNoExp) ere = max(ere, xr + ev[t]);
      if (xi != kNoExp) eim = max(eim, xi + ev[t]);
    }
  }
  ere = warp_max_int(ere);
  eim = warp_max_int(eim);
  if (ere == kNoExp) ere = 0;
  if (eim == kNoExp) eim = 0;
  if (lane == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  const size_t r0 = ((size_t)m * R + 2 * q) * thetaPad;
  for (int j4 = lane; j4 < nq; j4 += 32) {
    const int4 e = te4[j4];
    const int ev[4] = {e.x, e.y, e.z, e.w};
    double re[4], im[4];
    int sre[4], sim[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const double2 v = row[4 * j4 + t];
      re[t] = v.x;
      im[t] = v.y;
      sre[t] = ev[t] - ere;
      sim[t] = ev[t] - eim;
    }
    write_slices4<kS>(re, sre, op + r0 + 4 * j4, plane);
    write_slices4<kS>(im, sim, op + r0 + thetaPad + 4 * j4, plane);
  }
}


// Row-per-block forms of the two preparations: 128 threads read a row once
// and hold it while they reduce its exponent, then slice it, so the row is
// read from memory once for both (the warp-per-row kernels above read it
// twice, and with many rows in flight the second read misses L2). The
// inverse holds its row in shared memory (16 B per value; few registers, so
// up to ten blocks per SM keep the strided gathers in flight), the forward in
// registers. Same arithmetic, bit-identical slices.
constexpr int kRowThreads = 128;

__device__ __forceinline__ void block_max2(int& a, int& b) {
  __shared__ int red[2][kRowThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  a = warp_max_int(a);
  b = warp_max_int(b);
  if (lane == 0) {
    red[0][warp] = a;
    red[1][warp] = b;
  }
  __syncthreads();
#pragma unroll
  for (int w = 0; w < kRowThreads / 32; w++) {
    a = max(a, red[0][w]);
    b = max(b, red[1][w]);
  }
}

// Dynamic shared memory: pitch double2 (the row).
// tail: when set, the FP64 table column of the last colatitude (one value
// per table row, rows of order m from rowOff[m]); the block then also
// contracts its row with it in FP64 and writes that colatitude's spectrum,
// spec[(m Q + q) thetaPad + nTheta - 1] (the -m rows' spectra at the
// mirrored index, as the tensor-core epilogue writes them), which the
// inverse's M tiles then leave out.
template <int kS>
__global__ void __launch_bounds__(kRowThreads, 10) k_prep_inverse_oz_row(
    int lmax, int n, int na, int count, int Q, int R, int isReal, long coefSize, int pitch,
    size_t plane, const double2* __restrict__ coef, int8_t* __restrict__ op,
    int* __restrict__ rowExp, const double* __restrict__ tail,
    const long long* __restrict__ rowOff, double2* __restrict__ spec, int nTheta, int thetaPad) {
  extern __shared__ double2 rowBuf[];
  const int row = blockIdx.x;  // m * Q + q
  const int m = row / Q, q = row - m * Q;
  const int sgn = q / count, f = q - sgn * count;
  const int l0 = m > na ? m : na;
  const int keff = lmax - l0 + 1;
  const int kp = (keff + kBK - 1) / kBK * kBK;
  const double2* src = coef + (size_t)f * coefSize;
  int ere = kNoExp, eim = kNoExp;
  double tre = 0.0, tim = 0.0;  // this thread's part of the tail contraction
  const double* tcol = tail ? tail + rowOff[m] : nullptr;
  for (int k4 = 4 * (int)threadIdx.x; k4 < kp; k4 += 4 * kRowThreads) {
    double2 v[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int k = k4 + t, l = l0 + k;
      v[t] = make_double2(0.0, 0.0);
      if (k < keff && !(sgn == 1 && m == 0)) {
        const long idx = isReal ? (long)l * (l + 1) / 2 - (long)na * (na + 1) / 2 + m
                                : (long)l * l - (long)n * n + l + (sgn ? -m : m);
        v[t] = src[idx];
        if (sgn == 1 && ((l + n) & 1)) v[t] = make_double2(-v[t].x, -v[t].y);
      }
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
      ere = max(ere, exp_of(v[t].x));
      eim = max(eim, exp_of(v[t].y));
      rowBuf[k4 + t] = v[t];
    }
  }
  block_max2(ere, eim);  // its barrier also orders the row buffer
  if (ere == kNoExp) ere = 0;
  if (eim == kNoExp) eim = 0;
  if (threadIdx.x == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  const size_t r0 = ((size_t)m * R + 2 * q) * pitch;
  const int sre[4] = {-ere, -ere, -ere, -ere}, sim[4] = {-eim, -eim, -eim, -eim};
  for (int k4 = 4 * (int)threadIdx.x; k4 < kp; k4 += 4 * kRowThreads) {
    double re[4], im[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const double2 v = rowBuf[k4 + t];
      re[t] = v.x;
      im[t] = v.y;
    }
    write_slices4<kS>(re, sre, op + r0 + k4, plane);
    write_slices4<kS>(im, sim, op + r0 + pitch + k4, plane);
  }
  if (tcol) {
    // The tail contraction, from the buffered row (a second pass over
    // shared memory keeps the gather loop's registers as they were).
    for (int k = (int)threadIdx.x; k < keff; k += kRowThreads) {
      const double d = tcol[k];
      const double2 v = rowBuf[k];
      tre = fma(d, v.x, tre);
      tim = fma(d, v.y, tim);
    }
    __shared__ double tred[2][kRowThreads / 32];
    for (int o = 16; o; o >>= 1) {
      tre += __shfl_xor_sync(0xffffffffu, tre, o);
      tim += __shfl_xor_sync(0xffffffffu, tim, o);
    }
    if ((threadIdx.x & 31) == 0) {
      tred[0][threadIdx.x >> 5] = tre;
      tred[1][threadIdx.x >> 5] = tim;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
#pragma unroll
      for (int w = 0; w < kRowThreads / 32; w++) {
        a += tred[0][w];
        b += tred[1][w];
      }
      spec[((size_t)m * Q + q) * thetaPad + (nTheta - 1)] = make_double2(a, b);
    }
  }
}

// The forward keeps its row in registers instead (up to 512 kQ values, four
// consecutive per thread and pass): measured faster than the shared-memory
// buffer here (0.97 against 1.13 ms at lmax 1024, 64 fields, 7 slices),
// while the inverse's strided gathers want the occupancy that the small
// register footprint of the buffered form gives (0.82 against 0.93 ms).
// tailOut: when set, the row's spectrum at colatitude column nTheta - 1 is
// saved to tailOut[m Q + q] (the forward's tiles then stop before that
// column and their epilogue adds its FP64 product with the table).
template <int kS, int kQ>
__global__ void __launch_bounds__(kRowThreads) k_prep_forward_oz_row(
    int lmax, int Q, int R, int thetaPad, size_t plane, const double2* __restrict__ spec,
    const int* __restrict__ tabExp, int8_t* __restrict__ op, int* __restrict__ rowExp,
    double2* __restrict__ tailOut, int nTheta) {
  const int row = blockIdx.x;  // m * Q + q
  const int m = row / Q, q = row - m * Q;
  const double2* src = spec + (size_t)row * thetaPad;
  const int4* te4 = reinterpret_cast<const int4*>(tabExp + (size_t)m * thetaPad);
  const int nq = thetaPad / 4;
  double2 v[kQ][4];
  int4 e[kQ];
#pragma unroll
  for (int i = 0; i < kQ; i++) {
    const int j4 = (int)threadIdx.x + kRowThreads * i;
    e[i] = make_int4(0, 0, 0, 0);
#pragma unroll
    for (int t = 0; t < 4; t++) v[i][t] = make_double2(0.0, 0.0);
    if (j4 < nq) {
      e[i] = te4[j4];
#pragma unroll
      for (int t = 0; t < 4; t++) v[i][t] = src[4 * j4 + t];
    }
  }
  if (tailOut && threadIdx.x == 0) tailOut[row] = src[nTheta - 1];
  // Row exponents of the column-scaled values x 2^{e_j}: the largest
  // exp(x) + e_j (0 for an all-zero row).
  int ere = kNoExp, eim = kNoExp;
#pragma unroll
  for (int i = 0; i < kQ; i++) {
    const int ev[4] = {e[i].x, e[i].y, e[i].z, e[i].w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int xr = exp_of(v[i][t].x), xi = exp_of(v[i][t].y);
      if (xr != kNoExp) ere = max(ere, xr + ev[t]);
      if (xi != kNoExp) eim = max(eim, xi + ev[t]);
    }
  }
  block_max2(ere, eim);
  if (ere == kNoExp) ere = 0;
  if (eim == kNoExp) eim = 0;
  if (threadIdx.x == 0) {
    rowExp[(size_t)m * R + 2 * q] = ere;
    rowExp[(size_t)m * R + 2 * q + 1] = eim;
  }
  const size_t r0 = ((size_t)m * R + 2 * q) * thetaPad;
#pragma unroll
  for (int i = 0; i < kQ; i++) {
    const int j4 = (int)threadIdx.x + kRowThreads * i;
    if (j4 >= nq) break;
    const int ev[4] = {e[i].x, e[i].y, e[i].z, e[i].w};
    double re[4], im[4];
    int sre[4], sim[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      re[t] = v[i][t].x;
      im[t] = v[i][t].y;
      sre[t] = ev[t] - ere;
      sim[t] = ev[t] - eim;
    }
    write_slices4<kS>(re, sre, op + r0 + 4 * j4, plane);
    write_slices4<kS>(im, sim, op + r0 + thetaPad + 4 * j4, plane);
  }
}

// Rows up to this many values run row-per-block (inverse: 48 KB of shared
// memory without opting in; forward: kQ = 2, 3 or 6 passes); longer ones
// take the warp-per-row kernels.
constexpr int kRowMax = 3072;

inline int row_passes(int len) {
  const int p = (len + 4 * kRowThreads - 1) / (4 * kRowThreads);
  return p <= 2 ? 2 : (p <= 3 ? 3 : 6);
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

template <int kDir, int kS, int kN>
gsht_status launch_oz(const gsht_grid* g, const OzArgs& a, const CUtensorMap& mapA,
                      const CUtensorMap& mapB, cudaStream_t s, int tail = 0) {
  gsht_status st;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
  const TileList* tl = tile_list(g, kDir == 0 ? 0 : 1, a.lmax, a.na, a.R, kN, kBK, &st, tail);
  if (!tl) return st;
  constexpr size_t kSmem = OzCfg<kS, kN>::kSmemBytes;
  const int blocks = tl->count < sms ? tl->count : sms;
  if (g_tc_trace) {
    // Traced copy (same results), counters of the form's direction.
    OzArgs b = a;
    b.trace = trace_slots(1, kDir, s);
    if (!b.trace) return fail(GSHT_ERR_CUDA, "trace counters unavailable");
    auto kern = k_legendre_oz<kDir, kS, kN, true>;
    GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    kern<<<blocks, kThreads, kSmem, s>>>(mapA, mapB, b, tl->d_tiles, tl->count);
  } else {
    auto kern = k_legendre_oz<kDir, kS, kN, false>;
    GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    kern<<<blocks, kThreads, kSmem, s>>>(mapA, mapB, a, tl->d_tiles, tl->count);
  }
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_oz<inverse>" : "k_legendre_oz<forward>");
  return GSHT_OK;
}

}  // namespace

size_t oz_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir,
                        int slices) {
  const int kS = slices;
  const int R = 2 * (is_real ? 1 : 2) * count;
  const long long pitch = dir == 0 ? g->theta_pad : round_up(lmax + 1, kBK);
  // Slice planes, row exponents, and (forward) one saved spectrum value per
  // field row for the tail colatitude.
  return round_up((size_t)kS * (lmax + 1) * R * pitch, 256) +
         round_up(sizeof(int) * (size_t)(lmax + 1) * R, 256) +
         sizeof(double2) * (size_t)(lmax + 1) * (R / 2) + 256;
}

namespace {

template <int kS, int kN>
gsht_status inverse_oz(const gsht_grid* g, const Table* t, int lmax, int is_real, int count,
                       const double* coef, void* operand, double* spec, cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int pitch = (int)round_up(lmax + 1, kBK);
  const size_t plane = (size_t)(lmax + 1) * R * pitch;
  auto* op = static_cast<int8_t*>(operand);
  int* rowExp = reinterpret_cast<int*>(static_cast<char*>(operand) + round_up(kS * plane, 256));
  // With nTheta = 128 k + 1 the last colatitude would take a 128-row tile of
  // its own in every order (1/9 of the MMAs at lmax 1024): the row-per-block
  // preparation contracts it in FP64 instead.
  const bool tail = t->tail64 && pitch <= kRowMax && g->n_theta % kBM == 1;
  {
    StageTimer tm(GSHT_STAGE_PREP_INVERSE, s);
    const long long warps = (long long)(lmax + 1) * Q;
    const auto* c2 = reinterpret_cast<const double2*>(coef);
    const long cs = coef_size(lmax, t->n, is_real);
    if (pitch > kRowMax) {
      k_prep_inverse_oz<kS><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
          lmax, t->n, na, count, Q, R, is_real, cs, pitch, plane, c2, op, rowExp);
    } else {
      k_prep_inverse_oz_row<kS><<<(unsigned)warps, kRowThreads, sizeof(double2) * pitch, s>>>(
          lmax, t->n, na, count, Q, R, is_real, cs, pitch, plane, c2, op, rowExp,
          tail ? t->tail64 : nullptr, t->d_row_off, reinterpret_cast<double2*>(spec), g->n_theta,
          g->theta_pad);
    }
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
  return launch_oz<0, kS, kN>(g, a, mapA, mapB, s, tail ? 1 : 0);
}

template <int kS, int kN>
gsht_status forward_oz(const gsht_grid* g, const Table* t, int lmax, int is_real, int count,
                       double* spec, void* operand, double* coef, cudaStream_t s) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int tp = g->theta_pad;
  const size_t plane = (size_t)(lmax + 1) * R * tp;
  auto* op = static_cast<int8_t*>(operand);
  int* rowExp = reinterpret_cast<int*>(static_cast<char*>(operand) + round_up(kS * plane, 256));
  // With nTheta = 128 k + 1 the last colatitude would cost a 64-colatitude
  // K step of its own in every tile: the preparation saves its spectra, the
  // tiles stop before it, and the accumulation adds its FP64 product.
  const bool tail = t->tail64 && tp <= kRowMax && g->n_theta % kBM == 1;
  auto* tailVals = reinterpret_cast<double2*>(
      reinterpret_cast<char*>(rowExp) + round_up(sizeof(int) * (size_t)(lmax + 1) * R, 256));
  {
    StageTimer tm(GSHT_STAGE_PREP_FORWARD, s);
    const long long warps = (long long)(lmax + 1) * Q;
    const auto* s2 = reinterpret_cast<const double2*>(spec);
    if (tp > kRowMax) {
      k_prep_forward_oz<kS><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(
          lmax, Q, R, tp, plane, s2, t->i8_exp, op, rowExp);
    } else {
      const int passes = row_passes(tp);
      auto kern = passes == 2 ? k_prep_forward_oz_row<kS, 2>
                              : (passes == 3 ? k_prep_forward_oz_row<kS, 3> : k_prep_forward_oz_row<kS, 6>);
      kern<<<(unsigned)warps, kRowThreads, 0, s>>>(lmax, Q, R, tp, plane, s2, t->i8_exp, op, rowExp,
                                                   tail ? tailVals : nullptr, g->n_theta);
    }
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
  // The spectra, sliced above, are no longer needed: the kernel's result rows
  // go into their buffer and are then added into the coefficients.
  a.out = reinterpret_cast<double2*>(spec);
  a.coefSize = coef_size(lmax, t->n, is_real); a.err = g->d_err;
  if (tail) {
    a.tail64 = t->tail64;
    a.tailVals = tailVals;
  }
  {
    StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
    st = launch_oz<1, kS, kN>(g, a, mapA, mapB, s, tail ? 1 : 0);
  }
  if (st != GSHT_OK) return st;
  return accumulate_forward(g->L, lmax, t->n, na, count, Q, is_real, a.coefSize, tp, spec, coef, s);
}

}  // namespace

// Slices 7 (FP64-class) run on 64-row field tiles, 4 (~1e-7) on 128-row ones
// (4 diagonals x 128 TMEM columns).
gsht_status legendre_inverse_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, const double* coef, void* operand, double* spec,
                                cudaStream_t s, int slices) {
  if (slices == 4) return inverse_oz<4, 128>(g, t, lmax, is_real, count, coef, operand, spec, s);
  return inverse_oz<7, 64>(g, t, lmax, is_real, count, coef, operand, spec, s);
}

gsht_status legendre_forward_oz(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                int count, double* spec, void* operand, double* coef,
                                cudaStream_t s, int slices) {
  if (slices == 4) return forward_oz<4, 128>(g, t, lmax, is_real, count, spec, operand, coef, s);
  return forward_oz<7, 64>(g, t, lmax, is_real, count, spec, operand, coef, s);
}

}  // namespace gsht
