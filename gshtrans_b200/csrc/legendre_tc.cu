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
// Warp roles (320 threads): warp 0 issues TMA loads, warp 1 owns TMEM and
// issues MMAs from one lane, warps 2-9 drain TMEM in the epilogue. Every
// mbarrier wait is bounded (tc_common.cuh) and reports a timeout through
// the grid's device error word instead of hanging.
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

using namespace tc;

constexpr int kBM = 128;       // tile rows (TMEM lanes)
// K per stage. Forward: 64 colatitudes = one 128 B swizzle row of both
// K-major operands, two 96 KB stages. Inverse: 32 degrees (the MN-major
// table tile is two 64-colatitude x 32-degree boxes with 128 B swizzle, the
// K-major field rows one 64 B swizzle row), four 48 KB stages; or, selected
// at run time (inverse_bk), 64 degrees in two 96 KB stages like the forward.
__host__ __device__ constexpr int bk_of(int dir) { return dir == 0 ? 32 : 64; }
__host__ __device__ constexpr int stages_for(int bk) { return bk == 32 ? 4 : 2; }
// The inverse's field operand rows are padded to a multiple of 64 degrees
// (zeros), which serves both K steps.
constexpr int kBKInv = 64;

struct TcArgs {
  int L, lmax, n, na, count, Q, R, nTheta, thetaPad, isReal;
  const long long* rowOff;
  double2* out;
  // Inverse only: when set, the spectra are written here in FP32 with the -m
  // rows at their own colatitudes (the FP32 spectral layout of fft.cu).
  float2* out32;
  long coefSize;
  int* err;
  unsigned long long* trace;  // kTrSlots counters of a traced launch
};

// One group of a multi-group launch (batch plans): its tensor maps live in
// global memory beside its arguments (64-byte aligned, as TMA requires).
struct alignas(64) TcGroup {
  CUtensorMap mapA, mapB;
  TcArgs a;
};
// Tile x of a multi-group launch: group << 16 | m.
constexpr int kGroupShift = 16;

// TMEM accumulators per tile: products of very different magnitude would
// otherwise share one FP32 accumulator whose every update truncates; hi.hi
// goes to up to kBigAcc accumulators by K block and the other five products to
// a separate one, all summed in FP64 in the epilogue (4 x 128 = 512 columns).
constexpr int kBigAcc = 3;
constexpr int kAccumulators = kBigAcc + 1;
constexpr int kNprodTc = 6;  // BF16x3 split products

// Products of the BF16x3 form: (A split, B split).
__host__ __device__ constexpr int prodA(int p) { return p == 0 ? 0 : p == 1 ? 0 : p == 2 ? 1 : p == 3 ? 0 : p == 4 ? 2 : 1; }
__host__ __device__ constexpr int prodB(int p) { return p == 0 ? 0 : p == 1 ? 1 : p == 2 ? 0 : p == 3 ? 2 : p == 4 ? 0 : 1; }

template <int kNA, int kNB, int kN, int kBK, int kStages>
constexpr size_t tc_smem_bytes() {
  return (size_t)kStages * (kNA * kBM * kBK * 2 + kNB * kN * kBK * 2) + 1024 + 256;
}

constexpr int kEpiWarps = 8;  // two warps per TMEM lane quarter, one column group each
constexpr int kThreads = 32 * (2 + kEpiWarps);

// Persistent kernel: each block walks the tile list with stride gridDim.x.
// The producer runs ahead across tile boundaries; the epilogue copies its
// accumulator columns out of TMEM, releases TMEM to the MMA warp (accEmpty),
// and only then writes results, so stores overlap the next tile's MMAs.
//
// kMulti: the tiles belong to several groups (the batch plans' single
// launch over all groups of a direction): tile x = group << 16 | m, and each
// tile takes its arguments and tensor maps from groups[group].
template <int kDir, int kNA, int kNB, int kNP, int kN, int kStages, int kBK, bool kTrace,
          bool kMulti>
__global__ void __launch_bounds__(kThreads, 1)
    k_legendre_tc(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB, TcArgs p,
                  const int4* __restrict__ tiles, int numTiles,
                  const TcGroup* __restrict__ groups) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int kTileA = kBM * kBK * 2;
  constexpr int kTileB = kN * kBK * 2;
  constexpr int kStageBytes = kNA * kTileA + kNB * kTileB;
  constexpr int kCols = kN / (kEpiWarps / 4);  // accumulator columns per epilogue warp
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accFull = empty + kStages;
  // The epilogue releases the accumulators in two steps: accEmptyA once it
  // has copied accumulators 0 and 1 (all the next tile's first K blocks
  // need), accEmptyB after the hi.hi accumulators 2 and 3.
  uint64_t* accEmptyA = accFull + 1;
  uint64_t* accEmptyB = accFull + 2;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(accFull + 3);

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
    mbar_init(accEmptyA, kEpiWarps);
    mbar_init(accEmptyB, kEpiWarps);
    fence_barrier_init();
    if constexpr (!kMulti) {
      prefetch_tmap(&mapA);
      prefetch_tmap(&mapB);
    }
  }
  if (warp == 1) tmem_alloc(tmemSlot, kAccumulators * kN);
  // The arguments of tile tl (its group's in a multi-group launch) and its order.
  auto args = [&](const int4& tl) -> const TcArgs& {
    if constexpr (kMulti) return groups[tl.x >> kGroupShift].a;
    else return p;
  };
  auto order = [](const int4& tl) { return kMulti ? (tl.x & ((1 << kGroupShift) - 1)) : tl.x; };
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmemSlot;

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < numTiles && ok; t += gridDim.x) {
        const int4 tl = tiles[t];  // (m, mtile, ntile, nk)
        const TcArgs& ta = args(tl);
        const int m = order(tl);
        const CUtensorMap* mA = &mapA;
        const CUtensorMap* mB = &mapB;
        if constexpr (kMulti) {
          mA = &groups[tl.x >> kGroupShift].mapA;
          mB = &groups[tl.x >> kGroupShift].mapB;
        }
        const long long tRow = ta.rowOff[m];
        const int bRow = m * ta.R + tl.z * kN;
        for (int kc = 0; kc < tl.w; kc++, it++) {
          const int s = it % kStages;
          if (it >= kStages && !timed_wait<kTrace>(trW1, &empty[s], ((it / kStages) - 1) & 1, p.err, 1)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * kStageBytes;
          mbar_arrive_expect_tx(&full[s], kStageBytes);
          for (int a = 0; a < kNA; a++) {
            unsigned char* dst = st + a * kTileA;
            if (kDir == 0) {
              // MN-major: two 64-colatitude halves of 64 degree rows each.
              tma_load_3d(dst, mA, &full[s], tl.y * kBM, (int)(tRow + kc * kBK), a);
              tma_load_3d(dst + kTileA / 2, mA, &full[s], tl.y * kBM + 64,
                          (int)(tRow + kc * kBK), a);
            } else {
              tma_load_3d(dst, mA, &full[s], kc * kBK, (int)(tRow + tl.y * kBM), a);
            }
          }
          for (int b = 0; b < kNB; b++)
            tma_load_3d(st + kNA * kTileA + b * kTileB, mB, &full[s], kc * kBK, bRow, b);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t id = idesc(1, 1, kDir == 0 ? 1 : 0, 0, kN, kBM);
      int it = 0, tc = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < numTiles && ok; t += gridDim.x, tc++) {
        const int4 tl = tiles[t];
        const int nk = tl.w;
        const TcArgs& ta = args(tl);
        const int m = order(tl);
        // K steps of 16 past the last degree (inverse) or colatitude
        // (forward) multiply zero padding and are not issued.
        const int kLim = kDir == 0 ? ta.lmax - (m > ta.na ? m : ta.na) + 1 : ta.nTheta;
        if (tc > 0 && !timed_wait<kTrace>(trW2, accEmptyA, (tc - 1) & 1, p.err, 4)) break;
        tc_fence_after();
        bool haveB = tc == 0;
        // hi.hi products go to one of nbig accumulators by K block; the five
        // smaller products share accumulator 0 (see kAccumulators).
        const int nbig = nk < kBigAcc ? nk : kBigAcc;
        for (int kc = 0; kc < nk; kc++, it++) {
          const int s = it % kStages;
          if (!timed_wait<kTrace>(trW1, &full[s], (it / kStages) & 1, p.err, 2)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int big = 1 + (kc * nbig) / nk;
          const int bigFirst = ((big - 1) * nk + nbig - 1) / nbig;
          if (!haveB && big >= 2) {
            if (!timed_wait<kTrace>(trW2, accEmptyB, (tc - 1) & 1, p.err, 5)) {
              ok = false;
              break;
            }
            tc_fence_after();
            haveB = true;
          }
          const uint32_t st = smem_u32(smem + s * kStageBytes);
          // The last K block may end inside the padding: its K steps past
          // kLim are skipped (a separate copy of the loop, so that the
          // full blocks keep the branch-free one).
          auto issue = [&](auto whole) {
#pragma unroll
          for (int pr = 0; pr < kNP; pr++) {
            const uint32_t aBase = st + prodA(pr) * kTileA;
            const uint32_t bBase = st + kNA * kTileA + prodB(pr) * kTileB;
            const uint32_t d = tmem + (uint32_t)((pr == 0 ? big : 0) * kN);
#pragma unroll
            for (int k16 = 0; k16 < kBK / 16; k16++) {
              if constexpr (!decltype(whole)::value)
                if (k16 > 0 && kc * kBK + k16 * 16 >= kLim) break;
              uint64_t ad, bd;
              if constexpr (kDir == 0) {
                ad = sdesc_sw128(aBase + k16 * 2048, kTileA / 2, 1024);
                bd = kBK == 32 ? sdesc_sw64(bBase + k16 * 32, 16, 512)
                               : sdesc_sw128(bBase + k16 * 32, 16, 1024);
              } else {
                ad = sdesc_sw128(aBase + k16 * 32, 16, 1024);
                bd = sdesc_sw128(bBase + k16 * 32, 16, 1024);
              }
              const bool first = pr == 0 ? (kc == bigFirst && k16 == 0)
                                         : (kc == 0 && k16 == 0 && pr == 1);
              mma_f16(d, ad, bd, id, first ? 0u : 1u);
            }
          }
          };
          if ((kc + 1) * kBK <= kLim) issue(std::true_type{});
          else issue(std::false_type{});
          mma_commit(&empty[s]);
        }
        // Keep accEmptyB in step with the tiles even if this one used no
        // accumulator above 1.
        if (ok && !haveB && !timed_wait<kTrace>(trW2, accEmptyB, (tc - 1) & 1, p.err, 5)) ok = false;
        if (!ok) break;
        mma_commit(accFull);
      }
    }
  } else {
    // Epilogue warps 2..9: lane quarter warp % 4, column group (warp - 2) / 4.
    const int quarter = warp & 3;
    const int group = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;
    int tc = 0;
    for (int t = blockIdx.x; t < numTiles; t += gridDim.x, tc++) {
      const int4 tl = tiles[t];
      const TcArgs& ta = args(tl);
      const int m = order(tl), nk = tl.w;
      if (!timed_wait<kTrace>(trW1, accFull, tc & 1, p.err, 3)) break;
      tc_fence_after();
      const int nbig = nk < kBigAcc ? nk : kBigAcc;
      double acc[kCols];
#pragma unroll
      for (int i = 0; i < kCols; i++) acc[i] = 0.0;
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + group * kCols;
      // Two column chunks per wait; accumulators 0 and 1 first.
      auto drain = [&](int a) {
#pragma unroll
        for (int c = 0; c < kCols / 16; c += 2) {
          constexpr bool kPair = kCols / 16 > 1;
          uint32_t v0[16], v1[16];
          tmem_ld16(tbase + a * kN + c * 16, v0);
          if (kPair) tmem_ld16(tbase + a * kN + (c + 1) * 16, v1);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; i++) {
            acc[c * 16 + i] += (double)__uint_as_float(v0[i]);
            if (kPair) acc[(c + 1) * 16 + i] += (double)__uint_as_float(v1[i]);
          }
        }
      };
      drain(0);
      drain(1);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(accEmptyA);
#pragma unroll
      for (int a = 2; a <= kBigAcc; a++)
        if (a <= nbig) drain(a);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(accEmptyB);
      const int l0 = m > ta.na ? m : ta.na;
      const int keff = ta.lmax - l0 + 1;
      const int tileRow = tl.y * kBM + row;
      const int rowsM = kDir == 0 ? ta.nTheta : keff;
      if (tileRow >= rowsM) continue;
      const int q0 = (tl.z * kN + group * kCols) / 2;
      // Both directions write order-major rows [m][q][row] (row = colatitude
      // for the inverse, degree offset l - l0 for the forward); the forward's
      // rows are added into the packed coefficients by k_accumulate_forward.
      if (kDir == 0 && ta.out32) {
#pragma unroll
        for (int i = 0; i < kCols / 2; i++) {
          const int q = q0 + i;
          if (q >= ta.Q) break;
          // Table column tileRow holds +m at colatitude tileRow and -m at
          // its mirror nTheta-1-tileRow.
          const int col = q >= ta.count ? ta.nTheta - 1 - tileRow : tileRow;
          ta.out32[((size_t)m * ta.Q + q) * ta.thetaPad + col] =
              make_float2((float)acc[2 * i], (float)acc[2 * i + 1]);
        }
      } else if (kDir == 1 && ta.out32) {
#pragma unroll
        for (int i = 0; i < kCols / 2; i++) {
          const int q = q0 + i;
          if (q < ta.Q)
            ta.out32[((size_t)m * ta.Q + q) * ta.thetaPad + tileRow] =
                make_float2((float)acc[2 * i], (float)acc[2 * i + 1]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < kCols / 2; i++) {
          const int q = q0 + i;
          if (q < ta.Q)
            ta.out[((size_t)m * ta.Q + q) * ta.thetaPad + tileRow] =
                make_double2(acc[2 * i], acc[2 * i + 1]);
        }
      }
    }
  }
  if constexpr (kTrace)
    if (lane == 0) trace_role(p.trace, warp, true, trStart, trW1, trW2);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kAccumulators * kN);
  }
}

// ---------------------------------------------------------------------------
// CTA-pair form (cta_group::2) for batches of at least 256 field rows. The
// roles of the operands swap: A is 256 field rows (128 in each CTA of the
// pair), B a 128-wide tile of the table (64 colatitudes or degrees in each
// CTA), D = A B^T lands as 128 field rows x 128 table columns in each CTA's
// TMEM, with the same four accumulators as above (hi.hi by K block, the other
// five products together). Per tensor-core clock an SM now reads 96 B of
// operands from shared memory instead of 128 B, and each table tile is
// fetched once per pair instead of once per 128 field rows.
//
// Roles per CTA as in k_legendre_tc: warp 0 loads (TMA into the CTA's own
// shared memory, counted on the rank-0 CTA's full barrier, no multicast),
// warp 1 owns TMEM (rank 0 also issues the MMAs for the pair), warps 2-9
// drain the accumulators. The MMA commits multicast their arrivals to both
// CTAs' empty / accFull barriers; both CTAs' epilogue warps arrive on the
// rank-0 accEmpty barriers. Both CTAs of a pair walk the same tiles.
// ---------------------------------------------------------------------------
constexpr int kPairM = 256;  // field rows per pair tile
constexpr int kPairN = 128;  // table columns per pair tile
// Output staging per epilogue warp: 16 complex rows x 8 FP32 or 4 FP64
// columns, XOR-swizzled so that both the per-lane writes and the
// row-segment reads are free of bank conflicts.
constexpr int kPairStage = 1024;

template <int kStages, int kBK>
constexpr size_t tc2_smem_bytes() {
  return (size_t)kStages * 3 * (kBM + kPairN / 2) * kBK * 2 + 1024 + 256 +
         kEpiWarps * kPairStage;
}

// Table columns one pair tile computes: kPairN, or for the last tile of an
// order its valid columns rounded up to 32 (16 per CTA), so that the MMAs
// of a short tail tile run at N = 32..96 instead of 128.
__device__ __forceinline__ int pair_tile_n(int valid) {
  return valid >= kPairN ? kPairN : (valid + 31) / 32 * 32;
}

template <int kDir, int kStages, int kBK, bool kTrace>
__global__ void __launch_bounds__(kThreads, 1)
    k_legendre_tc2(const __grid_constant__ CUtensorMap mapT,
                   const __grid_constant__ CUtensorMap mapF, TcArgs p,
                   const int4* __restrict__ tiles, int numTiles) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int kTileF = kBM * kBK * 2;          // one split plane of this CTA's field rows
  constexpr int kTileT = (kPairN / 2) * kBK * 2;  // one split plane of this CTA's table half
  constexpr int kStageBytes = 3 * kTileF + 3 * kTileT;
  constexpr int kCols = kPairN / (kEpiWarps / 4);  // 64 accumulator columns per epilogue warp
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accFull = empty + kStages;
  uint64_t* accEmptyA = accFull + 1;
  uint64_t* accEmptyB = accFull + 2;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(accFull + 3);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  if (pair >= numTiles) return;  // both CTAs of the pair leave together
  long long trStart = 0, trW1 = 0, trW2 = 0;  // trace: start, first and second wait
  if constexpr (kTrace) trStart = clock64();

  if (warp == 0 && lane == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accFull, 1);
    mbar_init(accEmptyA, 2 * kEpiWarps);
    mbar_init(accEmptyB, 2 * kEpiWarps);
    fence_barrier_init();
    prefetch_tmap(&mapT);
    prefetch_tmap(&mapF);
  }
  if (warp == 1) tmem_alloc_pair(tmemSlot, kAccumulators * kPairN);
  tc_fence_before();
  cluster_sync();  // barriers of both CTAs initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tmem = *tmemSlot;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t fullRemote0 = cluster_addr(&full[0], 0);
      int it = 0;
      bool ok = true;
      for (int t = pair; t < numTiles && ok; t += npairs) {
        const int4 tl = tiles[t];  // (m, table tile, field tile, K blocks)
        const long long tRow = p.rowOff[tl.x];
        const int fRow = tl.x * p.R + tl.z * kPairM + (int)rank * kBM;
        // Rank 1 holds table columns [nT/2, nT) of a tile nT wide.
        const int limit = kDir == 0 ? p.nTheta : p.lmax - (tl.x > p.na ? tl.x : p.na) + 1;
        const int half = (int)rank * (pair_tile_n(limit - tl.y * kPairN) / 2);
        for (int kc = 0; kc < tl.w; kc++, it++) {
          const int s = it % kStages;
          if (it >= kStages && !timed_wait<kTrace>(trW1, &empty[s], ((it / kStages) - 1) & 1, p.err, 11)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * kStageBytes;
          const uint32_t fbar = fullRemote0 + (uint32_t)(s * sizeof(uint64_t));
          // The rank-0 CTA expects the bytes of both CTAs' loads.
          if (rank == 0) mbar_arrive_expect_tx(&full[s], 2 * kStageBytes);
          for (int a = 0; a < 3; a++)
            tma_load_3d_pair(st + a * kTileF, &mapF, fbar, kc * kBK, fRow, a);
          for (int a = 0; a < 3; a++) {
            unsigned char* dst = st + 3 * kTileF + a * kTileT;
            if (kDir == 0) {
              // MN-major: 64 colatitudes (this CTA's half) x kBK degree rows.
              tma_load_3d_pair(dst, &mapT, fbar, tl.y * kPairN + half, (int)(tRow + kc * kBK), a);
            } else {
              // K-major: 64 degree rows (this CTA's half) x kBK colatitudes.
              tma_load_3d_pair(dst, &mapT, fbar, kc * kBK, (int)(tRow + tl.y * kPairN + half), a);
            }
          }
        }
      }
      // Wait until the pair's MMAs have released every stage this CTA
      // filled, so that no commit arrival is still on its way here when
      // the CTA leaves.
      const int pending = it < kStages ? it : kStages;
      for (int i = it - pending; i < it && ok; i++)
        if (!timed_wait<kTrace>(trW1, &empty[i % kStages], (i / kStages) & 1, p.err, 16)) ok = false;
    }
  } else if (warp == 1) {
    if (rank == 0 && lane == 0) {
      int it = 0, tc = 0;
      bool ok = true;
      for (int t = pair; t < numTiles && ok; t += npairs, tc++) {
        const int4 tl = tiles[t];
        const int nk = tl.w;
        const int kLim = kDir == 0 ? p.lmax - (tl.x > p.na ? tl.x : p.na) + 1 : p.nTheta;
        const int limit = kDir == 0 ? p.nTheta : p.lmax - (tl.x > p.na ? tl.x : p.na) + 1;
        const uint32_t id =
            idesc(1, 1, 0, kDir == 0 ? 1 : 0, pair_tile_n(limit - tl.y * kPairN), kPairM);
        if (tc > 0 && !timed_wait<kTrace>(trW2, accEmptyA, (tc - 1) & 1, p.err, 14)) break;
        tc_fence_after();
        bool haveB = tc == 0;
        const int nbig = nk < kBigAcc ? nk : kBigAcc;
        for (int kc = 0; kc < nk; kc++, it++) {
          const int s = it % kStages;
          if (!timed_wait<kTrace>(trW1, &full[s], (it / kStages) & 1, p.err, 12)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int big = 1 + (kc * nbig) / nk;
          const int bigFirst = ((big - 1) * nk + nbig - 1) / nbig;
          if (!haveB && big >= 2) {
            if (!timed_wait<kTrace>(trW2, accEmptyB, (tc - 1) & 1, p.err, 15)) {
              ok = false;
              break;
            }
            tc_fence_after();
            haveB = true;
          }
          const uint32_t st = smem_u32(smem + s * kStageBytes);
          auto issue = [&](auto whole) {
#pragma unroll
          for (int pr = 0; pr < kNprodTc; pr++) {
            // A = field rows (split prodB), B = table (split prodA).
            const uint32_t aBase = st + prodB(pr) * kTileF;
            const uint32_t bBase = st + 3 * kTileF + prodA(pr) * kTileT;
            const uint32_t d = tmem + (uint32_t)((pr == 0 ? big : 0) * kPairN);
#pragma unroll
            for (int k16 = 0; k16 < kBK / 16; k16++) {
              if constexpr (!decltype(whole)::value)
                if (k16 > 0 && kc * kBK + k16 * 16 >= kLim) break;
              uint64_t ad, bd;
              if constexpr (kDir == 0) {
                ad = kBK == 32 ? sdesc_sw64(aBase + k16 * 32, 16, 512)
                               : sdesc_sw128(aBase + k16 * 32, 16, 1024);
                bd = sdesc_sw128(bBase + k16 * 2048, kTileT, 1024);
              } else {
                ad = sdesc_sw128(aBase + k16 * 32, 16, 1024);
                bd = sdesc_sw128(bBase + k16 * 32, 16, 1024);
              }
              const bool first = pr == 0 ? (kc == bigFirst && k16 == 0)
                                         : (kc == 0 && k16 == 0 && pr == 1);
              mma_f16_pair(d, ad, bd, id, first ? 0u : 1u);
            }
          }
          };
          if ((kc + 1) * kBK <= kLim) issue(std::true_type{});
          else issue(std::false_type{});
          mma_commit_pair(&empty[s], 0x3);
        }
        if (ok && !haveB && !timed_wait<kTrace>(trW2, accEmptyB, (tc - 1) & 1, p.err, 15)) ok = false;
        if (!ok) break;
        mma_commit_pair(accFull, 0x3);
      }
    }
  } else {
    // Epilogue warps 2..9: TMEM lane quarter warp % 4 (field rows), column
    // group (warp - 2) / 4 (64 table columns each).
    const int quarter = warp & 3;
    const int group = (warp - 2) >> 2;
    const uint32_t emptyA0 = cluster_addr(accEmptyA, 0), emptyB0 = cluster_addr(accEmptyB, 0);
    unsigned char* stg = smem + kStages * kStageBytes + 256 + (warp - 2) * kPairStage;
    // Lane = field row 2 ql + part of the warp's 32 (16 complex rows).
    const int ql = lane >> 1, part = lane & 1;
    const bool fp32 = kDir == 1 || p.out32 != nullptr;
    int tc = 0;
    for (int t = pair; t < numTiles; t += npairs, tc++) {
      const int4 tl = tiles[t];
      const int m = tl.x, nk = tl.w;
      const int l0 = m > p.na ? m : p.na;
      const int limit = kDir == 0 ? p.nTheta : p.lmax - l0 + 1;
      const int colW = tl.y * kPairN + group * kCols;  // first table column of this warp
      // Columns of a narrowed tail tile past its width hold stale values:
      // a warp whose 64 columns all lie there drains nothing.
      const bool live = group * kCols < pair_tile_n(limit - tl.y * kPairN);
      if (!timed_wait<kTrace>(trW1, accFull, tc & 1, p.err, 13)) break;
      tc_fence_after();
      const int nbig = nk < kBigAcc ? nk : kBigAcc;
      double acc[kCols];
#pragma unroll
      for (int i = 0; i < kCols; i++) acc[i] = 0.0;
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + group * kCols;
      auto drain = [&](int a) {
#pragma unroll
        for (int c = 0; c < kCols / 16; c += 2) {
          uint32_t v0[16], v1[16];
          tmem_ld16(tbase + a * kPairN + c * 16, v0);
          tmem_ld16(tbase + a * kPairN + (c + 1) * 16, v1);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; i++) {
            acc[c * 16 + i] += (double)__uint_as_float(v0[i]);
            acc[(c + 1) * 16 + i] += (double)__uint_as_float(v1[i]);
          }
        }
      };
      if (live) {
        drain(0);
        drain(1);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(emptyA0);
      if (live) {
#pragma unroll
        for (int a = 2; a <= kBigAcc; a++)
          if (a <= nbig) drain(a);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(emptyB0);
      if (!live) continue;
      // First complex row of this warp's 16.
      const int qw = (tl.z * kPairM + (int)rank * kBM + quarter * 32) >> 1;
      // Rows leave in chunks through the warp's staging buffer: each lane
      // writes its row's values, then each store instruction writes 64
      // contiguous bytes of 4 (FP32) or 2 (FP64) complex rows.
      if (fp32) {
        float* sf = reinterpret_cast<float*>(stg);
        const int swW = 2 * ((ql >> 1) & 7);
        const int c = lane & 7;
#pragma unroll
        for (int cc = 0; cc < kCols; cc += 8) {
          if (colW + cc < limit) {
#pragma unroll
            for (int u = 0; u < 8; u++) sf[ql * 16 + ((2 * u + part) ^ swW)] = (float)acc[cc + u];
            __syncwarp();
            const int col = colW + cc + c;
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int qr = (lane >> 3) + 4 * i;
              const float2 v =
                  *reinterpret_cast<const float2*>(sf + qr * 16 + ((2 * c) ^ (2 * ((qr >> 1) & 7))));
              const int q = qw + qr;
              if (col < limit && q < p.Q) {
                // Inverse: table column col holds +m at colatitude col and
                // -m at its mirror nTheta-1-col.
                const int cj = (kDir == 0 && q >= p.count) ? p.nTheta - 1 - col : col;
                p.out32[((size_t)m * p.Q + q) * p.thetaPad + cj] = v;
              }
            }
            __syncwarp();
          }
        }
      } else {
        double* sd = reinterpret_cast<double*>(stg);
        const int swW = 2 * ((ql >> 1) & 3);
        const int c = lane & 3;
#pragma unroll
        for (int cc = 0; cc < kCols; cc += 4) {
          if (colW + cc < limit) {
#pragma unroll
            for (int u = 0; u < 4; u++) sd[ql * 8 + ((2 * u + part) ^ swW)] = acc[cc + u];
            __syncwarp();
            const int col = colW + cc + c;
#pragma unroll
            for (int i = 0; i < 2; i++) {
              const int qr = (lane >> 2) + 8 * i;
              const double2 v =
                  *reinterpret_cast<const double2*>(sd + qr * 8 + ((2 * c) ^ (2 * ((qr >> 1) & 3))));
              const int q = qw + qr;
              if (col < limit && q < p.Q) p.out[((size_t)m * p.Q + q) * p.thetaPad + col] = v;
            }
            __syncwarp();
          }
        }
      }
    }
  }
  if constexpr (kTrace)
    if (lane == 0) trace_role(p.trace, warp, rank == 0, trStart, trW1, trW2);
  tc_fence_before();
  cluster_sync();  // no arrival is still on its way into either CTA
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem, kAccumulators * kPairN);
  }
}

// ---------------------------------------------------------------------------
// Field-side operands: BF16 hi/mid/lo planes of the real rows r = 2q + part.
// ---------------------------------------------------------------------------
// FP64 value: hi rounds x itself; the residual x - hi (at most 2^-8 |x|) is
// rounded once to FP32 (a relative error of 2^-24 of the residual, below
// 2^-32 |x|) and split on the FP32 pipe: four FP64-pipe operations per
// value instead of seven.
__device__ __forceinline__ void split3(double x, __nv_bfloat16& h, __nv_bfloat16& md,
                                       __nv_bfloat16& lo) {
  h = __double2bfloat16(x);
  const float r1 = (float)(x - (double)__bfloat162float(h));
  md = __float2bfloat16_rn(r1);
  lo = __float2bfloat16_rn(r1 - __bfloat162float(md));
}

// FP32 value: every residual is exact in FP32, so this equals the FP64
// split of the same value, on the FP32 pipe.
__device__ __forceinline__ void split3(float x, __nv_bfloat16& h, __nv_bfloat16& md,
                                       __nv_bfloat16& lo) {
  h = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h);
  md = __float2bfloat16_rn(r1);
  lo = __float2bfloat16_rn(r1 - __bfloat162float(md));
}

// Inverse: packed coefficients -> B[split][m*R + 2q + part][k], k = l - l0(m)
// < Kp_m (zero beyond lmax). One block per 32 degrees x 32 orders of kQB
// field rows q: the packed layout is contiguous along orders for a fixed
// degree, so each tile is read order-major (coalesced), transposed in shared
// memory and written degree-major, two degrees per lane as BF16 pairs. A
// pair starts at an even k; so that every k is written exactly once the tile
// holds degrees lt-1 .. lt+31 and order m writes k in [kb, kb + 32), kb =
// lt - l0 rounded down to even (consecutive degree tiles of one order then
// cover consecutive k ranges). blockIdx.x walks the triangle of (degree tile
// a, order tile b <= a) pairs row by row (row b holds nA - b tiles), so no
// block is launched for the empty upper half.
// fieldPtrs: when set, field f's coefficients are read from fieldPtrs[f]
// (batch plans: the callers' buffers) instead of coef + f * coefSize.
template <int kQB>
__global__ void __launch_bounds__(256) k_prep_inverse_bf16(
    int lmax, int n, int na, int count, int Q, int R, int isReal, long coefSize, int pitch,
    size_t plane, int nA, const double2* __restrict__ coef, __nv_bfloat16* __restrict__ op,
    const double2* const* __restrict__ fieldPtrs) {
  constexpr int kRows = 33;  // degrees lt-1 .. lt+31
  __shared__ double2 tile[kQB][kRows][33];
  int i0 = blockIdx.x, b = 0;
  while (i0 >= nA - b) {
    i0 -= nA - b;
    b++;
  }
  const int lt = (b + i0) * 32, mt = b * 32, qBase = blockIdx.z * kQB;
  if (lt + 31 < (mt > na ? mt : na) || mt > lmax) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Every load of the block's kQB tiles is issued into registers before any
  // of them is used, then the tiles are filled and the block synchronises
  // once: a warp keeps all its rows in flight at the same time.
  constexpr int kPer = (kRows + 7) / 8;  // rows per warp (warp 0 takes the 33rd)
  double2 v[kQB][kPer];
#pragma unroll
  for (int u = 0; u < kQB; u++) {
    const int q = qBase + u;
    const int sgn = q / count, f = q - sgn * count;
    const double2* src = q < Q ? (fieldPtrs ? fieldPtrs[f] : coef + (size_t)f * coefSize) : coef;
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int i = warp + 8 * r;
      const int l = lt - 1 + i, m = mt + lane;
      v[u][r] = make_double2(0.0, 0.0);
      if (i < kRows && q < Q && l >= 0 && l <= lmax && m <= l && l >= na &&
          !(sgn == 1 && m == 0)) {
        const long idx = isReal ? (long)l * (l + 1) / 2 - (long)na * (na + 1) / 2 + m
                                : (long)l * l - (long)n * n + l + (sgn ? -m : m);
        v[u][r] = src[idx];
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kQB; u++) {
    const int sgn = (qBase + u) / count;
#pragma unroll
    for (int r = 0; r < kPer; r++) {
      const int i = warp + 8 * r;
      if (i >= kRows) continue;
      double2 x = v[u][r];
      if (sgn == 1 && ((lt - 1 + i + n) & 1)) x = make_double2(-x.x, -x.y);
      tile[u][i][lane] = x;
    }
  }
  __syncthreads();
  // Half-warp h of warp w writes order jj = 2 (w + 8 it) + h; lane p of the
  // half-warp the pair k = kb + 2p, kb + 2p + 1.
  const int h = lane >> 4, pr = lane & 15;
#pragma unroll
  for (int u = 0; u < kQB; u++) {
    const int q = qBase + u;
    if (q >= Q) break;
#pragma unroll
    for (int it = 0; it < 2; it++) {
      const int jj = 2 * (warp + 8 * it) + h;
      const int m = mt + jj;
      if (m > lmax) continue;
      const int l0 = m > na ? m : na;
      const int kp = (lmax - l0 + 1 + kBKInv - 1) / kBKInv * kBKInv;
      const int d = lt - l0;
      const int k = d - (d & 1) + 2 * pr;
      if (k < 0 || k >= kp) continue;
      const int i = k + l0 - (lt - 1);  // tile row of degree l0 + k
      const double2 v0 = tile[u][i][jj], v1 = tile[u][i + 1][jj];
      const size_t r0 = ((size_t)m * R + 2 * q) * pitch + k;
      __nv_bfloat162 hh, mm, ll;
      split3(v0.x, hh.x, mm.x, ll.x);
      split3(v1.x, hh.y, mm.y, ll.y);
      *reinterpret_cast<__nv_bfloat162*>(op + r0) = hh;
      *reinterpret_cast<__nv_bfloat162*>(op + plane + r0) = mm;
      *reinterpret_cast<__nv_bfloat162*>(op + 2 * plane + r0) = ll;
      split3(v0.y, hh.x, mm.x, ll.x);
      split3(v1.y, hh.y, mm.y, ll.y);
      *reinterpret_cast<__nv_bfloat162*>(op + r0 + pitch) = hh;
      *reinterpret_cast<__nv_bfloat162*>(op + plane + r0 + pitch) = mm;
      *reinterpret_cast<__nv_bfloat162*>(op + 2 * plane + r0 + pitch) = ll;
    }
  }
}

// Forward: order-major result rows R[m][q][l - l0] (pitch thetaPad) added
// into the packed coefficients, with the -m rows' factor (-1)^(l+n) and the
// c_{L,L} = 0 rule of complex fields (GaussLegendreGrid.h:209-215). One block
// per 32 degrees x 32 orders of one row q: rows are read degree-contiguous,
// transposed in shared memory, and the packed layout (order-contiguous for a
// fixed degree) is read-modify-written coalesced. RowT: double2, or float2
// for the rows of the BF16x3 form.
// fieldPtrs: when set, field f's coefficients are fieldPtrs[f] (batch
// plans: the callers' buffers) instead of coef + f * coefSize.
template <typename RowT>
__global__ void __launch_bounds__(256) k_accumulate_forward(
    int L, int lmax, int n, int na, int count, int Q, int isReal, long coefSize, int pitch,
    const RowT* __restrict__ rows, double2* __restrict__ coef,
    double2* const* __restrict__ fieldPtrs) {
  __shared__ double2 tile[32][33];
  const int lt = blockIdx.x * 32, mt = blockIdx.y * 32, q = blockIdx.z;
  if (mt > lt + 31 || mt > lmax) return;
  const int sgn = q / count, f = q - sgn * count;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = warp; i < 32; i += 8) {
    const int m = mt + i, l = lt + lane;
    const int l0 = m > na ? m : na;
    double2 v = make_double2(0.0, 0.0);
    if (m <= lmax && l <= lmax && l >= l0) {
      const RowT x = rows[((size_t)m * Q + q) * pitch + (l - l0)];
      v = make_double2(x.x, x.y);
    }
    tile[i][lane] = v;
  }
  __syncthreads();
#pragma unroll
  for (int i = warp; i < 32; i += 8) {
    const int l = lt + i, m = mt + lane;
    if (l > lmax || l < na || m > l || m > lmax || (sgn == 1 && m == 0)) continue;
    const long idx = isReal ? (long)l * (l + 1) / 2 - (long)na * (na + 1) / 2 + m
                            : (long)l * l - (long)n * n + l + (sgn ? -m : m);
    double2* ptr = (fieldPtrs ? fieldPtrs[f] : coef + (size_t)f * coefSize) + idx;
    double2 v = tile[lane][i];
    if (sgn == 1 && ((l + n) & 1)) v = make_double2(-v.x, -v.y);
    if (!isReal && sgn == 0 && m == L && l == L && lmax == L) {
      *ptr = make_double2(0.0, 0.0);
    } else {
      const double2 o = *ptr;
      *ptr = make_double2(o.x + v.x, o.y + v.y);
    }
  }
}

// Forward: weighted spectra (FP64, or FP32 with unmirrored -m rows) ->
// B[split][m*R + 2q + part][j]; column j of a -m row is the spectrum at the
// mirrored colatitude nTheta-1-j (zero in the padding). Two colatitudes per
// thread, written as BF16 pairs (thetaPad is even).
template <typename SpecT>
__global__ void k_prep_forward_bf16(int lmax, int Q, int R, int count, int nTheta, int thetaPad,
                                    size_t plane, const SpecT* __restrict__ spec,
                                    __nv_bfloat16* __restrict__ op) {
  const int m = blockIdx.y;
  const int q = blockIdx.z;
  const int j = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= thetaPad) return;
  const size_t row = ((size_t)m * Q + q) * thetaPad;
  // double2 for FP64 spectra, float2 (split on the FP32 pipe) for FP32 ones.
  using V = typename std::conditional<std::is_same<SpecT, double2>::value, double2, float2>::type;
  V v[2] = {};
  if constexpr (std::is_same<SpecT, double2>::value) {
    v[0] = spec[row + j];
    v[1] = spec[row + j + 1];
  } else if (q < count) {
    const float4 f = *reinterpret_cast<const float4*>(spec + row + j);
    v[0] = make_float2(f.x, f.y);
    v[1] = make_float2(f.z, f.w);
  } else {
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const int col = nTheta - 1 - (j + t);
      if (col >= 0) v[t] = spec[row + col];
    }
  }
  const size_t r0 = ((size_t)m * R + 2 * q) * thetaPad + j;
  __nv_bfloat162 h, md, lo;
  split3(v[0].x, h.x, md.x, lo.x);
  split3(v[1].x, h.y, md.y, lo.y);
  *reinterpret_cast<__nv_bfloat162*>(op + r0) = h;
  *reinterpret_cast<__nv_bfloat162*>(op + plane + r0) = md;
  *reinterpret_cast<__nv_bfloat162*>(op + 2 * plane + r0) = lo;
  split3(v[0].y, h.x, md.x, lo.x);
  split3(v[1].y, h.y, md.y, lo.y);
  *reinterpret_cast<__nv_bfloat162*>(op + r0 + thetaPad) = h;
  *reinterpret_cast<__nv_bfloat162*>(op + plane + r0 + thetaPad) = md;
  *reinterpret_cast<__nv_bfloat162*>(op + 2 * plane + r0 + thetaPad) = lo;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// 3-D BF16 tensor [planes][rows][inner] with a [1][boxRows][boxInner] box.
gsht_status make_map_bf16(CUtensorMap* map, const void* base, uint64_t inner, uint64_t rows,
                          uint64_t planes, uint64_t rowPitchElems, uint64_t planeElems,
                          uint32_t boxInner, uint32_t boxRows, CUtensorMapSwizzle sw) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {inner, rows, planes};
  cuuint64_t strides[2] = {rowPitchElems * 2, planeElems * 2};
  cuuint32_t box[3] = {boxInner, boxRows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(GSHT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return GSHT_OK;
}

constexpr int kNsplit = 3, kNprod = 6;

template <int kDir, int kN, int kBK>
gsht_status launch_bf16_n(const gsht_grid* g, const TcArgs& a, const CUtensorMap& mapA,
                          const CUtensorMap& mapB, cudaStream_t s) {
  gsht_status st;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
  const TileList* tl = tile_list(g, kDir == 0 ? 0 : 1, a.lmax, a.na, a.R, kN, kBK, &st);
  if (!tl) return st;
  constexpr int kSt = stages_for(kBK);
  const size_t sm = tc_smem_bytes<kNsplit, kNsplit, kN, kBK, kSt>();
  const int blocks = tl->count < sms ? tl->count : sms;
  if constexpr (kN == 128) {
    if (g_tc_trace) {
      // Traced copy (same results) of the 128-row tile kernel.
      TcArgs b = a;
      b.trace = trace_slots(0, kDir, s);
      if (!b.trace) return fail(GSHT_ERR_CUDA, "trace counters unavailable");
      auto kern = k_legendre_tc<kDir, kNsplit, kNsplit, kNprod, kN, kSt, kBK, true, false>;
      GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      kern<<<blocks, kThreads, sm, s>>>(mapA, mapB, b, tl->d_tiles, tl->count, nullptr);
      GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_tc<inverse,bf16x3,traced>"
                                  : "k_legendre_tc<forward,bf16x3,traced>");
      return GSHT_OK;
    }
  }
  auto kern = k_legendre_tc<kDir, kNsplit, kNsplit, kNprod, kN, kSt, kBK, false, false>;
  GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  kern<<<blocks, kThreads, sm, s>>>(mapA, mapB, a, tl->d_tiles, tl->count, nullptr);
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_tc<inverse,bf16x3>" : "k_legendre_tc<forward,bf16x3>");
  return GSHT_OK;
}

// Field-row tile width N of the BF16x3 kernels: 128 by default; 64 and 32
// waste fewer MMA columns on small batches (chosen by the batch autotuner).
bool valid_ntile(int ntile) { return ntile == 32 || ntile == 64 || ntile == 128; }

template <int kDir, int kBK>
gsht_status launch_bf16(const gsht_grid* g, int ntile, const TcArgs& a, const CUtensorMap& mapA,
                        const CUtensorMap& mapB, cudaStream_t s) {
  if (ntile == 32) return launch_bf16_n<kDir, 32, kBK>(g, a, mapA, mapB, s);
  if (ntile == 64) return launch_bf16_n<kDir, 64, kBK>(g, a, mapA, mapB, s);
  return launch_bf16_n<kDir, 128, kBK>(g, a, mapA, mapB, s);
}

// K step of the inverse kernels: 32 or 64 degrees per stage
// (GSHT_BF16X3_INV_K=32 / 64 for comparisons; default kInverseBK). Measured
// at lmax 1024, 64 fields, after the other forms in one run: 64 runs the
// inverse in 1.78 against 1.97 ms, with an error against the FP64 path of
// 8.1e-7 against 7.4e-7 (relative; the hi.hi accumulators split the degrees
// at other points).
constexpr int kInverseBK = 64;
int inverse_bk() {
  const char* e = getenv("GSHT_BF16X3_INV_K");
  if (e && atoi(e) == 64) return 64;
  if (e && atoi(e) == 32) return 32;
  return kInverseBK;
}

// The CTA-pair kernels serve batches of at least kPairM field rows. By
// default the forward takes them and the inverse keeps the one-CTA kernel
// (measured at lmax 1024, 64 fields: forward 1.69 against 1.75 ms, inverse
// 2.12 against 1.84 ms); GSHT_BF16X3_PAIR=0 / =1 selects the one-CTA / pair
// kernels for both directions (comparisons and tests).
bool pair_form(int R, int dir) {
  if (R < kPairM) return false;
  const char* e = getenv("GSHT_BF16X3_PAIR");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return dir == 1;
}

template <int kDir, int kBK>
gsht_status launch_bf16_pair(const gsht_grid* g, const TcArgs& a, const CUtensorMap& mapT,
                             const CUtensorMap& mapF, cudaStream_t s) {
  gsht_status st;
  // (m, 128-wide table tile, 256-row field tile, K blocks), table tiles innermost.
  const TileList* tl = tile_list(g, kDir == 0 ? 0 : 1, a.lmax, a.na, a.R, kPairM, kBK, &st);
  if (!tl) return st;
  constexpr int kSt = kBK == 32 ? 5 : 3;
  TcArgs b = a;
  if (g_tc_trace) {
    b.trace = trace_slots(0, kDir, s);
    if (!b.trace) return fail(GSHT_ERR_CUDA, "trace counters unavailable");
  }
  auto kern = g_tc_trace ? k_legendre_tc2<kDir, kSt, kBK, true> : k_legendre_tc2<kDir, kSt, kBK, false>;
  const size_t sm = tc2_smem_bytes<kSt, kBK>();
  GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg{};
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
  cfg.gridDim = dim3(sms & ~1);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    clusters = sms / 2;
  }
  const int pairs = tl->count < clusters ? tl->count : clusters;
  cfg.gridDim = dim3(2 * pairs);
  GSHT_CUDA(cudaLaunchKernelEx(&cfg, kern, mapT, mapF, b, (const int4*)tl->d_tiles, tl->count));
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_tc2<inverse,bf16x3>" : "k_legendre_tc2<forward,bf16x3>");
  return GSHT_OK;
}

}  // namespace

// Tiles (m, M tile, N tile, K blocks), N tiles innermost: neighbouring
// blocks of the persistent grid work on the same table tile at the same
// time, so it comes from DRAM once and from L2 for the others.
const TileList* tile_list(const gsht_grid* g, int dir, int lmax, int na, int rows, int ntile,
                          int kstep, gsht_status* st, int tail) {
  *st = GSHT_OK;
  for (auto* t : g->tile_lists)
    if (t->dir == dir && t->lmax == lmax && t->na == na && t->rows == rows && t->ntile == ntile &&
        t->kstep == kstep && t->tail == tail)
      return t;
  std::vector<int4> v;
  const int ntiles = (rows + ntile - 1) / ntile;
  for (int m = 0; m <= lmax; m++) {
    const int l0 = m > na ? m : na;
    const int keff = lmax - l0 + 1;
    const int mtiles = dir == 0 ? (g->n_theta - tail + kBM - 1) / kBM : (keff + kBM - 1) / kBM;
    const int nk = dir == 0 ? (keff + kstep - 1) / kstep
                            : (tail ? (g->n_theta - tail + kstep - 1) / kstep
                                    : (g->theta_pad + kstep - 1) / kstep);
    for (int mt = 0; mt < mtiles; mt++)
      for (int nt = 0; nt < ntiles; nt++) v.push_back(make_int4(m, mt, nt, nk));
  }
  auto* t = new TileList();
  t->dir = dir; t->lmax = lmax; t->na = na; t->rows = rows; t->ntile = ntile; t->kstep = kstep;
  t->tail = tail;
  t->count = (int)v.size();
  if (dev_malloc(&t->d_tiles, sizeof(int4) * v.size()) != cudaSuccess ||
      cudaMemcpy(t->d_tiles, v.data(), sizeof(int4) * v.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaGetLastError();
    dev_free(t->d_tiles);
    delete t;
    *st = fail(GSHT_ERR_OOM, "tile list allocation failed");
    return nullptr;
  }
  g->tile_lists.push_back(t);
  return t;
}

size_t bf16_operand_bytes(const gsht_grid* g, int lmax, int is_real, int count, int dir) {
  const int R = 2 * (is_real ? 1 : 2) * count;
  const long long pitch = dir == 0 ? g->theta_pad : round_up(lmax + 1, kBKInv);
  return sizeof(__nv_bfloat16) * kNsplit * (size_t)(lmax + 1) * R * pitch;
}

gsht_status bf16_prep_inverse(const gsht_grid* g, const Table* t, int lmax, int is_real,
                              int count, const double* coef, void* operand, cudaStream_t s,
                              const double* const* fieldPtrs) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int pitch = (int)round_up(lmax + 1, kBKInv);
  const size_t plane = (size_t)(lmax + 1) * R * pitch;
  StageTimer tm(GSHT_STAGE_PREP_INVERSE, s);
  // Degrees up to l0 + kp - 1 <= lmax + kBKInv - 1: the zero padding of
  // every order's row up to its K-step multiple is written too.
  const int nA = (lmax + kBKInv + 31) / 32, nB = (lmax + 32) / 32;
  // One field row per block: 18 KB of shared memory and 40 registers, eight
  // blocks per SM (0.48 ms at lmax 1024, 64 fields; two rows per block: 0.49
  // ms at four blocks per SM, 0.51 ms before the loads went to registers).
  constexpr int kQB = 1;
  dim3 pg(nB * nA - nB * (nB - 1) / 2, 1, (Q + kQB - 1) / kQB);
  k_prep_inverse_bf16<kQB><<<pg, 256, 0, s>>>(lmax, t->n, na, count, Q, R, is_real,
                                              coef_size(lmax, t->n, is_real), pitch, plane, nA,
                                              reinterpret_cast<const double2*>(coef),
                                              static_cast<__nv_bfloat16*>(operand),
                                              reinterpret_cast<const double2* const*>(fieldPtrs));
  GSHT_LAUNCH_CHECK("k_prep_inverse_bf16");
  return GSHT_OK;
}

gsht_status bf16_prep_forward(const gsht_grid* g, int lmax, int is_real, int count,
                              const double* spec, void* operand, cudaStream_t s, bool spec32) {
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int tp = g->theta_pad;
  const size_t plane = (size_t)(lmax + 1) * R * tp;
  auto* op = static_cast<__nv_bfloat16*>(operand);
  StageTimer tm(GSHT_STAGE_PREP_FORWARD, s);
  dim3 pg((tp / 2 + 127) / 128, lmax + 1, Q);
  if (spec32)
    k_prep_forward_bf16<float2><<<pg, 128, 0, s>>>(lmax, Q, R, count, g->n_theta, tp, plane,
                                                   reinterpret_cast<const float2*>(spec), op);
  else
    k_prep_forward_bf16<double2><<<pg, 128, 0, s>>>(lmax, Q, R, count, g->n_theta, tp, plane,
                                                    reinterpret_cast<const double2*>(spec), op);
  GSHT_LAUNCH_CHECK("k_prep_forward_bf16");
  return GSHT_OK;
}

namespace {

// Arguments and tensor maps of one Legendre launch of the BF16x3 form over
// the prepared operand rows (dir 0 inverse: K step bk, results into the
// spectra, FP32 when spec32; dir 1 forward: K step 64, FP32 result rows into
// the spectra's buffer). fieldRows: field rows per box (the launch's tile
// width, or 128 for one CTA's share of a pair tile); tableRows likewise for
// the table boxes (128, or 64 for a pair's half tile).
gsht_status bf16_stage(const gsht_grid* g, const Table* t, int dir, int lmax, int is_real,
                       int count, void* operand, double* spec, bool spec32, int bk, int fieldRows,
                       int tableRows, TcArgs* a, CUtensorMap* mapA, CUtensorMap* mapB) {
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  const int tp = g->theta_pad;
  const int pitch = dir == 0 ? (int)round_up(lmax + 1, kBKInv) : tp;
  const size_t plane = (size_t)(lmax + 1) * R * pitch;
  const size_t tplane = (size_t)(t->rows + kTablePadRows) * tp;
  gsht_status st;
  if (dir == 0) {
    // MN-major table boxes of 64 colatitudes x bk degrees.
    st = make_map_bf16(mapA, t->tbf, tp, t->rows + kTablePadRows, 3, tp, tplane, 64, bk,
                       CU_TENSOR_MAP_SWIZZLE_128B);
    if (st != GSHT_OK) return st;
    st = make_map_bf16(mapB, operand, pitch, (uint64_t)(lmax + 1) * R, 3, pitch, plane, bk,
                       fieldRows, bk == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B);
  } else {
    st = make_map_bf16(mapA, t->tbf, tp, t->rows + kTablePadRows, 3, tp, tplane, bk_of(1),
                       tableRows, CU_TENSOR_MAP_SWIZZLE_128B);
    if (st != GSHT_OK) return st;
    st = make_map_bf16(mapB, operand, tp, (uint64_t)(lmax + 1) * R, 3, tp, plane, bk_of(1),
                       fieldRows, CU_TENSOR_MAP_SWIZZLE_128B);
  }
  if (st != GSHT_OK) return st;
  *a = TcArgs{};
  a->L = g->L; a->lmax = lmax; a->n = t->n; a->na = na; a->count = count; a->Q = Q; a->R = R;
  a->nTheta = g->n_theta; a->thetaPad = tp; a->isReal = is_real;
  a->rowOff = t->d_row_off; a->out = reinterpret_cast<double2*>(spec);
  // The forward's spectra are consumed (split into the BF16 planes) by the
  // time the kernel writes: their buffer holds its order-major result rows
  // (keff <= thetaPad), in FP32 (the form's accuracy is FP32-class; half the
  // bytes of FP64 for the kernel to write and the accumulation to read).
  a->out32 = (dir == 1 || spec32) ? reinterpret_cast<float2*>(spec) : nullptr;
  a->coefSize = coef_size(lmax, t->n, is_real); a->err = g->d_err;
  return GSHT_OK;
}

}  // namespace

gsht_status legendre_inverse_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, const double* coef, void* operand, double* spec,
                                  int ntile, cudaStream_t s, bool spec32) {
  if (!valid_ntile(ntile)) return fail(GSHT_ERR_BAD_ARG, "BF16x3 tile width %d not in {32, 64, 128}", ntile);
  const int R = 2 * (is_real ? 1 : 2) * count;
  gsht_status st = bf16_prep_inverse(g, t, lmax, is_real, count, coef, operand, s);
  if (st != GSHT_OK) return st;
  CUtensorMap mapA, mapB;
  TcArgs a;
  const int bk = inverse_bk();
  const bool pairForm = pair_form(R, 0);
  st = bf16_stage(g, t, 0, lmax, is_real, count, operand, spec, spec32, bk,
                  pairForm ? kBM : ntile, kBM, &a, &mapA, &mapB);
  if (st != GSHT_OK) return st;
  StageTimer tm(GSHT_STAGE_LEGENDRE_INVERSE, s);
  if (bk == 64)
    return pairForm ? launch_bf16_pair<0, 64>(g, a, mapA, mapB, s)
                    : launch_bf16<0, 64>(g, ntile, a, mapA, mapB, s);
  return pairForm ? launch_bf16_pair<0, 32>(g, a, mapA, mapB, s)
                  : launch_bf16<0, 32>(g, ntile, a, mapA, mapB, s);
}

gsht_status legendre_forward_bf16(const gsht_grid* g, const Table* t, int lmax, int is_real,
                                  int count, double* spec, void* operand, double* coef,
                                  int ntile, cudaStream_t s, bool spec32) {
  if (!valid_ntile(ntile)) return fail(GSHT_ERR_BAD_ARG, "BF16x3 tile width %d not in {32, 64, 128}", ntile);
  const int na = t->n < 0 ? -t->n : t->n;
  const int Q = (is_real ? 1 : 2) * count, R = 2 * Q;
  gsht_status st = bf16_prep_forward(g, lmax, is_real, count, spec, operand, s, spec32);
  if (st != GSHT_OK) return st;
  CUtensorMap mapA, mapB;
  TcArgs a;
  const bool pairForm = pair_form(R, 1);
  // Table boxes: 128 degree rows (one CTA's M), or 64 (one CTA's half of a
  // pair's 128-wide table tile).
  st = bf16_stage(g, t, 1, lmax, is_real, count, operand, spec, spec32, bk_of(1),
                  pairForm ? kBM : ntile, pairForm ? kPairN / 2 : kBM, &a, &mapA, &mapB);
  if (st != GSHT_OK) return st;
  {
    StageTimer tm(GSHT_STAGE_LEGENDRE_FORWARD, s);
    st = pairForm ? launch_bf16_pair<1, 64>(g, a, mapA, mapB, s)
                  : launch_bf16<1, 64>(g, ntile, a, mapA, mapB, s);
  }
  if (st != GSHT_OK) return st;
  return accumulate_forward(g->L, lmax, t->n, na, count, Q, is_real, a.coefSize, g->theta_pad,
                            spec, coef, s, true);
}

// ---------------------------------------------------------------------------
// Multi-group launches (batch plans): one persistent launch of the one-CTA
// kernel over the tiles of every group of a direction.
// ---------------------------------------------------------------------------
namespace {

template <int kDir, int kN, int kBK>
gsht_status launch_multi_n(const Bf16Multi& mp, cudaStream_t s) {
  constexpr int kSt = stages_for(kBK);
  auto kern = k_legendre_tc<kDir, kNsplit, kNsplit, kNprod, kN, kSt, kBK, false, true>;
  const size_t sm = tc_smem_bytes<kNsplit, kNsplit, kN, kBK, kSt>();
  GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, mp.device);
  const int blocks = mp.numTiles < sms ? mp.numTiles : sms;
  // The launch's own maps and arguments are unused by a multi-group kernel
  // except the error word (the first group's grid).
  CUtensorMap none{};
  TcArgs a{};
  a.err = mp.err;
  kern<<<blocks, kThreads, sm, s>>>(none, none, a, static_cast<const int4*>(mp.d_tiles),
                                    mp.numTiles, static_cast<const TcGroup*>(mp.d_groups));
  GSHT_LAUNCH_CHECK(kDir == 0 ? "k_legendre_tc<inverse,bf16x3,groups>"
                              : "k_legendre_tc<forward,bf16x3,groups>");
  return GSHT_OK;
}

template <int kDir, int kBK>
gsht_status launch_multi(const Bf16Multi& mp, cudaStream_t s) {
  if (mp.ntile == 32) return launch_multi_n<kDir, 32, kBK>(mp, s);
  if (mp.ntile == 64) return launch_multi_n<kDir, 64, kBK>(mp, s);
  return launch_multi_n<kDir, 128, kBK>(mp, s);
}

}  // namespace

gsht_status bf16_multi_build(int dir, const Bf16MultiGroup* gs, int ngroups, int ntile,
                             Bf16Multi* out) {
  *out = Bf16Multi{};
  if (ngroups < 1 || ngroups >= (1 << (31 - kGroupShift)))
    return fail(GSHT_ERR_BAD_ARG, "%d groups for one multi-group launch", ngroups);
  if (!valid_ntile(ntile)) return fail(GSHT_ERR_BAD_ARG, "BF16x3 tile width %d not in {32, 64, 128}", ntile);
  const int bk = dir == 0 ? inverse_bk() : bk_of(1);
  std::vector<TcGroup> hg(ngroups);
  std::vector<int4> tiles;
  for (int gi = 0; gi < ngroups; gi++) {
    const Bf16MultiGroup& q = gs[gi];
    if (q.lmax >= (1 << kGroupShift))
      return fail(GSHT_ERR_BAD_ARG, "lmax %d beyond a multi-group tile's order field", q.lmax);
    gsht_status st = bf16_stage(q.g, q.t, dir, q.lmax, q.isReal, q.count, q.operand, q.spec,
                                q.spec32, bk, ntile, kBM, &hg[gi].a, &hg[gi].mapA, &hg[gi].mapB);
    if (st != GSHT_OK) return st;
    // The group's tiles as tile_list lays them out, tagged with the group.
    const int na = q.t->n < 0 ? -q.t->n : q.t->n;
    const int R = hg[gi].a.R;
    const int ntiles = (R + ntile - 1) / ntile;
    for (int m = 0; m <= q.lmax; m++) {
      const int l0 = m > na ? m : na;
      const int keff = q.lmax - l0 + 1;
      const int mtiles = dir == 0 ? (q.g->n_theta + kBM - 1) / kBM : (keff + kBM - 1) / kBM;
      const int nk = dir == 0 ? (keff + bk - 1) / bk : (q.g->theta_pad + bk - 1) / bk;
      for (int mt = 0; mt < mtiles; mt++)
        for (int nt = 0; nt < ntiles; nt++)
          tiles.push_back(make_int4((gi << kGroupShift) | m, mt, nt, nk));
    }
  }
  out->dir = dir;
  out->ntile = ntile;
  out->bk = bk;
  out->device = gs[0].g->device;
  out->err = gs[0].g->d_err;
  out->numTiles = (int)tiles.size();
  if (dev_malloc_bytes(&out->d_groups, sizeof(TcGroup) * hg.size()) != cudaSuccess ||
      dev_malloc_bytes(&out->d_tiles, sizeof(int4) * tiles.size()) != cudaSuccess ||
      cudaMemcpy(out->d_groups, hg.data(), sizeof(TcGroup) * hg.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(out->d_tiles, tiles.data(), sizeof(int4) * tiles.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    bf16_multi_free(out);
    return fail(GSHT_ERR_OOM, "multi-group launch tables allocation failed");
  }
  return GSHT_OK;
}

gsht_status bf16_multi_launch(const Bf16Multi& mp, cudaStream_t s) {
  if (mp.numTiles == 0) return GSHT_OK;
  StageTimer tm(mp.dir == 0 ? GSHT_STAGE_LEGENDRE_INVERSE : GSHT_STAGE_LEGENDRE_FORWARD, s);
  if (mp.dir == 0)
    return mp.bk == 64 ? launch_multi<0, 64>(mp, s) : launch_multi<0, 32>(mp, s);
  return launch_multi<1, 64>(mp, s);
}

void bf16_multi_free(Bf16Multi* mp) {
  dev_free(mp->d_groups);
  dev_free(mp->d_tiles);
  *mp = Bf16Multi{};
}

gsht_status accumulate_forward(int L, int lmax, int n, int na, int count, int Q, int is_real,
                               long coefSize, int pitch, const double* rows, double* coef,
                               cudaStream_t s, bool rows32, double* const* fieldPtrs) {
  StageTimer tm(GSHT_STAGE_ACCUMULATE_FORWARD, s);
  dim3 ag((lmax + 32) / 32, (lmax + 32) / 32, Q);
  auto* fp = reinterpret_cast<double2* const*>(fieldPtrs);
  if (rows32)
    k_accumulate_forward<float2><<<ag, 256, 0, s>>>(L, lmax, n, na, count, Q, is_real, coefSize,
                                                    pitch, reinterpret_cast<const float2*>(rows),
                                                    reinterpret_cast<double2*>(coef), fp);
  else
    k_accumulate_forward<double2><<<ag, 256, 0, s>>>(L, lmax, n, na, count, Q, is_real, coefSize,
                                                     pitch, reinterpret_cast<const double2*>(rows),
                                                     reinterpret_cast<double2*>(coef), fp);
  GSHT_LAUNCH_CHECK("k_accumulate_forward");
  return GSHT_OK;
}

}  // namespace gsht
