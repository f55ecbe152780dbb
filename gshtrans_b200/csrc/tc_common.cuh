// sm_100a building blocks for the tensor-core Legendre kernels: mbarriers
// with bounded waits, TMA tile loads (no multicast), tcgen05 MMA / commit /
// TMEM load, and the shared-memory matrix descriptors of the 128-byte
// swizzled canonical layouts.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace gsht {
namespace tc {

// Polls before a wait gives up and flags a timeout (well under a second with
// the back-off below); a healthy pipeline completes a wait in microseconds.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.b32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase; returns false (and raises *err) on
// timeout instead of spinning forever. A wait also gives up early once any
// block of the launch has raised the error word.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
  for (uint32_t i = 0; i < kWaitLimit; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(64);
    if ((i & 4095) == 4095 && *reinterpret_cast<volatile int*>(err) != 0) return false;
  }
  atomicMax(err, code);
  return false;
}

// 3-D tiled TMA load into shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// 4-D tiled TMA load into shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completion counted on `bar` (no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// its later async-proxy (TMA) ones.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2), sm100
// version bits (46..47 = 1). Addresses and offsets in bytes.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Same with 64-byte swizzle (layout type 4): 8-row atoms of 64 B rows.
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;
  return d;
}

// Instruction descriptor of kind::f16 / kind::i8 MMAs (M = 128).
//   dfmt: 1 = F32, 2 = S32; abfmt: kind::f16 0 = F16, 1 = BF16; kind::i8 1 = signed.
__host__ __device__ constexpr uint32_t idesc(uint32_t dfmt, uint32_t abfmt, uint32_t aMN,
                                             uint32_t bMN, uint32_t n, uint32_t m) {
  return (dfmt << 4) | (abfmt << 7) | (abfmt << 10) | (aMN << 15) | (bMN << 16) |
         ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate));
}

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate));
}

// Arrives on `bar` once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// TMEM allocation by one full warp; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(base), "r"(ncols)
               : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns; thread i of the warp receives lane
// (taddr.lane + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%"
      "15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// CTA pairs (clusters of 2) sharing one MMA: tcgen05 with cta_group::2. The
// even CTA (rank 0) issues the MMAs for both; each CTA holds half of the A
// rows and half of the B rows in its own shared memory and half of the D
// rows in its own TMEM. No multicast loads: every TMA load fills the issuing
// CTA's own shared memory (it only signals the rank-0 barrier).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}

// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void* local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
  return r;
}

// All threads of both CTAs; orders earlier shared-memory and barrier
// operations before the other CTA's later ones.
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Arrive on an mbarrier given by its cluster address (possibly the peer's).
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(caddr)
               : "memory");
}

// 3-D tiled TMA load into this CTA's shared memory whose completion counts on
// the barrier at cluster address `cbar` (the pair's rank-0 barrier).
__device__ __forceinline__ void tma_load_3d_pair(void* dst, const CUtensorMap* map, uint32_t cbar,
                                                 int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(cbar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_f16_pair(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                             uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate));
}

// Arrives on `bar` (same offset) in every CTA of `mask` once the pair's
// previously issued MMAs complete.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;\n" ::"r"(smem_u32(bar)),
      "h"(mask)
      : "memory");
}

// TMEM allocation for a pair: the same warp of both CTAs calls it with the
// same slot offset.
__device__ __forceinline__ void tmem_alloc_pair(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(base), "r"(ncols)
               : "memory");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver stub); nullptr if unavailable.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_fn() {
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

// ---------------------------------------------------------------------------
// Per-role cycle trace of the tensor-core pipelines (a diagnostic; the
// traced kernels are separate instantiations, so the untraced ones carry no
// trace code). Slots, summed over CTAs with atomics at the end of a launch:
// ---------------------------------------------------------------------------
enum TraceSlot {
  kTrProducer = 0,      // TMA producer thread: cycles from kernel start to its end
  kTrProducerWait = 1,  //   of which waiting for a free stage
  kTrMma = 2,           // MMA issuing thread: cycles from kernel start to its end
  kTrMmaWaitFull = 3,   //   of which waiting for a loaded stage
  kTrMmaWaitAcc = 4,    //   of which waiting for the epilogue to free TMEM
  kTrEpilogue = 5,      // epilogue warps (summed over warps)
  kTrEpilogueWait = 6,  //   of which waiting for finished accumulators
  kTrCtas = 7,          // CTAs that ran
  kTrMmaCtas = 8,       // CTAs whose thread issued MMAs
  kTrSlots = 9
};

// mbar_wait that adds its cycles to `acc` when kOn.
template <bool kOn>
__device__ __forceinline__ bool timed_wait(long long& acc, uint64_t* bar, uint32_t parity,
                                           int* err, int code) {
  if constexpr (kOn) {
    const long long t0 = clock64();
    const bool r = mbar_wait(bar, parity, err, code);
    acc += clock64() - t0;
    return r;
  } else {
    return mbar_wait(bar, parity, err, code);
  }
}

// Called by lane 0 of every warp at the end of a traced launch: warp 0 is
// the producer, warp 1 the MMA issuer (when `issues`), warps 2.. the
// epilogue; w1 / w2 are the role's waits in slot order.
__device__ __forceinline__ void trace_role(unsigned long long* slots, int warp, bool issues,
                                           long long start, long long w1, long long w2) {
  const unsigned long long total = (unsigned long long)(clock64() - start);
  if (warp == 0) {
    atomicAdd(&slots[kTrProducer], total);
    atomicAdd(&slots[kTrProducerWait], (unsigned long long)w1);
    atomicAdd(&slots[kTrCtas], 1ull);
  } else if (warp == 1) {
    if (issues) {
      atomicAdd(&slots[kTrMma], total);
      atomicAdd(&slots[kTrMmaWaitFull], (unsigned long long)w1);
      atomicAdd(&slots[kTrMmaWaitAcc], (unsigned long long)w2);
      atomicAdd(&slots[kTrMmaCtas], 1ull);
    }
  } else {
    atomicAdd(&slots[kTrEpilogue], total);
    atomicAdd(&slots[kTrEpilogueWait], (unsigned long long)w1);
  }
}

}  // namespace tc
}  // namespace gsht
