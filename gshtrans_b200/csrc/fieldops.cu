// Fused pointwise evaluation of canonical-component field expressions.
//
// Replaces the materialising assignment of the reference's expression
// templates (CanonicalComponentFieldBase.h:201-211 and the compound forms
// :222-339), which walk every grid point serially and evaluate the lazy node
// tree (CanonicalComponentFieldBinary.h:100-305: + - * /;
// CanonicalComponentFieldUnary.h:103-354: conj, real, imag, unary functions;
// CanonicalComponentFieldOverloads.h:22-262: scalar forms). Here the tree is
// flattened by the host into a short postfix program that one kernel runs
// per grid point over a small stack: every input is read once (a complex
// value with one 128-bit load, a real value with one 64-bit load) and the
// result is written once, so the whole expression costs one pass over HBM.
#include <cstring>
#include <mutex>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

constexpr int kMaxOps = 64;
constexpr int kMaxInputs = 16;
constexpr int kMaxStack = 8;

struct Program {
  int nops, ninputs, outReal;
  int op[kMaxOps];
  int arg[kMaxOps];
  double re[kMaxOps], im[kMaxOps];
  int inReal[kMaxInputs];
  const void* in[kMaxInputs];
  void* out;
  long long npoints, stride;  // points per field, element stride between fields
  int count;
};

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // Smith's algorithm, as std::complex division avoids overflow.
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + r * b.y;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.y + r * b.x;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

template <int N>
struct Depth {
  static constexpr int value = N;
};

// Calls f(Depth<d>{}) for the run-time depth d (warp-uniform: every thread
// runs the same program), so that the stack slots f touches are compile-time
// indices and the stack stays in registers.
#define GSHT_DEPTH_CASE(k)                 \
  case k:                                  \
    if constexpr (k < kCap) f(Depth<k>{}); \
    break;
template <int kCap, typename F>
__device__ __forceinline__ void with_depth(int d, F&& f) {
  switch (d) {
    GSHT_DEPTH_CASE(0)
    GSHT_DEPTH_CASE(1)
    GSHT_DEPTH_CASE(2)
    GSHT_DEPTH_CASE(3)
    GSHT_DEPTH_CASE(4)
    GSHT_DEPTH_CASE(5)
    GSHT_DEPTH_CASE(6)
    GSHT_DEPTH_CASE(7)
    default:
      break;
  }
}
#undef GSHT_DEPTH_CASE

__device__ __forceinline__ double2 apply_binary(int op, double2 a, double2 b) {
  if (op == GSHT_OP_ADD) return make_double2(a.x + b.x, a.y + b.y);
  if (op == GSHT_OP_SUB) return make_double2(a.x - b.x, a.y - b.y);
  if (op == GSHT_OP_MUL) return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  return cdiv(a, b);
}

__device__ __forceinline__ double2 apply_unary(int op, double2 a) {
  if (op == GSHT_OP_NEG) return make_double2(-a.x, -a.y);
  if (op == GSHT_OP_CONJ) return make_double2(a.x, -a.y);
  if (op == GSHT_OP_REAL) return make_double2(a.x, 0.0);
  return make_double2(a.y, 0.0);  // GSHT_OP_IMAG
}

// One pass over the fields: blockIdx.y walks the fields, the x dimension the
// points of a field; each thread evaluates kP points spaced one grid-width
// apart (every warp access is 32 consecutive points), issuing the loads of
// all kP points of a LOAD before the next operation. The value stack is
// kD x kP registers, addressed through with_depth.
template <int kD, int kP>
__global__ void __launch_bounds__(256) k_field_eval(const __grid_constant__ Program p) {
  const long long width = (long long)gridDim.x * blockDim.x;
  for (long long f = blockIdx.y; f < p.count; f += gridDim.y) {
    const long long fieldBase = f * p.stride;
    for (long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; i0 < p.npoints;
         i0 += width * kP) {
      bool ok[kP];
#pragma unroll
      for (int j = 0; j < kP; j++) ok[j] = i0 + j * width < p.npoints;
      double2 st[kD][kP];
      int depth = 0;
      for (int k = 0; k < p.nops; k++) {
        const int op = p.op[k];
        if (op == GSHT_OP_LOAD) {
          const int a = p.arg[k];
          const bool real = p.inReal[a];
          const void* src = p.in[a];
          with_depth<kD>(depth, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) {
              const long long idx = fieldBase + i0 + j * width;
              double2 v = make_double2(0.0, 0.0);
              if (ok[j]) {
                v = real ? make_double2(__ldg(static_cast<const double*>(src) + idx), 0.0)
                         : __ldg(static_cast<const double2*>(src) + idx);
              }
              st[d][j] = v;
            }
          });
          depth++;
        } else if (op == GSHT_OP_CONST) {
          const double2 c = make_double2(p.re[k], p.im[k]);
          with_depth<kD>(depth, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) st[d][j] = c;
          });
          depth++;
        } else if (op >= GSHT_OP_NEG) {
          with_depth<kD>(depth - 1, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) st[d][j] = apply_unary(op, st[d][j]);
          });
        } else {
          with_depth<kD>(depth - 2, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
            if constexpr (d + 1 < kD) {
#pragma unroll
              for (int j = 0; j < kP; j++) st[d][j] = apply_binary(op, st[d][j], st[d + 1][j]);
            }
          });
          depth--;
        }
      }
#pragma unroll
      for (int j = 0; j < kP; j++) {
        if (!ok[j]) continue;
        const long long idx = fieldBase + i0 + j * width;
        if (p.outReal) {
          static_cast<double*>(p.out)[idx] = st[0][j].x;
        } else {
          static_cast<double2*>(p.out)[idx] = st[0][j];
        }
      }
    }
  }
}


// Streaming form: the inputs of a chunk of points reach shared memory by
// 1-D bulk copies (cp.async.bulk, completion counted on an mbarrier) issued
// by one producer warp kStagesF chunks ahead, so that the loads of later
// chunks are in flight while eight warps evaluate the program on the current
// one from shared memory (one point per thread per step, the value stack in
// registers as above) and store the results straight to global memory.
constexpr int kStagesF = 3;
constexpr int kEvalWarps = 8;
constexpr int kStageBudget = 32 * 1024;  // shared bytes per stage (two blocks per SM)

// Set when a wait of the streaming kernel ran out (reported by host-buffer calls).
__device__ int g_field_wait_err = 0;

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(tc::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
      : "memory");
}

template <int kD, int kP>
__global__ void __launch_bounds__(32 * (kEvalWarps + 1), 2)
    k_field_eval_stream(const __grid_constant__ Program p, int chunk, int stageBytes) {
  extern __shared__ __align__(128) unsigned char fsm[];
  uint64_t* full = reinterpret_cast<uint64_t*>(fsm + kStagesF * stageBytes);
  uint64_t* empty = full + kStagesF;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long perField = (p.npoints + chunk - 1) / chunk;
  const long long total = perField * p.count;
  // Offsets of the inputs inside a stage (16-byte aligned: chunk is a
  // multiple of 256 points).
  __shared__ int off[kMaxInputs];
  if (threadIdx.x == 0) {
    int o = 0;
    for (int a = 0; a < p.ninputs; a++) {
      off[a] = o;
      o += chunk * (p.inReal[a] ? 8 : 16);
    }
    for (int s = 0; s < kStagesF; s++) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], kEvalWarps);
    }
    tc::fence_barrier_init();
  }
  __syncthreads();
  if (warp == kEvalWarps) {
    if (lane == 0) {
      int it = 0;
      for (long long ch = blockIdx.x; ch < total; ch += gridDim.x, it++) {
        const int s = it % kStagesF;
        if (it >= kStagesF &&
            !tc::mbar_wait(&empty[s], ((it / kStagesF) - 1) & 1, &g_field_wait_err, 1))
          break;
        const long long f = ch / perField;
        const long long p0 = (ch - f * perField) * chunk;
        const long long rem = p.npoints - p0;
        const int n = rem < chunk ? (int)rem : chunk;
        uint32_t bytes = 0;
        for (int a = 0; a < p.ninputs; a++) bytes += (uint32_t)n * (p.inReal[a] ? 8 : 16);
        tc::mbar_arrive_expect_tx(&full[s], bytes);
        unsigned char* st = fsm + s * stageBytes;
        for (int a = 0; a < p.ninputs; a++) {
          const int esz = p.inReal[a] ? 8 : 16;
          const unsigned char* src =
              static_cast<const unsigned char*>(p.in[a]) + (f * p.stride + p0) * esz;
          bulk_g2s(st + off[a], src, (uint32_t)(n * esz), &full[s]);
        }
      }
    }
    return;
  }
  // Each thread evaluates kP points of a chunk per pass (256 apart), so that
  // one dispatch of an operation serves kP points.
  constexpr int kStride = 32 * kEvalWarps;
  int it = 0;
  for (long long ch = blockIdx.x; ch < total; ch += gridDim.x, it++) {
    const int s = it % kStagesF;
    if (!tc::mbar_wait(&full[s], (it / kStagesF) & 1, &g_field_wait_err, 2)) break;
    const long long f = ch / perField;
    const long long p0 = (ch - f * perField) * chunk;
    const long long rem = p.npoints - p0;
    const int n = rem < chunk ? (int)rem : chunk;
    const unsigned char* st = fsm + s * stageBytes;
    for (int i0 = threadIdx.x; i0 < n; i0 += kStride * kP) {
      double2 stk[kD][kP];
      int depth = 0;
      for (int k = 0; k < p.nops; k++) {
        const int op = p.op[k];
        if (op == GSHT_OP_LOAD) {
          const int a = p.arg[k];
          const bool real = p.inReal[a];
          const unsigned char* src = st + off[a];
          with_depth<kD>(depth, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) {
              const int i = i0 + j * kStride;
              double2 v = make_double2(0.0, 0.0);
              if (i < n)
                v = real ? make_double2(reinterpret_cast<const double*>(src)[i], 0.0)
                         : reinterpret_cast<const double2*>(src)[i];
              stk[d][j] = v;
            }
          });
          depth++;
        } else if (op == GSHT_OP_CONST) {
          const double2 c = make_double2(p.re[k], p.im[k]);
          with_depth<kD>(depth, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) stk[d][j] = c;
          });
          depth++;
        } else if (op >= GSHT_OP_NEG) {
          with_depth<kD>(depth - 1, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
#pragma unroll
            for (int j = 0; j < kP; j++) stk[d][j] = apply_unary(op, stk[d][j]);
          });
        } else {
          with_depth<kD>(depth - 2, [&](auto dc) {
            constexpr int d = decltype(dc)::value;
            if constexpr (d + 1 < kD) {
#pragma unroll
              for (int j = 0; j < kP; j++) stk[d][j] = apply_binary(op, stk[d][j], stk[d + 1][j]);
            }
          });
          depth--;
        }
      }
#pragma unroll
      for (int j = 0; j < kP; j++) {
        const int i = i0 + j * kStride;
        if (i >= n) continue;
        const long long idx = f * p.stride + p0 + i;
        if (p.outReal) {
          static_cast<double*>(p.out)[idx] = stk[0][j].x;
        } else {
          static_cast<double2*>(p.out)[idx] = stk[0][j];
        }
      }
    }
    __syncwarp();
    if (lane == 0) tc::mbar_arrive(&empty[s]);
  }
}

std::mutex g_stage_mu;
void* g_stage = nullptr;
size_t g_stage_bytes = 0;

}  // namespace
}  // namespace gsht

using namespace gsht;

extern "C" gsht_status gsht_field_eval(const gsht_expr_op* program, int nops,
                                       const void* const* inputs, const int* input_is_real,
                                       int ninputs, void* out, int out_is_real, long npoints,
                                       int count, long field_stride, void* stream) {
  if (!program || nops < 1 || nops > kMaxOps)
    return fail(GSHT_ERR_BAD_ARG, "program must hold 1..%d operations", kMaxOps);
  if (ninputs < 0 || ninputs > kMaxInputs || (ninputs && (!inputs || !input_is_real)))
    return fail(GSHT_ERR_BAD_ARG, "between 0 and %d inputs", kMaxInputs);
  if (!out || npoints < 1 || count < 1 || field_stride < npoints)
    return fail(GSHT_ERR_BAD_ARG, "bad output, point count, field count or stride");
  Program p{};
  p.nops = nops;
  p.ninputs = ninputs;
  p.outReal = out_is_real ? 1 : 0;
  int depth = 0, maxDepth = 0;
  for (int k = 0; k < nops; k++) {
    const int op = program[k].op;
    p.op[k] = op;
    p.arg[k] = program[k].arg;
    p.re[k] = program[k].re;
    p.im[k] = program[k].im;
    if (op == GSHT_OP_LOAD) {
      if (program[k].arg < 0 || program[k].arg >= ninputs)
        return fail(GSHT_ERR_BAD_ARG, "operation %d loads input %d of %d", k, program[k].arg, ninputs);
      depth++;
    } else if (op == GSHT_OP_CONST) {
      depth++;
    } else if (op >= GSHT_OP_ADD && op <= GSHT_OP_DIV) {
      if (depth < 2) return fail(GSHT_ERR_BAD_ARG, "operation %d needs two operands", k);
      depth--;
    } else if (op >= GSHT_OP_NEG && op <= GSHT_OP_IMAG) {
      if (depth < 1) return fail(GSHT_ERR_BAD_ARG, "operation %d needs an operand", k);
    } else {
      return fail(GSHT_ERR_BAD_ARG, "unknown operation code %d", op);
    }
    maxDepth = depth > maxDepth ? depth : maxDepth;
  }
  if (depth != 1) return fail(GSHT_ERR_BAD_ARG, "program leaves %d values on the stack", depth);
  if (maxDepth > kMaxStack) return fail(GSHT_ERR_BAD_ARG, "program needs a deeper stack than %d", kMaxStack);
  for (int a = 0; a < ninputs; a++) {
    if (!inputs[a]) return fail(GSHT_ERR_BAD_ARG, "input %d is NULL", a);
    p.in[a] = inputs[a];
    p.inReal[a] = input_is_real[a] ? 1 : 0;
  }
  p.out = out;
  p.npoints = npoints;
  p.stride = field_stride;
  p.count = count;
  int dev = 0;
  GSHT_CUDA(cudaGetDevice(&dev));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // Host buffers (e.g. fields stored in host vectors, as the reference's are)
  // are staged through a device workspace kept by the library; the call then
  // returns with the result in host memory.
  const PtrKind outKind = pointer_kind(out, dev);
  bool anyHost = outKind == kHostPtr, anyOther = outKind == kOtherDevicePtr;
  for (int a = 0; a < ninputs; a++) {
    const PtrKind k = pointer_kind(inputs[a], dev);
    anyHost = anyHost || k == kHostPtr;
    anyOther = anyOther || k == kOtherDevicePtr;
  }
  if (anyOther) return fail(GSHT_ERR_BAD_ARG, "a buffer lives on another GPU than the current one (%d)", dev);
  std::unique_lock<std::mutex> lk(g_stage_mu, std::defer_lock);
  const size_t span = (size_t)field_stride * (count - 1) + (size_t)npoints;
  if (anyHost) {
    lk.lock();
    const size_t need = (size_t)(ninputs + 1) * round_up(sizeof(double) * 2 * span, 256);
    if (g_stage_bytes < need) {
      GSHT_CUDA(cudaDeviceSynchronize());
      dev_free(g_stage);
      g_stage = nullptr;
      g_stage_bytes = 0;
      if (dev_malloc(&g_stage, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(GSHT_ERR_OOM, "field staging allocation of %zu bytes failed", need);
      }
      g_stage_bytes = need;
    }
    char* base = static_cast<char*>(g_stage);
    const size_t slot = round_up(sizeof(double) * 2 * span, 256);
    for (int a = 0; a < ninputs; a++) {
      if (pointer_kind(inputs[a], dev) == kDevicePtr) continue;
      const size_t bytes = sizeof(double) * (p.inReal[a] ? 1 : 2) * span;
      GSHT_CUDA(cudaMemcpyAsync(base + a * slot, inputs[a], bytes, cudaMemcpyHostToDevice, s));
      p.in[a] = base + a * slot;
    }
    if (outKind == kHostPtr) p.out = base + ninputs * slot;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Streaming form when every input chunk can be bulk-copied: 16-byte
  // aligned buffers, and for real inputs an even point count and stride
  // (chunk starts then stay 16-byte aligned).
  bool streamed = ninputs > 0;
  int bpp = 0;  // input bytes per point
  for (int a = 0; a < ninputs; a++) {
    const int esz = p.inReal[a] ? 8 : 16;
    bpp += esz;
    streamed = streamed && (reinterpret_cast<uintptr_t>(p.in[a]) % 16 == 0);
    if (p.inReal[a]) streamed = streamed && npoints % 2 == 0 && field_stride % 2 == 0;
  }
  if (streamed) {
    const int threads = 32 * (kEvalWarps + 1);
    // Shallow programs: 2 points per thread per pass over chunks of 512
    // points; deeper ones 1 point (the 8-slot stack) over chunks of 256.
    const bool shallow = maxDepth <= 4;
    const int unit = shallow ? 512 : 256;
    int k = kStageBudget / (unit * bpp);
    if (k < 1) k = 1;
    const int chunk = unit * k;
    const int stageBytes = chunk * bpp;
    const size_t smem = (size_t)kStagesF * stageBytes + 2 * kStagesF * sizeof(uint64_t);
    auto kern = shallow ? k_field_eval_stream<4, 2> : k_field_eval_stream<kMaxStack, 1>;
    GSHT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int perSm = 0;
    GSHT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, threads, smem));
    if (perSm < 1) perSm = 1;
    const long long chunks = ((long long)npoints + chunk - 1) / chunk * count;
    long long blocks = (long long)sms * perSm;
    if (blocks > chunks) blocks = chunks;
    kern<<<(unsigned)blocks, threads, smem, s>>>(p, chunk, stageBytes);
    GSHT_LAUNCH_CHECK("k_field_eval_stream");
    if (anyHost) {
      if (p.out != out)
        GSHT_CUDA(cudaMemcpyAsync(out, p.out, sizeof(double) * (p.outReal ? 1 : 2) * span,
                                  cudaMemcpyDeviceToHost, s));
      GSHT_CUDA(cudaStreamSynchronize(s));
      int werr = 0;
      GSHT_CUDA(cudaMemcpyFromSymbol(&werr, g_field_wait_err, sizeof(int)));
      if (werr) {
        const int zero = 0;
        GSHT_CUDA(cudaMemcpyToSymbol(g_field_wait_err, &zero, sizeof(int)));
        return fail(GSHT_ERR_TIMEOUT, "a bounded wait of the field kernel expired");
      }
    }
    return GSHT_OK;
  }
  // Programs up to 4 deep (the usual field expressions) run 4 points per
  // thread with a 4 x 4 register stack; deeper ones 1 point with 8 slots.
  const bool shallow = maxDepth <= 4;
  const int per = shallow ? 4 : 1;
  const long long perField = ((long long)npoints + 256LL * per - 1) / (256LL * per);
  const long long want = (long long)sms * 8;  // blocks in flight for the whole launch
  long long bx = perField;
  long long by = count;
  if (by > 65535) by = 65535;
  if (bx * by > want) bx = (want + by - 1) / by;
  if (bx < 1) bx = 1;
  const dim3 grid((unsigned)bx, (unsigned)by);
  if (shallow) {
    k_field_eval<4, 4><<<grid, 256, 0, s>>>(p);
  } else {
    k_field_eval<kMaxStack, 1><<<grid, 256, 0, s>>>(p);
  }
  GSHT_LAUNCH_CHECK("k_field_eval");
  if (anyHost) {
    if (p.out != out)
      GSHT_CUDA(cudaMemcpyAsync(out, p.out, sizeof(double) * (p.outReal ? 1 : 2) * span,
                                cudaMemcpyDeviceToHost, s));
    GSHT_CUDA(cudaStreamSynchronize(s));
  }
  return GSHT_OK;
}
