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

namespace gsht {
namespace {

constexpr int kMaxOps = 32;
constexpr int kMaxInputs = 8;
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

__device__ __forceinline__ double2 eval_point(const Program& p, long long f, long long i) {
  double2 st[kMaxStack];
  int sp = 0;
  for (int k = 0; k < p.nops; k++) {
    const int op = p.op[k];
    switch (op) {
      case GSHT_OP_LOAD: {
        const int a = p.arg[k];
        const long long idx = f * p.stride + i;
        st[sp++] = p.inReal[a]
                       ? make_double2(__ldg(static_cast<const double*>(p.in[a]) + idx), 0.0)
                       : __ldg(static_cast<const double2*>(p.in[a]) + idx);
        break;
      }
      case GSHT_OP_CONST:
        st[sp++] = make_double2(p.re[k], p.im[k]);
        break;
      case GSHT_OP_NEG:
        st[sp - 1] = make_double2(-st[sp - 1].x, -st[sp - 1].y);
        break;
      case GSHT_OP_CONJ:
        st[sp - 1].y = -st[sp - 1].y;
        break;
      case GSHT_OP_REAL:
        st[sp - 1].y = 0.0;
        break;
      case GSHT_OP_IMAG:
        st[sp - 1] = make_double2(st[sp - 1].y, 0.0);
        break;
      default: {
        const double2 b = st[--sp], a = st[sp - 1];
        double2 r;
        if (op == GSHT_OP_ADD) r = make_double2(a.x + b.x, a.y + b.y);
        else if (op == GSHT_OP_SUB) r = make_double2(a.x - b.x, a.y - b.y);
        else if (op == GSHT_OP_MUL) r = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        else r = cdiv(a, b);
        st[sp - 1] = r;
      }
    }
  }
  return st[0];
}

__global__ void __launch_bounds__(256) k_field_eval(const __grid_constant__ Program p) {
  const long long total = p.npoints * p.count;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long f = t / p.npoints, i = t - f * p.npoints;
    const double2 v = eval_point(p, f, i);
    const long long idx = f * p.stride + i;
    if (p.outReal) {
      static_cast<double*>(p.out)[idx] = v.x;
    } else {
      static_cast<double2*>(p.out)[idx] = v;
    }
  }
}

bool on_device(const void* ptr) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
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
  bool anyHost = !on_device(out);
  for (int a = 0; a < ninputs; a++) anyHost = anyHost || !on_device(inputs[a]);
  std::unique_lock<std::mutex> lk(g_stage_mu, std::defer_lock);
  const size_t span = (size_t)field_stride * (count - 1) + (size_t)npoints;
  if (anyHost) {
    lk.lock();
    const size_t need = (size_t)(ninputs + 1) * round_up(sizeof(double) * 2 * span, 256);
    if (g_stage_bytes < need) {
      GSHT_CUDA(cudaDeviceSynchronize());
      cudaFree(g_stage);
      g_stage = nullptr;
      g_stage_bytes = 0;
      if (cudaMalloc(&g_stage, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(GSHT_ERR_OOM, "field staging allocation of %zu bytes failed", need);
      }
      g_stage_bytes = need;
    }
    char* base = static_cast<char*>(g_stage);
    const size_t slot = round_up(sizeof(double) * 2 * span, 256);
    for (int a = 0; a < ninputs; a++) {
      if (on_device(inputs[a])) continue;
      const size_t bytes = sizeof(double) * (p.inReal[a] ? 1 : 2) * span;
      GSHT_CUDA(cudaMemcpyAsync(base + a * slot, inputs[a], bytes, cudaMemcpyHostToDevice, s));
      p.in[a] = base + a * slot;
    }
    if (!on_device(out)) p.out = base + ninputs * slot;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long total = (long long)npoints * count;
  long long blocks = (total + 255) / 256;
  if (blocks > (long long)sms * 16) blocks = (long long)sms * 16;
  k_field_eval<<<(unsigned)blocks, 256, 0, s>>>(p);
  GSHT_LAUNCH_CHECK("k_field_eval");
  if (anyHost) {
    if (p.out != out)
      GSHT_CUDA(cudaMemcpyAsync(out, p.out, sizeof(double) * (p.outReal ? 1 : 2) * span,
                                cudaMemcpyDeviceToHost, s));
    GSHT_CUDA(cudaStreamSynchronize(s));
  }
  return GSHT_OK;
}
