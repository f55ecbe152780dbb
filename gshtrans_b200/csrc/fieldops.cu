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
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

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
          tc::bulk_load(st + off[a], src, (uint32_t)(n * esz), &full[s]);
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

// ---------------------------------------------------------------------------
// Compiled form: the program is turned into CUDA C++ source (one statement per
// operation, every input loaded once per point however often the program
// reads it) and compiled for the device with NVRTC the first time it is seen;
// the kernel is cached per (device, source). Each thread evaluates four
// points 256 apart per pass, with all their loads issued before the
// arithmetic; complex values move as 128-bit loads and stores. The arithmetic
// is written as the interpreter's (the same complex product, Smith's division),
// compiled with the same contraction settings. Where NVRTC cannot be loaded
// or a program fails to compile, the interpreting kernels above run instead;
// GSHT_FIELD_JIT=0 selects them for comparisons.
// ---------------------------------------------------------------------------
struct JitArgs {
  const void* in[kMaxInputs];
  void* out;
  long long npoints, stride;
};

constexpr int kJitThreads = 256, kJitPoints = 4;

struct Nvrtc {
  bool ok = false;
  nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                        const char* const*) = nullptr;
  nvrtcResult (*compile)(nvrtcProgram, int, const char* const*) = nullptr;
  nvrtcResult (*cubinSize)(nvrtcProgram, size_t*) = nullptr;
  nvrtcResult (*cubin)(nvrtcProgram, char*) = nullptr;
  nvrtcResult (*destroy)(nvrtcProgram*) = nullptr;
};

const Nvrtc& nvrtc() {
  static Nvrtc n;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
    n.cubinSize = reinterpret_cast<decltype(n.cubinSize)>(dlsym(h, "nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.cubinSize && n.cubin && n.destroy;
  });
  return n;
}

// A double as an exact source literal.
std::string dlit(double v) {
  unsigned long long b;
  std::memcpy(&b, &v, sizeof b);
  char buf[64];
  std::snprintf(buf, sizeof buf, "__longlong_as_double(0x%016llxLL)", b);
  return buf;
}

std::string jit_source(const Program& p) {
  std::string s =
      "struct JitArgs { const void* in[" + std::to_string(kMaxInputs) + "]; void* out;"
      " long long npoints, stride; };\n"
      "__device__ __forceinline__ double2 cmul(double2 a, double2 b) {\n"
      "  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);\n}\n"
      "__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {\n"
      "  if (fabs(b.x) >= fabs(b.y)) {\n"
      "    const double r = b.y / b.x, d = b.x + r * b.y;\n"
      "    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);\n  }\n"
      "  const double r = b.x / b.y, d = b.y + r * b.x;\n"
      "  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);\n}\n"
      "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(kJitThreads) +
      ") gsht_field_jit(JitArgs p) {\n"
      "  const long long base = (long long)blockIdx.y * p.stride;\n"
      "  for (long long i0 = (long long)blockIdx.x * " + std::to_string(kJitThreads * kJitPoints) +
      " + threadIdx.x; i0 < p.npoints; i0 += (long long)gridDim.x * " +
      std::to_string(kJitThreads * kJitPoints) + ") {\n";
  const std::string P = std::to_string(kJitPoints), T = std::to_string(kJitThreads);
  // Every input the program reads, loaded once per point.
  std::vector<int> used(p.ninputs, 0);
  for (int k = 0; k < p.nops; k++)
    if (p.op[k] == GSHT_OP_LOAD) used[p.arg[k]] = 1;
  for (int a = 0; a < p.ninputs; a++) {
    if (!used[a]) continue;
    const std::string A = std::to_string(a);
    s += "    double2 in" + A + "[" + P + "];\n";
    s += "    #pragma unroll\n    for (int j = 0; j < " + P + "; j++) {\n";
    s += "      const long long i = i0 + " + T + " * j;\n";
    if (p.inReal[a])
      s += "      in" + A + "[j] = i < p.npoints ? make_double2(static_cast<const double*>(p.in[" + A +
           "])[base + i], 0.0) : make_double2(0.0, 0.0);\n";
    else
      s += "      in" + A + "[j] = i < p.npoints ? static_cast<const double2*>(p.in[" + A +
           "])[base + i] : make_double2(0.0, 0.0);\n";
    s += "    }\n";
  }
  s += "    #pragma unroll\n    for (int j = 0; j < " + P + "; j++) {\n";
  s += "      const long long i = i0 + " + T + " * j;\n      if (i >= p.npoints) break;\n";
  std::vector<std::string> stk;
  int tmp = 0;
  auto fresh = [&](const std::string& expr) {
    const std::string name = "t" + std::to_string(tmp++);
    s += "      const double2 " + name + " = " + expr + ";\n";
    stk.push_back(name);
  };
  for (int k = 0; k < p.nops; k++) {
    const int op = p.op[k];
    if (op == GSHT_OP_LOAD) {
      stk.push_back("in" + std::to_string(p.arg[k]) + "[j]");
    } else if (op == GSHT_OP_CONST) {
      fresh("make_double2(" + dlit(p.re[k]) + ", " + dlit(p.im[k]) + ")");
    } else if (op >= GSHT_OP_NEG) {
      const std::string a = stk.back();
      stk.pop_back();
      if (op == GSHT_OP_NEG) fresh("make_double2(-" + a + ".x, -" + a + ".y)");
      else if (op == GSHT_OP_CONJ) fresh("make_double2(" + a + ".x, -" + a + ".y)");
      else if (op == GSHT_OP_REAL) fresh("make_double2(" + a + ".x, 0.0)");
      else fresh("make_double2(" + a + ".y, 0.0)");
    } else {
      const std::string b = stk.back();
      stk.pop_back();
      const std::string a = stk.back();
      stk.pop_back();
      if (op == GSHT_OP_ADD) fresh("make_double2(" + a + ".x + " + b + ".x, " + a + ".y + " + b + ".y)");
      else if (op == GSHT_OP_SUB) fresh("make_double2(" + a + ".x - " + b + ".x, " + a + ".y - " + b + ".y)");
      else if (op == GSHT_OP_MUL) fresh("cmul(" + a + ", " + b + ")");
      else fresh("cdiv(" + a + ", " + b + ")");
    }
  }
  if (p.outReal)
    s += "      static_cast<double*>(p.out)[base + i] = " + stk.back() + ".x;\n";
  else
    s += "      static_cast<double2*>(p.out)[base + i] = " + stk.back() + ";\n";
  s += "    }\n  }\n}\n";
  return s;
}

std::mutex g_jit_mu;
std::map<std::pair<int, std::string>, cudaKernel_t> g_jit_kernels;  // null: failed to build

// The cached compiled kernel of p on device dev (compiled on first use), or
// null when NVRTC is unavailable or the program does not compile.
cudaKernel_t jit_kernel(const Program& p, int dev) {
  const char* e = getenv("GSHT_FIELD_JIT");
  if (e && e[0] == '0') return nullptr;
  const Nvrtc& nv = nvrtc();
  if (!nv.ok) return nullptr;
  const std::string src = jit_source(p);
  std::lock_guard<std::mutex> lk(g_jit_mu);
  const auto key = std::make_pair(dev, src);
  auto it = g_jit_kernels.find(key);
  if (it != g_jit_kernels.end()) return it->second;
  cudaKernel_t kern = nullptr;
  nvrtcProgram prog = nullptr;
  if (nv.create(&prog, src.c_str(), "gsht_field_jit.cu", 0, nullptr, nullptr) == NVRTC_SUCCESS) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, dev);
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(prop.major * 10 + prop.minor) +
                             (prop.major >= 9 ? "a" : "");
    const char* opts[] = {arch.c_str(), "--std=c++17"};
    size_t n = 0;
    if (nv.compile(prog, 2, opts) == NVRTC_SUCCESS && nv.cubinSize(prog, &n) == NVRTC_SUCCESS &&
        n > 0) {
      std::vector<char> cubin(n);
      cudaLibrary_t lib = nullptr;
      if (nv.cubin(prog, cubin.data()) == NVRTC_SUCCESS &&
          cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) ==
              cudaSuccess &&
          cudaLibraryGetKernel(&kern, lib, "gsht_field_jit") != cudaSuccess) {
        kern = nullptr;
      }
      cudaGetLastError();
    }
    nv.destroy(&prog);
  }
  g_jit_kernels[key] = kern;
  return kern;
}

// Runs p through its compiled kernel; false when there is none (the caller
// then interprets it).
bool jit_launch(const Program& p, int dev, int sms, cudaStream_t s, gsht_status* st) {
  if (p.count > 65535) return false;
  cudaKernel_t kern = jit_kernel(p, dev);
  if (!kern) return false;
  JitArgs a{};
  for (int i = 0; i < p.ninputs; i++) a.in[i] = p.in[i];
  a.out = p.out;
  a.npoints = p.npoints;
  a.stride = p.stride;
  const long long per = (long long)kJitThreads * kJitPoints;
  long long bx = (p.npoints + per - 1) / per;
  const long long cap = ((long long)sms * 8 + p.count - 1) / p.count;
  if (bx > cap) bx = cap < 1 ? 1 : cap;
  void* args[] = {&a};
  const cudaError_t e = cudaLaunchKernel(reinterpret_cast<const void*>(kern),
                                         dim3((unsigned)bx, (unsigned)p.count), dim3(kJitThreads),
                                         args, 0, s);
  if (e != cudaSuccess) {
    *st = cuda_fail(e, "compiled field kernel launch");
    return true;
  }
  t_launches++;
  g_launches++;
  *st = GSHT_OK;
  return true;
}

std::mutex g_stage_mu;
void* g_stage = nullptr;
size_t g_stage_bytes = 0;

}  // namespace
}  // namespace gsht

using namespace gsht;

extern "C" gsht_status gsht_field_jit_stats(int* compiled, int* failed) {
  std::lock_guard<std::mutex> lk(g_jit_mu);
  int c = 0, f = 0;
  for (const auto& kv : g_jit_kernels) (kv.second ? c : f)++;
  if (compiled) *compiled = c;
  if (failed) *failed = f;
  return GSHT_OK;
}

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
  gsht_status jst = GSHT_OK;
  if (jit_launch(p, dev, sms, s, &jst)) {
    if (jst != GSHT_OK) return jst;
    if (anyHost) {
      if (p.out != out)
        GSHT_CUDA(cudaMemcpyAsync(out, p.out, sizeof(double) * (p.outReal ? 1 : 2) * span,
                                  cudaMemcpyDeviceToHost, s));
      GSHT_CUDA(cudaStreamSynchronize(s));
    }
    return GSHT_OK;
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
