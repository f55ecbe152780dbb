// Batched transforms of many fields of uneven sizes in one CUDA graph.
//
// No counterpart in the reference, whose transforms take one field per call
// (GaussLegendreGrid.h:108-321); a caller with many fields loops over them.
// Here a plan takes a list of fields, each with its own degree lmax (and so
// its own Gauss-Legendre grid nTheta = lmax + 1, nPhi = 2 lmax), upper index
// and kind, and
//   - groups them by (lmax, n, real/complex): one grid per distinct lmax,
//     whose Wigner tables (one per upper index) every field of that degree
//     shares, and one batched transform per group (each stage runs once over
//     the group and reads the table once);
//   - gathers each group's inputs from the callers' buffers into contiguous
//     batch buffers and scatters the results back (the forward adds into the
//     callers' coefficients, as ForwardTransformation does);
//   - autotunes, for the BF16x3 form, the field-row tile width of the
//     tensor-core kernels per group (32, 64 or 128 columns: small groups
//     waste fewer MMA columns with narrow tiles) by timing each candidate;
//   - gives every group its own workspace, so that groups run concurrently
//     on several streams (groups of the same degree share only read-only
//     tables), and autotunes that schedule too: the number of streams the
//     groups are spread over (largest groups first), by timing the captured
//     round-trip graph of each candidate;
//   - captures the whole sequence (gathers, transforms, scatters) for each
//     direction into a CUDA graph, so an execution is one graph launch;
//   - for the BF16x3 form, runs each direction's Legendre stage as ONE
//     persistent tensor-core launch over the (group, order, tile) work list
//     of all groups (every group's tensor maps and arguments in device
//     memory), between the per-group operand preparations / ring FFTs, which
//     run concurrently on the plan's streams; the field-row tile width of
//     that launch is autotuned (GSHT_BATCH_FUSED=0 keeps one transform per
//     group, for comparisons).
#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "gsht_internal.cuh"

namespace gsht {
namespace {

constexpr int kMaxLanes = 16;  // streams a batch graph spreads its groups over

// Copies `count` vectors of `elems` 16-byte elements between callers'
// buffers and a contiguous batch buffer; mode 0: gather (dst contiguous),
// 1: scatter (src contiguous), 2: scatter-add (src contiguous, dst += src),
// 3: scatter-add with the last element set to 0 (the c_{L,L} = 0 rule the
// forward applies to complex fields whose lmax is the grid degree,
// GaussLegendreGrid.h:209-215; it overwrites rather than adds). For real
// grids elems counts pairs of doubles (fields are nTheta*nPhi doubles; nPhi
// is even).
__global__ void k_batch_copy(int mode, long elems, double2* const* ptrs, double2* contiguous) {
  const int f = blockIdx.y;
  double2* user = ptrs[f];
  double2* flat = contiguous + (size_t)f * elems;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < elems;
       i += (long)gridDim.x * blockDim.x) {
    if (mode == 0) {
      flat[i] = user[i];
    } else if (mode == 1) {
      user[i] = flat[i];
    } else if (mode == 3 && i == elems - 1) {
      user[i] = make_double2(0.0, 0.0);
    } else {
      const double2 a = user[i], b = flat[i];
      user[i] = make_double2(a.x + b.x, a.y + b.y);
    }
  }
}

struct Group {
  int lmax = 0, n = 0, isReal = 0, ntile = 128;
  std::vector<int> fields;
  gsht_grid* grid = nullptr;
  long coefElems = 0, gridElems = 0;  // 16-byte elements per field
  double2* coefIn = nullptr;          // contiguous batch buffers
  double2* gridBuf = nullptr;
  double2* coefOut = nullptr;
  double2** coefInPtrs = nullptr;     // callers' pointers (device arrays)
  double2** gridPtrs = nullptr;
  double2** coefOutPtrs = nullptr;
  void* ws = nullptr;                 // private workspace of the group's transforms
  size_t wsBytes = 0;
  double* spec = nullptr;             // fused BF16x3 path: spectra / forward result rows
  void* op = nullptr;                 //   and the operand rows of either direction
  bool spec32 = false;                //   FP32 spectra (three-pass ring FFTs)
  double work = 0.0;                  // estimated cost (fields x lmax^3), for the schedule
};

}  // namespace
}  // namespace gsht

struct gsht_batch {
  int device = 0, precision = 0;
  std::vector<gsht_field_desc> fields;
  std::map<int, gsht_grid*> grids;  // by degree
  std::vector<gsht::Group> groups;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> lanes;     // streams the groups are spread over
  std::vector<cudaEvent_t> laneDone;   // join events (one per lane) and the fork event
  int nlanes = 1;                      // chosen by the schedule autotuner
  bool fused = false;                  // one Legendre launch over all groups (BF16x3)
  gsht::Bf16Multi multi[2];            // its work lists: [0] inverse, [1] forward
  int fusedTile = 64;                  // its field-row tile width (autotuned)
  cudaGraph_t graph[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
  size_t nodes[3] = {0, 0, 0};
};

namespace gsht {
namespace {

gsht_status copy_group(const Group& gr, int mode, long elems, double2** ptrs, double2* flat,
                       cudaStream_t s) {
  const int count = (int)gr.fields.size();
  long blocks = (elems + 255) / 256;
  blocks = blocks > 1184 ? 1184 : blocks;
  dim3 grid((unsigned)blocks, count);
  k_batch_copy<<<grid, 256, 0, s>>>(mode, elems, ptrs, flat);
  GSHT_LAUNCH_CHECK("k_batch_copy");
  return GSHT_OK;
}

// One direction for one group: 0 forward (grids -> coefficients, added into
// the callers' coefficients), 1 inverse (coefficients -> grids).
// `gather`/`scatter` select whether the callers' buffers are read/written.
gsht_status run_group(gsht_batch* b, Group& gr, int dir, bool gather, bool scatter, cudaStream_t s) {
  const int count = (int)gr.fields.size();
  gsht_status st;
  if (dir == 1) {
    if (gather && (st = copy_group(gr, 0, gr.coefElems, gr.coefInPtrs, gr.coefIn, s)) != GSHT_OK)
      return st;
    PrivateWorkspace pw{gr.ws, gr.wsBytes, nullptr};
    st = transform(gr.grid, 1, gr.lmax, gr.n, gr.isReal, b->precision, count, gr.coefIn,
                   gr.gridBuf, s, gr.ntile, &pw);
    if (st != GSHT_OK) return st;
    if (scatter && (st = copy_group(gr, 1, gr.gridElems, gr.gridPtrs, gr.gridBuf, s)) != GSHT_OK)
      return st;
  } else {
    if (gather && (st = copy_group(gr, 0, gr.gridElems, gr.gridPtrs, gr.gridBuf, s)) != GSHT_OK)
      return st;
    GSHT_CUDA(cudaMemsetAsync(gr.coefOut, 0, sizeof(double2) * gr.coefElems * count, s));
    PrivateWorkspace pw{gr.ws, gr.wsBytes, nullptr};
    st = transform(gr.grid, 0, gr.lmax, gr.n, gr.isReal, b->precision, count, gr.gridBuf,
                   gr.coefOut, s, gr.ntile, &pw);
    if (st != GSHT_OK) return st;
    // Every field's lmax is its grid's degree, so complex fields get c_{L,L} = 0.
    const int mode = gr.isReal ? 2 : 3;
    if (scatter && (st = copy_group(gr, mode, gr.coefElems, gr.coefOutPtrs, gr.coefOut, s)) != GSHT_OK)
      return st;
  }
  return GSHT_OK;
}

// userIO: read and write the callers' buffers (false for the tuning runs,
// which must leave them untouched).
gsht_status run_one(gsht_batch* b, Group& gr, int mode, cudaStream_t s, bool userIO) {
  gsht_status st;
  if (mode == 2) {
    if ((st = run_group(b, gr, 1, userIO, userIO, s)) != GSHT_OK) return st;
    return run_group(b, gr, 0, false, userIO, s);
  }
  return run_group(b, gr, mode, userIO, userIO, s);
}

// Everything one execution of `mode` does (0 forward, 1 inverse, 2 inverse
// then forward, the grids of the round trip also written back), with the
// groups (ordered largest first) dealt round-robin over `lanes` streams
// forked from and joined back into s.
gsht_status run_all_fused(gsht_batch* b, int mode, cudaStream_t s, int lanes, bool userIO);

gsht_status run_all(gsht_batch* b, int mode, cudaStream_t s, int lanes, bool userIO = true) {
  if (b->fused) return run_all_fused(b, mode, s, lanes, userIO);
  gsht_status st;
  if (lanes <= 1) {
    for (auto& gr : b->groups)
      if ((st = run_one(b, gr, mode, s, userIO)) != GSHT_OK) return st;
    return GSHT_OK;
  }
  cudaEvent_t fork = b->laneDone[0];
  GSHT_CUDA(cudaEventRecord(fork, s));
  for (int i = 0; i < lanes; i++) GSHT_CUDA(cudaStreamWaitEvent(b->lanes[i], fork, 0));
  for (size_t gi = 0; gi < b->groups.size(); gi++) {
    st = run_one(b, b->groups[gi], mode, b->lanes[gi % lanes], userIO);
    if (st != GSHT_OK) return st;
  }
  for (int i = 0; i < lanes; i++) {
    GSHT_CUDA(cudaEventRecord(b->laneDone[1 + i], b->lanes[i]));
    GSHT_CUDA(cudaStreamWaitEvent(s, b->laneDone[1 + i], 0));
  }
  return GSHT_OK;
}

// The fused BF16x3 execution of `mode` (as run_all): per direction, the
// groups' gathers and operand preparations (and forward ring FFTs) spread
// over the lanes, one multi-group Legendre launch on s, then the groups'
// inverse ring FFTs or forward accumulations and scatters over the lanes.
gsht_status run_all_fused(gsht_batch* b, int mode, cudaStream_t s, int lanes, bool userIO) {
  gsht_status st = GSHT_OK;
  const int L = lanes < 1 ? 1 : lanes;
  auto lane = [&](size_t gi) { return L == 1 ? s : b->lanes[gi % L]; };
  auto fork = [&]() -> gsht_status {
    if (L == 1) return GSHT_OK;
    GSHT_CUDA(cudaEventRecord(b->laneDone[0], s));
    for (int i = 0; i < L; i++) GSHT_CUDA(cudaStreamWaitEvent(b->lanes[i], b->laneDone[0], 0));
    return GSHT_OK;
  };
  auto join = [&]() -> gsht_status {
    if (L == 1) return GSHT_OK;
    for (int i = 0; i < L; i++) {
      GSHT_CUDA(cudaEventRecord(b->laneDone[1 + i], b->lanes[i]));
      GSHT_CUDA(cudaStreamWaitEvent(s, b->laneDone[1 + i], 0));
    }
    return GSHT_OK;
  };
  auto inverse = [&](bool gather, bool scatter) -> gsht_status {
    gsht_status r;
    if ((r = fork()) != GSHT_OK) return r;
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
      Group& gr = b->groups[gi];
      const int k = (int)gr.fields.size();
      // With the callers' buffers, the preparation reads their coefficients
      // through the group's pointer array (no gather).
      r = bf16_prep_inverse(gr.grid, gr.grid->table(gr.n), gr.lmax, gr.isReal, k,
                            reinterpret_cast<const double*>(gr.coefIn), gr.op, lane(gi),
                            gather ? reinterpret_cast<const double* const*>(gr.coefInPtrs) : nullptr);
      if (r != GSHT_OK) return r;
    }
    if ((r = join()) != GSHT_OK) return r;
    if ((r = bf16_multi_launch(b->multi[0], s)) != GSHT_OK) return r;
    if ((r = fork()) != GSHT_OK) return r;
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
      Group& gr = b->groups[gi];
      const int k = (int)gr.fields.size();
      {
        // With the callers' buffers, the ring FFTs write their grids through
        // the group's pointer array (no scatter).
        StageTimer tm(GSHT_STAGE_FFT_INVERSE, lane(gi));
        double* out = reinterpret_cast<double*>(gr.gridBuf);
        double* const* ptrs = scatter ? reinterpret_cast<double* const*>(gr.gridPtrs) : nullptr;
        RingRange rr;
        rr.fields = ptrs;
        r = gr.spec32 ? fft_inverse32(gr.grid, gr.lmax, gr.isReal, k,
                                      reinterpret_cast<const float*>(gr.spec), out, lane(gi), ptrs)
                      : fft_inverse(gr.grid, gr.lmax, gr.isReal, k, gr.spec, out, lane(gi), rr);
      }
      if (r != GSHT_OK) return r;
    }
    return join();
  };
  auto forward = [&](bool gridsAtCaller, bool scatter) -> gsht_status {
    gsht_status r;
    if ((r = fork()) != GSHT_OK) return r;
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
      Group& gr = b->groups[gi];
      const int k = (int)gr.fields.size();
      {
        // The grids: the callers' through the group's pointer array when
        // gathering (a forward on its own) or after an inverse that wrote
        // them there (a round trip with the callers' buffers), else the
        // group's contiguous buffer.
        StageTimer tm(GSHT_STAGE_FFT_FORWARD, lane(gi));
        const double* in = reinterpret_cast<const double*>(gr.gridBuf);
        double* const* ptrs = gridsAtCaller ? reinterpret_cast<double* const*>(gr.gridPtrs) : nullptr;
        RingRange rr;
        rr.fields = ptrs;
        r = gr.spec32 ? fft_forward32(gr.grid, gr.lmax, gr.isReal, k, in,
                                      reinterpret_cast<float*>(gr.spec), lane(gi), ptrs)
                      : fft_forward(gr.grid, gr.lmax, gr.isReal, k, in, gr.spec, lane(gi), rr);
      }
      if (r != GSHT_OK) return r;
      r = bf16_prep_forward(gr.grid, gr.lmax, gr.isReal, k, gr.spec, gr.op, lane(gi), gr.spec32);
      if (r != GSHT_OK) return r;
    }
    if ((r = join()) != GSHT_OK) return r;
    if ((r = bf16_multi_launch(b->multi[1], s)) != GSHT_OK) return r;
    if ((r = fork()) != GSHT_OK) return r;
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
      Group& gr = b->groups[gi];
      const int k = (int)gr.fields.size();
      const int na = gr.n < 0 ? -gr.n : gr.n;
      // With the callers' buffers, the accumulation adds straight into their
      // coefficients through the group's pointer array (it also applies
      // c_{L,L} = 0 to complex fields, whose lmax is the grid degree).
      if (!scatter)
        GSHT_CUDA(cudaMemsetAsync(gr.coefOut, 0, sizeof(double2) * gr.coefElems * k, lane(gi)));
      r = accumulate_forward(gr.grid->L, gr.lmax, gr.n, na, k, (gr.isReal ? 1 : 2) * k, gr.isReal,
                             gr.coefElems, gr.grid->theta_pad, gr.spec,
                             reinterpret_cast<double*>(gr.coefOut), lane(gi), true,
                             scatter ? reinterpret_cast<double* const*>(gr.coefOutPtrs) : nullptr);
      if (r != GSHT_OK) return r;
    }
    return join();
  };
  if (mode == 1 || mode == 2) st = inverse(userIO, userIO);
  if (st == GSHT_OK && (mode == 0 || mode == 2)) st = forward(userIO, userIO);
  return st;
}

// Buffers of the fused path and its two work lists at tile width `tile`.
gsht_status fused_build(gsht_batch* b, int tile) {
  for (auto& mp : b->multi) bf16_multi_free(&mp);
  std::vector<Bf16MultiGroup> gs;
  for (auto& gr : b->groups) {
    Bf16MultiGroup q;
    q.g = gr.grid;
    q.t = gr.grid->table(gr.n);
    q.lmax = gr.lmax;
    q.isReal = gr.isReal;
    q.count = (int)gr.fields.size();
    q.operand = gr.op;
    q.spec = gr.spec;
    q.spec32 = gr.spec32;
    gs.push_back(q);
  }
  for (int dir = 0; dir < 2; dir++) {
    gsht_status st = bf16_multi_build(dir, gs.data(), (int)gs.size(), tile, &b->multi[dir]);
    if (st != GSHT_OK) return st;
  }
  b->fusedTile = tile;
  return GSHT_OK;
}

void free_batch(gsht_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (int i = 0; i < 3; i++) {
    if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
    if (b->graph[i]) cudaGraphDestroy(b->graph[i]);
  }
  for (auto& gr : b->groups) {
    dev_free(gr.coefIn);
    dev_free(gr.gridBuf);
    dev_free(gr.coefOut);
    dev_free(gr.coefInPtrs);
    dev_free(gr.gridPtrs);
    dev_free(gr.coefOutPtrs);
    dev_free(gr.ws);
    dev_free(gr.spec);
    dev_free(gr.op);
  }
  for (auto& mp : b->multi) bf16_multi_free(&mp);
  for (auto& kv : b->grids) gsht_grid_destroy(kv.second);
  for (cudaStream_t l : b->lanes) cudaStreamDestroy(l);
  for (cudaEvent_t e : b->laneDone) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

gsht_status upload_ptrs(double2*** dst, const std::vector<const void*>& host) {
  GSHT_CUDA(dev_malloc(dst, sizeof(double2*) * host.size()));
  GSHT_CUDA(cudaMemcpy(*dst, host.data(), sizeof(double2*) * host.size(), cudaMemcpyHostToDevice));
  return GSHT_OK;
}


// Times one round trip of a group (after a warm-up) on the plan's stream.
gsht_status time_group(gsht_batch* b, Group& gr, float* ms) {
  cudaEvent_t e0, e1;
  GSHT_CUDA(cudaEventCreate(&e0));
  GSHT_CUDA(cudaEventCreate(&e1));
  gsht_status st = GSHT_OK;
  for (int rep = 0; rep < 3 && st == GSHT_OK; rep++) {
    if (rep == 1) cudaEventRecord(e0, b->stream);
    st = run_group(b, gr, 1, false, false, b->stream);
    if (st == GSHT_OK) st = run_group(b, gr, 0, false, false, b->stream);
  }
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

gsht_status plan(const gsht_field_desc* fields, int count, int precision, int autotune,
                 gsht_batch* b) {
  b->precision = precision;
  b->fields.assign(fields, fields + count);
  GSHT_CUDA(cudaGetDevice(&b->device));
  GSHT_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  // Groups by (lmax, n, kind); grids by lmax with the widest upper index.
  std::map<std::tuple<int, int, int>, int> index;
  std::map<int, int> nmax;
  for (int i = 0; i < count; i++) {
    const auto& f = fields[i];
    const auto key = std::make_tuple(f.lmax, f.n, f.is_real ? 1 : 0);
    auto it = index.find(key);
    if (it == index.end()) {
      Group gr;
      gr.lmax = f.lmax;
      gr.n = f.n;
      gr.isReal = f.is_real ? 1 : 0;
      it = index.emplace(key, (int)b->groups.size()).first;
      b->groups.push_back(gr);
    }
    b->groups[it->second].fields.push_back(i);
    const int na = f.n < 0 ? -f.n : f.n;
    nmax[f.lmax] = std::max(nmax[f.lmax], na);
  }
  const unsigned forms = GSHT_FORM_FP64 | (precision == GSHT_BF16X3 ? GSHT_FORM_BF16X3 : 0u) |
                         ((precision == GSHT_OZAKI || precision == GSHT_OZAKI4) ? GSHT_FORM_OZAKI : 0u);
  for (auto& kv : nmax) {
    gsht_grid* g = nullptr;
    gsht_status st = gsht_grid_create(kv.first, kv.second, GSHT_RANGE_ALL, GSHT_RANGE_ALL, forms, &g);
    if (st != GSHT_OK) return st;
    b->grids[kv.first] = g;
  }
  for (auto& gr : b->groups) {
    gr.grid = b->grids[gr.lmax];
    const int k = (int)gr.fields.size();
    gr.coefElems = coef_size(gr.lmax, gr.n, gr.isReal);
    const long points = (long)(gr.lmax + 1) * 2 * gr.lmax;
    gr.gridElems = gr.isReal ? points / 2 : points;
    GSHT_CUDA(dev_malloc(&gr.coefIn, sizeof(double2) * gr.coefElems * k));
    GSHT_CUDA(dev_malloc(&gr.gridBuf, sizeof(double2) * gr.gridElems * k));
    GSHT_CUDA(dev_malloc(&gr.coefOut, sizeof(double2) * gr.coefElems * k));
    std::vector<const void*> ci, gp, co;
    for (int i : gr.fields) {
      ci.push_back(b->fields[i].coef_in);
      gp.push_back(b->fields[i].grid);
      co.push_back(b->fields[i].coef_out);
    }
    gsht_status st;
    if ((st = upload_ptrs(&gr.coefInPtrs, ci)) != GSHT_OK) return st;
    if ((st = upload_ptrs(&gr.gridPtrs, gp)) != GSHT_OK) return st;
    if ((st = upload_ptrs(&gr.coefOutPtrs, co)) != GSHT_OK) return st;
    // Defined batch inputs for the warm-up and tuning runs.
    GSHT_CUDA(cudaMemsetAsync(gr.coefIn, 0, sizeof(double2) * gr.coefElems * k, b->stream));
    GSHT_CUDA(cudaMemsetAsync(gr.gridBuf, 0, sizeof(double2) * gr.gridElems * k, b->stream));
    // The group's own workspace: the larger of the two directions' needs.
    size_t needInv = 0, needFwd = 0;
    PrivateWorkspace qi{nullptr, 0, &needInv}, qf{nullptr, 0, &needFwd};
    if ((st = transform(gr.grid, 1, gr.lmax, gr.n, gr.isReal, precision, k, gr.coefIn,
                        gr.gridBuf, b->stream, gr.ntile, &qi)) != GSHT_OK ||
        (st = transform(gr.grid, 0, gr.lmax, gr.n, gr.isReal, precision, k, gr.gridBuf,
                        gr.coefOut, b->stream, gr.ntile, &qf)) != GSHT_OK)
      return st;
    gr.wsBytes = std::max(needInv, needFwd);
    GSHT_CUDA(dev_malloc(&gr.ws, gr.wsBytes));
    gr.work = (double)k * (gr.lmax + 1.0) * (gr.lmax + 1.0) * (gr.lmax + 1.0) * (gr.isReal ? 0.5 : 1.0);
  }
  // Largest groups first: with the round-robin over streams the long
  // transforms start early and the small ones fill in behind them.
  std::stable_sort(b->groups.begin(), b->groups.end(),
                   [](const Group& x, const Group& y) { return x.work > y.work; });
  const char* fusedEnv = getenv("GSHT_BATCH_FUSED");
  b->fused = precision == GSHT_BF16X3 && !(fusedEnv && fusedEnv[0] == '0');
  if (b->fused) {
    for (auto& gr : b->groups) {
      const int k = (int)gr.fields.size();
      const size_t specBytes = sizeof(double) * 2 * spec_elems(gr.grid, gr.lmax, gr.isReal, k);
      const size_t opBytes = std::max(bf16_operand_bytes(gr.grid, gr.lmax, gr.isReal, k, 0),
                                      bf16_operand_bytes(gr.grid, gr.lmax, gr.isReal, k, 1));
      GSHT_CUDA(dev_malloc(&gr.spec, specBytes));
      GSHT_CUDA(dev_malloc_bytes(&gr.op, opBytes));
      gr.spec32 = fft_spec32_supported(gr.grid, gr.isReal);
    }
  }
  // Warm-up (sizes every workspace, builds tile lists and layouts), then
  // the autotuner: per group, the fastest BF16x3 tile width (the fused path
  // tunes the tile width of its one launch further below).
  for (auto& gr : b->groups) {
    if (b->fused) break;
    gsht_status st = run_group(b, gr, 1, false, false, b->stream);
    if (st == GSHT_OK) st = run_group(b, gr, 0, false, false, b->stream);
    if (st != GSHT_OK) return st;
    if (precision == GSHT_BF16X3 && autotune) {
      float best = 3.4e38f;
      int bestTile = 128;
      for (int tile : {32, 64, 128}) {
        gr.ntile = tile;
        float ms = 0.f;
        if ((st = time_group(b, gr, &ms)) != GSHT_OK) return st;
        if (ms < best) {
          best = ms;
          bestTile = tile;
        }
      }
      gr.ntile = bestTile;
    }
  }
  GSHT_CUDA(cudaStreamSynchronize(b->stream));
  for (auto& kv : b->grids) {
    gsht_status st = gsht_device_status(kv.second);
    if (st != GSHT_OK) return st;
  }
  // Streams for the concurrent schedule and their fork / join events.
  const int maxLanes = (int)std::min<size_t>(kMaxLanes, b->groups.size());
  for (int i = 0; i < maxLanes; i++) {
    cudaStream_t l;
    GSHT_CUDA(cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking));
    b->lanes.push_back(l);
  }
  for (int i = 0; i <= maxLanes; i++) {
    cudaEvent_t e;
    GSHT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->laneDone.push_back(e);
  }
  // Schedule autotuner: the round-trip graph for each candidate number of
  // streams, timed over a few launches; the fastest count is used for all
  // three modes.
  auto capture = [&](int mode, int lanes, cudaGraph_t* graph, bool userIO) -> gsht_status {
    GSHT_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    gsht_status st = run_all(b, mode, b->stream, lanes, userIO);
    *graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, graph);
    if (st != GSHT_OK) {
      if (*graph) cudaGraphDestroy(*graph);
      *graph = nullptr;
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
    return GSHT_OK;
  };
  // Time of the round-trip graph with `lanes` streams (callers' buffers
  // untouched), over three launches after one.
  auto time_graph = [&](int lanes, float* ms) -> gsht_status {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    gsht_status st = capture(2, lanes, &graph, false);
    if (st != GSHT_OK) return st;
    if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      return cuda_fail(cudaGetLastError(), "batch graph instantiation");
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaGraphLaunch(exec, b->stream);
    cudaEventRecord(e0, b->stream);
    for (int r = 0; r < 3; r++) cudaGraphLaunch(exec, b->stream);
    cudaEventRecord(e1, b->stream);
    const cudaError_t se = cudaEventSynchronize(e1);
    *ms = 0.f;
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (se != cudaSuccess) return cuda_fail(se, "batch schedule tuning");
    return GSHT_OK;
  };
  // Fused path: the tile width of the one Legendre launch per direction
  // (each candidate warmed up uncaptured, then timed as a graph).
  if (b->fused) {
    const int guessLanes = std::min(maxLanes, 8);
    int bestTile = 64;
    float best = 3.4e38f;
    for (int tile : {32, 64, 128}) {
      if (!autotune && tile != 64) continue;
      gsht_status st = fused_build(b, tile);
      if (st == GSHT_OK) st = run_all_fused(b, 2, b->stream, 1, false);
      if (st != GSHT_OK) return st;
      GSHT_CUDA(cudaStreamSynchronize(b->stream));
      if (!autotune) break;
      float ms = 0.f;
      if ((st = time_graph(guessLanes, &ms)) != GSHT_OK) return st;
      if (ms < best) {
        best = ms;
        bestTile = tile;
      }
    }
    if (b->fusedTile != bestTile) {
      gsht_status st = fused_build(b, bestTile);
      if (st != GSHT_OK) return st;
    }
    for (auto& gr : b->groups) gr.ntile = b->fusedTile;
    for (auto& kv : b->grids) {
      gsht_status st = gsht_device_status(kv.second);
      if (st != GSHT_OK) return st;
    }
  }
  b->nlanes = 1;
  if (maxLanes > 1 && autotune) {
    float best = 3.4e38f;
    for (int lanes : {1, 2, 4, 8, 16}) {
      if (lanes > maxLanes) break;
      float ms = 0.f;
      gsht_status st = time_graph(lanes, &ms);
      if (st != GSHT_OK) return st;
      if (ms < best) {
        best = ms;
        b->nlanes = lanes;
      }
    }
  } else if (maxLanes > 1) {
    b->nlanes = std::min(maxLanes, 8);
  }
  // One graph per execution mode.
  for (int mode = 0; mode < 3; mode++) {
    cudaGraph_t graph = nullptr;
    gsht_status st = capture(mode, b->nlanes, &graph, true);
    if (st != GSHT_OK) return st;
    b->graph[mode] = graph;
    GSHT_CUDA(cudaGraphGetNodes(graph, nullptr, &b->nodes[mode]));
    GSHT_CUDA(cudaGraphInstantiate(&b->exec[mode], graph, 0));
  }
  return GSHT_OK;
}

}  // namespace
}  // namespace gsht

using namespace gsht;

extern "C" {

gsht_status gsht_plan_batch(const gsht_field_desc* fields, int count, int precision,
                            int autotune, gsht_batch** out) {
  if (!out) return fail(GSHT_ERR_BAD_ARG, "output handle pointer is NULL");
  *out = nullptr;
  if (!fields || count < 1) return fail(GSHT_ERR_BAD_ARG, "need at least one field");
  if (precision != GSHT_FP64 && precision != GSHT_BF16X3 && precision != GSHT_OZAKI &&
      precision != GSHT_OZAKI4)
    return fail(GSHT_ERR_UNSUPPORTED, "precision %d not available", precision);
  for (int i = 0; i < count; i++) {
    const auto& f = fields[i];
    const int na = f.n < 0 ? -f.n : f.n;
    if (f.lmax < 1 || f.lmax > 8192)
      return fail(GSHT_ERR_BAD_ARG, "field %d: lmax %d outside [1, 8192]", i, f.lmax);
    if (na > f.lmax) return fail(GSHT_ERR_BAD_ARG, "field %d: |n| = %d exceeds lmax", i, na);
    if (!f.coef_in || !f.grid || !f.coef_out)
      return fail(GSHT_ERR_BAD_ARG, "field %d: coef_in, grid and coef_out must all be set", i);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GSHT_ERR_NO_DEVICE, "no CUDA device visible");
  }
  int dev = 0;
  GSHT_CUDA(cudaGetDevice(&dev));
  for (int i = 0; i < count; i++)
    if (pointer_kind(fields[i].coef_in, dev) != kDevicePtr ||
        pointer_kind(fields[i].grid, dev) != kDevicePtr ||
        pointer_kind(fields[i].coef_out, dev) != kDevicePtr)
      return fail(GSHT_ERR_BAD_ARG, "field %d: batch buffers must be memory of the current device", i);
    else if (!aligned16(fields[i].coef_in) || !aligned16(fields[i].grid) ||
             !aligned16(fields[i].coef_out))
      return fail(GSHT_ERR_BAD_ARG, "field %d: batch buffers must be 16-byte aligned", i);
  auto* b = new gsht_batch();
  const gsht_status st = plan(fields, count, precision, autotune, b);
  if (st != GSHT_OK) {
    const std::string msg = gsht_last_error();
    free_batch(b);
    return fail(st, "%s", msg.c_str());
  }
  *out = b;
  return GSHT_OK;
}

gsht_status gsht_batch_execute(gsht_batch* b, int mode, void* stream) {
  if (!b) return fail(GSHT_ERR_BAD_ARG, "batch is NULL");
  if (mode < GSHT_BATCH_FORWARD || mode > GSHT_BATCH_ROUND_TRIP)
    return fail(GSHT_ERR_BAD_ARG, "bad batch mode %d", mode);
  GSHT_CUDA(cudaSetDevice(b->device));
  GSHT_CUDA(cudaGraphLaunch(b->exec[mode], reinterpret_cast<cudaStream_t>(stream)));
  g_launches += b->nodes[mode];
  return GSHT_OK;
}

gsht_status gsht_batch_info(const gsht_batch* b, int* groups, int* grids, long* graph_nodes) {
  if (!b) return fail(GSHT_ERR_BAD_ARG, "batch is NULL");
  if (groups) *groups = (int)b->groups.size();
  if (grids) *grids = (int)b->grids.size();
  if (graph_nodes) {
    for (int i = 0; i < 3; i++) graph_nodes[i] = (long)b->nodes[i];
  }
  return GSHT_OK;
}

gsht_status gsht_batch_group(const gsht_batch* b, int index, int* lmax, int* n, int* is_real,
                             int* count, int* ntile) {
  if (!b || index < 0 || index >= (int)b->groups.size())
    return fail(GSHT_ERR_BAD_ARG, "no group %d", index);
  const auto& gr = b->groups[index];
  if (lmax) *lmax = gr.lmax;
  if (n) *n = gr.n;
  if (is_real) *is_real = gr.isReal;
  if (count) *count = (int)gr.fields.size();
  if (ntile) *ntile = gr.ntile;
  return GSHT_OK;
}

gsht_status gsht_batch_schedule(const gsht_batch* b, int* streams) {
  if (!b) return fail(GSHT_ERR_BAD_ARG, "batch is NULL");
  if (streams) *streams = b->nlanes;
  return GSHT_OK;
}

gsht_status gsht_batch_destroy(gsht_batch* b) {
  free_batch(b);
  return GSHT_OK;
}

}  // extern "C"
