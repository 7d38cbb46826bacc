// batch.cu -- batches of independent periodic systems (include/ffxcuda.h, ffxg_batch_*).
//
// Many small boxes of uneven size (conformer, rotamer or lambda-window energies) are
// launch-bound one at a time: a 96-atom system runs ~150 kernels of a few blocks each.
// A batch keeps one handle per system (its own lists, grids and solver state).
//
// GRAPH mode runs the batch stage by stage: every system's evaluation is recorded once
// (each launch with its grid and packed arguments, launch.cuh), the recordings are merged
// into one sequence of stages -- a stage is one kernel body at one point of the
// evaluation -- and each stage becomes ONE launch of k_many over all systems that have
// it: system s owns a contiguous range of the grid's blocks and reads its own arguments.
// So every small PME mesh of the batch is transformed by the same FFT launches, and every
// pair kernel sees the atoms of all systems at once.  The solver's loop is one conditional
// WHILE node for the whole batch: its body's launches skip the systems whose solve has
// stopped, and a one-warp kernel keeps the loop going while any system continues.  The
// results each system copies to the host are gathered on the device into one staging
// buffer and read back with one copy.  The batch is one CUDA graph: one launch.
//
// BRANCHES mode captures every system's own evaluation graph (its PCG loop its own WHILE
// node) as an independent branch of one graph; LOOP mode evaluates the systems one after
// another through the single-system path.  GRAPH mode falls back to BRANCHES when the
// recordings cannot be merged.
//
// Results are those of the single-system path: the same bodies run on the same buffers
// with the same grids.  (A system with a 64 x 64 mixed-form mesh takes the per-axis FFT
// passes inside a stage-by-stage batch instead of its four-CTA cluster passes: the same
// transform, rounded differently.)
#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "ffx_internal.cuh"

using namespace ffx;

namespace {

constexpr size_t kStageSlot = 256;   // bytes of results each system reads back

// Keeps the batch's solver loop going while any system's solve continues.
__global__ void k_batch_cond(const int *const *__restrict__ cont, int ns, cudaGraphConditionalHandle cond) {
  int any = 0;
  for (int s = threadIdx.x; s < ns; s += 32) any |= *cont[s];
  any = __any_sync(0xffffffffu, any);
  if (threadIdx.x == 0) cudaGraphSetConditional(cond, any ? 1u : 0u);
}

// One stage of a stage-by-stage batch: one k_many launch over the systems that have it.
struct Stage {
  const void *fn = nullptr;
  int block = 0, phase = 0;
  size_t smem = 0, pack_size = 0;
  int rank = 1 << 30;                    // earliest position in any system's recording
  std::vector<int> sys, grid;
  std::vector<const unsigned char *> pack;
  size_t off_pre = 0, off_pack = 0, off_cont = 0;
  int blocks = 0;
};

}  // namespace

struct ffxg_batch {
  std::vector<ffxg_handle *> sys;
  std::vector<int64_t> off;              // first atom of each system; off[n] = total atoms
  int mode = FFXG_BATCH_GRAPH;
  double *d_xyz = nullptr, *d_grad = nullptr;    // [total][3] on the device
  double *h_xyz = nullptr, *h_grad = nullptr;    // pinned mirrors
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};  // by want_grad
  bool staged[2] = {false, false};               // exec[key] is a stage-by-stage graph
  std::vector<int64_t> gen;               // each handle's graph generation at capture
  int64_t graph_builds = 0;
  std::string err;
  // Stage-by-stage form: argument tables, result staging, each system's result copies.
  unsigned char *d_tab[2] = {nullptr, nullptr};
  unsigned char *d_stage = nullptr, *h_stage = nullptr;
  std::vector<std::vector<Recorder::Copy>> copies[2];
  int n_stages[2] = {0, 0};
};

static std::string g_batch_create_error;

static void batch_drop_graphs(ffxg_batch &b) {
  for (int k = 0; k < 2; k++) {
    if (b.exec[k]) { cudaGraphExecDestroy(b.exec[k]); b.exec[k] = nullptr; }
    if (b.d_tab[k]) { cudaFree(b.d_tab[k]); b.d_tab[k] = nullptr; }
    b.staged[k] = false;
    b.copies[k].clear();
    b.n_stages[k] = 0;
  }
}

static void batch_free(ffxg_batch &b) {
  batch_drop_graphs(b);
  for (ffxg_handle *h : b.sys) ffxg_destroy(h);
  b.sys.clear();
  if (b.d_xyz) cudaFree(b.d_xyz);
  if (b.d_grad) cudaFree(b.d_grad);
  if (b.d_stage) cudaFree(b.d_stage);
  if (b.h_xyz) cudaFreeHost(b.h_xyz);
  if (b.h_grad) cudaFreeHost(b.h_grad);
  if (b.h_stage) cudaFreeHost(b.h_stage);
  if (b.ev_fork) cudaEventDestroy(b.ev_fork);
  if (b.ev_join) cudaEventDestroy(b.ev_join);
  if (b.stream) cudaStreamDestroy(b.stream);
  if (b.side) cudaStreamDestroy(b.side);
}

// The systems' recordings merged into stages, phase by phase: a stage is (phase, kernel
// instance, its k-th launch in that phase) and gathers the systems that have it; the
// stages are put in an order that keeps every system's own order (Kahn's algorithm,
// earliest recorded position first).  Systems share no data, so any such order is
// correct for each of them.  False when one stage's block size differs between systems
// or the orders cannot be reconciled.
static bool merge_recordings(const std::vector<Recorder> &rec, std::vector<Stage> &out, std::string &why) {
  out.clear();
  for (int phase = 0; phase < 3; phase++) {
    std::map<std::tuple<const void *, int>, int> id;
    std::vector<Stage> nodes;
    std::vector<std::set<int>> succ;
    for (size_t s = 0; s < rec.size(); s++) {
      std::map<const void *, int> ordinal;
      int prev = -1, pos = 0;
      for (const RecLaunch &L : rec[s].seq) {
        if (L.phase != phase) continue;
        const int o = ordinal[L.fn]++;
        auto it = id.find({L.fn, o});
        int v;
        if (it == id.end()) {
          v = (int)nodes.size();
          id[{L.fn, o}] = v;
          nodes.emplace_back();
          succ.emplace_back();
          nodes[v].fn = L.fn;
          nodes[v].block = L.block;
          nodes[v].phase = phase;
          nodes[v].pack_size = L.pack.size();
        } else {
          v = it->second;
        }
        Stage &st = nodes[v];
        if (st.block != L.block || st.pack_size != L.pack.size()) {
          why = "a stage's launch shape differs between systems";
          return false;
        }
        st.sys.push_back((int)s);
        st.grid.push_back(L.grid);
        st.pack.push_back(L.pack.data());
        st.smem = std::max(st.smem, L.smem);
        st.rank = std::min(st.rank, pos++);
        if (prev >= 0 && prev != v) succ[prev].insert(v);
        prev = v;
      }
    }
    std::vector<int> indeg(nodes.size(), 0);
    for (const auto &sc : succ)
      for (int v : sc) indeg[v]++;
    std::set<std::pair<int, int>> ready;   // (rank, node)
    for (size_t v = 0; v < nodes.size(); v++)
      if (!indeg[v]) ready.insert({nodes[v].rank, (int)v});
    size_t done = 0;
    std::vector<int> order;
    while (!ready.empty()) {
      const int v = ready.begin()->second;
      ready.erase(ready.begin());
      order.push_back(v);
      done++;
      for (int w : succ[v])
        if (--indeg[w] == 0) ready.insert({nodes[w].rank, w});
    }
    if (done != nodes.size()) {
      why = "the systems order their stages differently";
      return false;
    }
    for (int v : order) out.push_back(std::move(nodes[v]));
  }
  return true;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static void launch_stage(const Stage &st, const unsigned char *tab, cudaStream_t stream) {
  const void *packs = tab + st.off_pack;
  const int *pre = reinterpret_cast<const int *>(tab + st.off_pre);
  const int *const *cont = st.phase == 1 ? reinterpret_cast<const int *const *>(tab + st.off_cont) : nullptr;
  int ns = (int)st.sys.size();
  void *args[4] = {(void *)&packs, (void *)&pre, (void *)&cont, (void *)&ns};
  cudaLaunchKernel(st.fn, dim3(st.blocks), dim3(st.block), args, st.smem, stream);
}

// Record every system's evaluation, merge the recordings into stages and capture the
// stage-by-stage graph (exec[key]).  Returns FFXG_OK, or a status with b.err set; the
// caller then falls back to the branch graph.
static int staged_capture(ffxg_batch &b, int key) {
  const size_t S = b.sys.size();
  std::vector<Recorder> rec(S);
  for (size_t s = 0; s < S; s++) {
    Handle &h = handle_of(b.sys[s]);
    h.want_grad = key != 0;
    const bool pin = h.grad_to_pin;
    h.grad_to_pin = false;
    h.batch_branch = true;
    h.rec = &rec[s];
    h.d_stage = b.d_stage + s * kStageSlot;
    // Recorded under a throwaway capture of the handle's stream: anything the recording
    // missed (a launch or copy not routed through the recorder) would appear in it.
    int st = FFXG_OK;
    size_t stray = 0;
    if (cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      st = FFXG_ERR_CUDA;
    } else {
      st = eval_capture_body(h, b.d_xyz + 3 * b.off[s], b.d_grad + 3 * b.off[s]);
      cudaGraph_t g = nullptr;
      if (cudaStreamEndCapture(h.stream, &g) != cudaSuccess) st = FFXG_ERR_CUDA;
      if (g) {
        cudaGraphGetNodes(g, nullptr, &stray);
        cudaGraphDestroy(g);
      }
    }
    h.rec = nullptr;
    h.d_stage = nullptr;
    h.batch_branch = false;
    h.grad_to_pin = pin;
    cudaGetLastError();
    if (st != FFXG_OK || stray != 0 || rec[s].stage_bytes > kStageSlot) {
      b.err = "system " + std::to_string(s) + ": evaluation could not be recorded";
      return FFXG_ERR_CUDA;
    }
  }
  std::vector<Stage> stages;
  if (!merge_recordings(rec, stages, b.err)) return FFXG_ERR_CUDA;

  // Argument tables: per stage the block prefix, the packed arguments and (loop stages)
  // each system's solver flag; then the flags of every system in the loop.
  size_t bytes = 0;
  for (Stage &st : stages) {
    const size_t ns = st.sys.size();
    st.off_pre = bytes = align_up(bytes, 16);
    bytes += (ns + 1) * sizeof(int);
    st.off_pack = bytes = align_up(bytes, 16);
    bytes += ns * st.pack_size;
    st.off_cont = bytes = align_up(bytes, 16);
    if (st.phase == 1) bytes += ns * sizeof(const int *);
  }
  std::vector<unsigned char> tab(std::max<size_t>(bytes, 16), 0);
  std::set<int> in_loop;
  for (Stage &st : stages) {
    const size_t ns = st.sys.size();
    int *pre = reinterpret_cast<int *>(tab.data() + st.off_pre);
    pre[0] = 0;
    for (size_t j = 0; j < ns; j++) {
      pre[j + 1] = pre[j] + st.grid[j];
      std::memcpy(tab.data() + st.off_pack + j * st.pack_size, st.pack[j], st.pack_size);
      if (st.phase == 1) {
        const int *c = &handle_of(b.sys[st.sys[j]]).d_pcg->cont;
        std::memcpy(tab.data() + st.off_cont + j * sizeof(const int *), &c, sizeof(c));
        in_loop.insert(st.sys[j]);
      }
    }
    st.blocks = pre[ns];
  }
  std::vector<const int *> loop_cont;
  for (int sidx : in_loop) loop_cont.push_back(&handle_of(b.sys[sidx]).d_pcg->cont);
  const size_t off_loop = align_up(tab.size(), 16);
  tab.resize(off_loop + std::max<size_t>(1, loop_cont.size()) * sizeof(const int *));
  if (!loop_cont.empty()) std::memcpy(tab.data() + off_loop, loop_cont.data(), loop_cont.size() * sizeof(const int *));
  unsigned char *d_tab = nullptr;
  if (cudaMalloc(&d_tab, tab.size()) != cudaSuccess ||
      cudaMemcpy(d_tab, tab.data(), tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    if (d_tab) cudaFree(d_tab);
    b.err = "batch stage tables: could not be uploaded";
    return FFXG_ERR_CUDA;
  }
  const int *const *d_loop = reinterpret_cast<const int *const *>(d_tab + off_loop);
  const int n_loop = (int)loop_cont.size();

  // The graph: phase 0, the loop (a WHILE node whose body is phase 1 and the loop test),
  // phase 2, then the results read back in one copy.
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    for (const Stage &st : stages)
      if (st.phase == 0) launch_stage(st, d_tab, b.stream);
    if (n_loop > 0) {
      cudaStreamCaptureStatus cs;
      cudaGraph_t g = nullptr;
      const cudaGraphNode_t *deps = nullptr;
      size_t ndeps = 0;
      cudaGraphConditionalHandle cond{};
      ok = cudaStreamGetCaptureInfo(b.stream, &cs, nullptr, &g, &deps, &ndeps) == cudaSuccess &&
           cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
      if (ok) {
        k_batch_cond<<<1, 32, 0, b.stream>>>(d_loop, n_loop, cond);
        ok = cudaStreamGetCaptureInfo(b.stream, &cs, nullptr, &g, &deps, &ndeps) == cudaSuccess;
      }
      cudaGraphNodeParams cp = {};
      cudaGraphNode_t node;
      if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, g, deps, ndeps, &cp) == cudaSuccess &&
             cudaStreamUpdateCaptureDependencies(b.stream, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
      }
      if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(b.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
             cudaSuccess;
        if (ok) {
          for (const Stage &st : stages)
            if (st.phase == 1) launch_stage(st, d_tab, b.side);
          k_batch_cond<<<1, 32, 0, b.side>>>(d_loop, n_loop, cond);
          ok = cudaStreamEndCapture(b.side, &body) == cudaSuccess;
        }
      }
    }
    for (const Stage &st : stages)
      if (st.phase == 2) launch_stage(st, d_tab, b.stream);
    cudaMemcpyAsync(b.h_stage, b.d_stage, S * kStageSlot, cudaMemcpyDeviceToHost, b.stream);
    const bool ended = cudaStreamEndCapture(b.stream, &graph) == cudaSuccess;
    ok = ok && ended;
  }
  cudaGraphExec_t exec = nullptr;
  if (ok && graph) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    cudaGetLastError();
    if (exec) cudaGraphExecDestroy(exec);
    cudaFree(d_tab);
    b.err = "the stage-by-stage batch graph could not be built";
    return FFXG_ERR_CUDA;
  }
  b.exec[key] = exec;
  b.d_tab[key] = d_tab;
  b.staged[key] = true;
  b.n_stages[key] = (int)stages.size();
  b.copies[key].resize(S);
  for (size_t s = 0; s < S; s++) b.copies[key][s] = rec[s].copies;
  b.gen.clear();
  for (ffxg_handle *hh : b.sys) b.gen.push_back(handle_of(hh).graph_gen);
  b.graph_builds++;
  return FFXG_OK;
}

// One graph: a fork from the batch stream into every system's stream, each system's
// captured evaluation on its slice of the batch buffers, and a join back.  The fork event
// is recorded once, before any branch, so every branch depends only on the graph's start
// (a join event re-recorded per branch would chain the branches one after another).
static int batch_capture(ffxg_batch &b, int key) {
  if (cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FFXG_ERR_CUDA;
  cudaEventRecord(b.ev_fork, b.stream);
  int st = FFXG_OK;
  size_t entered = 0;
  for (size_t s = 0; s < b.sys.size() && st == FFXG_OK; s++, entered++) {
    Handle &h = handle_of(b.sys[s]);
    h.want_grad = key != 0;
    h.batch_branch = true;   // the reciprocal chains stay in line inside a batch (measured faster)
    cudaStreamWaitEvent(h.stream, b.ev_fork, 0);
    st = eval_capture_body(h, b.d_xyz + 3 * b.off[s], b.d_grad + 3 * b.off[s]);
    h.batch_branch = false;
  }
  for (size_t s = 0; s < entered; s++) {   // join every stream that entered the capture
    cudaEventRecord(b.ev_join, handle_of(b.sys[s]).stream);
    cudaStreamWaitEvent(b.stream, b.ev_join, 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(b.stream, &graph);
  if (st != FFXG_OK || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return FFXG_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&b.exec[key], graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    b.exec[key] = nullptr;
    cudaGetLastError();
    return FFXG_ERR_CUDA;
  }
  b.gen.clear();
  for (ffxg_handle *hh : b.sys) b.gen.push_back(handle_of(hh).graph_gen);
  b.graph_builds++;
  return FFXG_OK;
}

// Whether the batch may run as one graph, dropping a captured one that went stale (a
// handle changed lists, lambda or modes since the capture).
static bool batch_graph_ready(ffxg_batch &b) {
  bool stale = b.gen.size() != b.sys.size();
  for (size_t s = 0; s < b.sys.size(); s++) {
    const Handle &h = handle_of(b.sys[s]);
    if (!h.list_valid || !h.use_graphs || h.timing) return false;
    if (h.elec.on && h.alch.active) return false;   // electrostatic lambda runs as direct launches
    if (!stale && b.gen[s] != h.graph_gen) stale = true;
  }
  if (stale) batch_drop_graphs(b);
  return true;
}

extern "C" {

int ffxg_batch_create(int32_t n_systems, const ffxg_system *systems, const ffxg_params *params, ffxg_batch **out) {
  if (!systems || !params || !out || n_systems <= 0) {
    g_batch_create_error = "null argument or empty batch";
    return FFXG_ERR_BAD_ARG;
  }
  *out = nullptr;
  ffxg_batch *b = new ffxg_batch();
  b->off.assign(1, 0);
  for (int32_t s = 0; s < n_systems; s++) {
    ffxg_handle *h = nullptr;
    const int st = ffxg_create(&systems[s], &params[s], &h);
    if (st != FFXG_OK) {
      g_batch_create_error = "system " + std::to_string(s) + ": " + ffxg_last_error(nullptr);
      batch_free(*b);
      delete b;
      return st;
    }
    b->sys.push_back(h);
    b->off.push_back(b->off.back() + systems[s].n_atoms);
  }
  const size_t m = 3 * (size_t)b->off.back();
  if (cudaMalloc(&b->d_xyz, m * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_grad, m * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_xyz, m * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_grad, m * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_stage, (size_t)n_systems * kStageSlot) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_stage, (size_t)n_systems * kStageSlot) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    g_batch_create_error = std::string("batch buffers: ") + cudaGetErrorString(cudaGetLastError());
    batch_free(*b);
    delete b;
    return FFXG_ERR_CUDA;
  }
  for (int32_t s = 0; s < n_systems; s++)
    std::memcpy(b->h_xyz + 3 * b->off[s], systems[s].xyz, 3 * (size_t)systems[s].n_atoms * sizeof(double));
  *out = b;
  return FFXG_OK;
}

void ffxg_batch_destroy(ffxg_batch *b) {
  if (!b) return;
  cudaStreamSynchronize(b->stream);
  batch_free(*b);
  delete b;
}

const char *ffxg_batch_last_error(const ffxg_batch *b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int ffxg_batch_set_mode(ffxg_batch *b, int mode) {
  if (!b) return FFXG_ERR_BAD_ARG;
  if (mode != FFXG_BATCH_GRAPH && mode != FFXG_BATCH_LOOP && mode != FFXG_BATCH_BRANCHES) {
    b->err = "unknown batch mode";
    return FFXG_ERR_BAD_ARG;
  }
  if (mode != b->mode) batch_drop_graphs(*b);
  b->mode = mode;
  return FFXG_OK;
}

int64_t ffxg_batch_atoms(const ffxg_batch *b, int64_t *offsets) {
  if (!b) return -1;
  if (offsets) std::copy(b->off.begin(), b->off.end(), offsets);
  return b->off.back();
}

ffxg_handle *ffxg_batch_system(ffxg_batch *b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->sys.size()) return nullptr;
  return b->sys[i];
}

int64_t ffxg_batch_graph_builds(const ffxg_batch *b) { return b ? b->graph_builds : -1; }

int32_t ffxg_batch_stages(const ffxg_batch *b, int want_grad) {
  if (!b) return -1;
  const int key = want_grad ? 1 : 0;
  return b->staged[key] ? b->n_stages[key] : 0;
}

int ffxg_batch_energy(ffxg_batch *b, const double *xyz, int want_grad, double *terms, double *grad, int64_t *counts,
                      int32_t *status) {
  if (!b || !terms || (want_grad && !grad)) return FFXG_ERR_BAD_ARG;
  const size_t S = b->sys.size();
  const size_t m = 3 * (size_t)b->off.back();
  if (xyz) {
    for (size_t j = 0; j < m; j++)
      if (!std::isfinite(xyz[j])) { b->err = "non-finite coordinates"; return FFXG_ERR_NONFINITE; }
    std::memcpy(b->h_xyz, xyz, m * sizeof(double));
  }
  auto fail_cuda = [&]() {
    b->err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
    return FFXG_ERR_CUDA;
  };
  if (cudaMemcpyAsync(b->d_xyz, b->h_xyz, m * sizeof(double), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    return fail_cuda();
  const int key = want_grad ? 1 : 0;
  std::vector<int> st(S, FFXG_OK);
  bool graph = b->mode != FFXG_BATCH_LOOP && batch_graph_ready(*b);
  if (graph && !b->exec[key]) {
    // Stage by stage when the recordings merge, else one branch per system.
    const bool staged = b->mode == FFXG_BATCH_GRAPH && staged_capture(*b, key) == FFXG_OK;
    if (!staged && batch_capture(*b, key) != FFXG_OK) graph = false;
  }
  std::vector<char> redo(S, graph ? 0 : 1);
  if (graph) {
    if (cudaGraphLaunch(b->exec[key], b->stream) != cudaSuccess) return fail_cuda();
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail_cuda();
    for (size_t s = 0; s < S; s++) {
      Handle &h = handle_of(b->sys[s]);
      h.want_grad = want_grad != 0;
      h.growths = 0;
      if (b->staged[key])   // hand each system the results it staged
        for (const Recorder::Copy &c : b->copies[key][s])
          std::memcpy(c.host, b->h_stage + s * kStageSlot + c.off, c.bytes);
      const int r = eval_after_graph(h, terms + s * FFXG_N_TERMS, counts ? counts + s * FFXG_N_COUNTS : nullptr);
      if (r == -1) {           // a list grew: the batch graph holds the old buffers
        redo[s] = 1;
        batch_drop_graphs(*b);
      } else {
        st[s] = r;
      }
    }
  } else if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
    return fail_cuda();
  }
  for (size_t s = 0; s < S; s++) {
    if (!redo[s]) continue;
    Handle &h = handle_of(b->sys[s]);
    if (!graph) h.growths = 0;   // a graph replay counted its regrowth already
    st[s] = evaluate(h, b->d_xyz + 3 * b->off[s], b->d_grad + 3 * b->off[s], want_grad != 0,
                     terms + s * FFXG_N_TERMS, counts ? counts + s * FFXG_N_COUNTS : nullptr);
  }
  if (want_grad) {
    if (cudaMemcpyAsync(b->h_grad, b->d_grad, m * sizeof(double), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
      return fail_cuda();
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail_cuda();
    std::memcpy(grad, b->h_grad, m * sizeof(double));
  }
  int first = FFXG_OK;
  for (size_t s = 0; s < S; s++) {
    if (status) status[s] = st[s];
    if (st[s] != FFXG_OK && first == FFXG_OK) {
      first = st[s];
      b->err = "system " + std::to_string(s) + ": " + ffxg_last_error(b->sys[s]);
    }
  }
  return first;
}

}  // extern "C"
