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
  bool xyz_valid = true;   // h_xyz holds accepted coordinates (false after a rejected copy)
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
  std::vector<cudaStream_t> group_streams;        // one per concurrent group of systems
  // Autotuning of the number of groups: the choice (0 until the first staged build) and
  // the candidates' measured milliseconds per batch.
  int tuned_groups = 0;
  int tune_groups[4] = {0, 0, 0, 0};
  float tune_ms[4] = {0, 0, 0, 0};
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
  for (cudaStream_t st : b.group_streams) cudaStreamDestroy(st);
  b.group_streams.clear();
}

// The systems' recordings merged into stages, phase by phase: a stage is (phase, kernel
// instance, its k-th launch in that phase) and gathers the systems that have it; the
// stages are put in an order that keeps every system's own order (Kahn's algorithm,
// earliest recorded position first).  Systems share no data, so any such order is
// correct for each of them.  False when one stage's block size differs between systems
// or the orders cannot be reconciled.
static bool merge_recordings(const std::vector<Recorder> &rec, const std::vector<int> &group, std::vector<Stage> &out,
                             std::string &why) {
  out.clear();
  for (int phase = 0; phase < 3; phase++) {
    std::map<std::tuple<const void *, int>, int> id;
    std::vector<Stage> nodes;
    std::vector<std::set<int>> succ;
    for (int s : group) {
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

// Record every system's evaluation (rec[s]: its launches, phases and result copies).
static int record_all(ffxg_batch &b, int key, std::vector<Recorder> &rec) {
  const size_t S = b.sys.size();
  rec.assign(S, Recorder{});
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
  return FFXG_OK;
}

// The systems split into `groups` groups of near-equal atom count (longest first, each to
// the lightest group), each group in system order.
static std::vector<std::vector<int>> split_groups(const ffxg_batch &b, int groups) {
  const int S = (int)b.sys.size();
  groups = std::max(1, std::min(groups, S));
  std::vector<int> order(S);
  for (int s = 0; s < S; s++) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return b.off[x + 1] - b.off[x] > b.off[y + 1] - b.off[y];
  });
  std::vector<std::vector<int>> out(groups);
  std::vector<int64_t> load(groups, 0);
  for (int s : order) {
    const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    out[g].push_back(s);
    load[g] += b.off[s + 1] - b.off[s];
  }
  for (auto &g : out) std::sort(g.begin(), g.end());
  return out;
}

// The stage-by-stage graph of the recordings with the systems in `groups` groups: each
// group is one branch of the graph (its stages, its own solver loop), so the groups' kernels
// overlap on the device.  On success *exec and *tab hold the graph and its argument tables.
static int build_staged(ffxg_batch &b, const std::vector<Recorder> &rec, int groups, cudaGraphExec_t *exec_out,
                        unsigned char **tab_out, int *n_stages) {
  const std::vector<std::vector<int>> part = split_groups(b, groups);
  const int G = (int)part.size();
  std::vector<std::vector<Stage>> stages(G);
  *n_stages = 0;
  for (int g = 0; g < G; g++) {
    if (!merge_recordings(rec, part[g], stages[g], b.err)) return FFXG_ERR_CUDA;
    *n_stages += (int)stages[g].size();
  }
  // Argument tables: per stage the block prefix, the packed arguments and (loop stages)
  // each system's solver flag; then per group the flags of its systems in the loop.
  size_t bytes = 0;
  for (auto &sg : stages)
    for (Stage &st : sg) {
      const size_t ns = st.sys.size();
      st.off_pre = bytes = align_up(bytes, 16);
      bytes += (ns + 1) * sizeof(int);
      st.off_pack = bytes = align_up(bytes, 16);
      bytes += ns * st.pack_size;
      st.off_cont = bytes = align_up(bytes, 16);
      if (st.phase == 1) bytes += ns * sizeof(const int *);
    }
  std::vector<unsigned char> tab(std::max<size_t>(bytes, 16), 0);
  std::vector<size_t> off_loop(G);
  std::vector<int> n_loop(G, 0);
  for (int g = 0; g < G; g++) {
    std::set<int> in_loop;
    for (Stage &st : stages[g]) {
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
    off_loop[g] = align_up(tab.size(), 16);
    tab.resize(off_loop[g] + std::max<size_t>(1, in_loop.size()) * sizeof(const int *));
    size_t j = 0;
    for (int sidx : in_loop) {
      const int *c = &handle_of(b.sys[sidx]).d_pcg->cont;
      std::memcpy(tab.data() + off_loop[g] + (j++) * sizeof(const int *), &c, sizeof(c));
    }
    n_loop[g] = (int)in_loop.size();
  }
  unsigned char *d_tab = nullptr;
  if (cudaMalloc(&d_tab, tab.size()) != cudaSuccess ||
      cudaMemcpy(d_tab, tab.data(), tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    if (d_tab) cudaFree(d_tab);
    b.err = "batch stage tables: could not be uploaded";
    return FFXG_ERR_CUDA;
  }
  for (int g = (int)b.group_streams.size(); g < G; g++) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(d_tab);
      b.err = "batch streams could not be created";
      return FFXG_ERR_CUDA;
    }
    b.group_streams.push_back(st);
  }

  // One branch per group: phase 0, the loop (a WHILE node whose body is phase 1 and the
  // loop test), phase 2; after the join the results are read back in one copy.
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    cudaEventRecord(b.ev_fork, b.stream);
    for (int g = 0; g < G && ok; g++) {
      cudaStream_t gs = b.group_streams[g];
      ok = cudaStreamWaitEvent(gs, b.ev_fork, 0) == cudaSuccess;
      for (const Stage &st : stages[g])
        if (st.phase == 0) launch_stage(st, d_tab, gs);
      if (ok && n_loop[g] > 0) {
        const int *const *d_loop = reinterpret_cast<const int *const *>(d_tab + off_loop[g]);
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        cudaGraphConditionalHandle cond{};
        ok = cudaStreamGetCaptureInfo(gs, &cs, nullptr, &cg, &deps, &ndeps) == cudaSuccess &&
             cudaGraphConditionalHandleCreate(&cond, cg, 0, cudaGraphCondAssignDefault) == cudaSuccess;
        if (ok) {
          k_batch_cond<<<1, 32, 0, gs>>>(d_loop, n_loop[g], cond);
          ok = cudaStreamGetCaptureInfo(gs, &cs, nullptr, &cg, &deps, &ndeps) == cudaSuccess;
        }
        cudaGraphNodeParams cp = {};
        cudaGraphNode_t node;
        if (ok) {
          cp.type = cudaGraphNodeTypeConditional;
          cp.conditional.handle = cond;
          cp.conditional.type = cudaGraphCondTypeWhile;
          cp.conditional.size = 1;
          ok = cudaGraphAddNode(&node, cg, deps, ndeps, &cp) == cudaSuccess &&
               cudaStreamUpdateCaptureDependencies(gs, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
        }
        if (ok) {
          cudaGraph_t body = cp.conditional.phGraph_out[0];
          ok = cudaStreamBeginCaptureToGraph(b.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
               cudaSuccess;
          if (ok) {
            for (const Stage &st : stages[g])
              if (st.phase == 1) launch_stage(st, d_tab, b.side);
            k_batch_cond<<<1, 32, 0, b.side>>>(d_loop, n_loop[g], cond);
            ok = cudaStreamEndCapture(b.side, &body) == cudaSuccess;
          }
        }
      }
      for (const Stage &st : stages[g])
        if (st.phase == 2) launch_stage(st, d_tab, gs);
      cudaEventRecord(b.ev_join, gs);
      cudaStreamWaitEvent(b.stream, b.ev_join, 0);
    }
    cudaMemcpyAsync(b.h_stage, b.d_stage, b.sys.size() * kStageSlot, cudaMemcpyDeviceToHost, b.stream);
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
  *exec_out = exec;
  *tab_out = d_tab;
  return FFXG_OK;
}

// The stage-by-stage graph for key.  The number of groups (concurrent branches) is the
// batch's autotuned choice: on the first build each candidate (1, 2, 4, 8 groups, at
// most one per system) is built and timed over two replays after one, and the fastest
// kept; ffxg_batch_tuning reports the choice and the times.  A batch whose systems use
// the ASPC predictor (whose history every evaluation advances) is not timed: it takes
// four groups.
static int staged_capture(ffxg_batch &b, int key) {
  std::vector<Recorder> rec;
  if (int st = record_all(b, key, rec)) return st;
  bool aspc = false;
  for (ffxg_handle *hh : b.sys) aspc = aspc || handle_of(hh).scf_predictor == FFXG_PREDICTOR_ASPC;
  std::vector<int> cand;
  if (b.tuned_groups > 0) cand = {b.tuned_groups};
  else if (aspc) cand = {4};
  else
    for (int g : {1, 2, 4, 8})
      if (g == 1 || g <= (int)b.sys.size()) cand.push_back(g);
  cudaGraphExec_t best = nullptr;
  unsigned char *best_tab = nullptr;
  int best_groups = 0, best_stages = 0;
  float best_ms = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool timing = cand.size() > 1;
  if (timing) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
  }
  for (int g : cand) {
    cudaGraphExec_t ex = nullptr;
    unsigned char *tb = nullptr;
    int ns = 0;
    if (build_staged(b, rec, g, &ex, &tb, &ns) != FFXG_OK) continue;
    float ms = 0.f;
    if (timing) {
      bool ok = cudaGraphLaunch(ex, b.stream) == cudaSuccess;
      ok = ok && cudaEventRecord(e0, b.stream) == cudaSuccess;
      for (int r = 0; r < 2 && ok; r++) ok = cudaGraphLaunch(ex, b.stream) == cudaSuccess;
      ok = ok && cudaEventRecord(e1, b.stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
      if (!ok || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphExecDestroy(ex);
        cudaFree(tb);
        continue;
      }
      ms *= 0.5f;
      for (size_t k = 0; k < 4; k++)
        if (b.tune_groups[k] == g || b.tune_groups[k] == 0) {
          b.tune_groups[k] = g;
          b.tune_ms[k] = ms;
          break;
        }
    }
    if (!best || ms < best_ms) {
      if (best) {
        cudaGraphExecDestroy(best);
        cudaFree(best_tab);
      }
      best = ex;
      best_tab = tb;
      best_ms = ms;
      best_groups = g;
      best_stages = ns;
    } else {
      cudaGraphExecDestroy(ex);
      cudaFree(tb);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!best) return FFXG_ERR_CUDA;
  b.tuned_groups = best_groups;
  b.exec[key] = best;
  b.d_tab[key] = best_tab;
  b.staged[key] = true;
  b.n_stages[key] = best_stages;
  b.copies[key].resize(rec.size());
  for (size_t s = 0; s < rec.size(); s++) b.copies[key][s] = rec[s].copies;
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

int32_t ffxg_batch_tuning(const ffxg_batch *b, int32_t *candidates, double *ms) {
  if (!b) return -1;
  for (int k = 0; k < 4; k++) {
    if (candidates) candidates[k] = b->tune_groups[k];
    if (ms) ms[k] = b->tune_ms[k];
  }
  return b->tuned_groups;
}

int ffxg_batch_set_groups(ffxg_batch *b, int32_t groups) {
  if (!b || groups < 0 || groups > 64) return FFXG_ERR_BAD_ARG;
  if (groups != b->tuned_groups) batch_drop_graphs(*b);
  b->tuned_groups = groups;
  for (int k = 0; k < 4; k++) { b->tune_groups[k] = 0; b->tune_ms[k] = 0.f; }
  return FFXG_OK;
}

int ffxg_batch_energy(ffxg_batch *b, const double *xyz, int want_grad, double *terms, double *grad, int64_t *counts,
                      int32_t *status) {
  if (!b || !terms || (want_grad && !grad)) return FFXG_ERR_BAD_ARG;
  const size_t S = b->sys.size();
  const size_t m = 3 * (size_t)b->off.back();
  // Checked while copied (one pass, several host threads); a rejected copy leaves no
  // coordinates to reuse.
  if (xyz) {
    b->xyz_valid = copy_finite_parallel(b->h_xyz, xyz, m);
    if (!b->xyz_valid) {
      b->err = "non-finite coordinates";
      return FFXG_ERR_NONFINITE;
    }
  } else if (!b->xyz_valid) {
    b->err = "no coordinates to reuse: the last ones were rejected";
    return FFXG_ERR_BAD_ARG;
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
    copy_parallel(grad, b->h_grad, m);
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
