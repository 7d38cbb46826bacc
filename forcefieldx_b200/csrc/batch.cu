// batch.cu -- batches of independent periodic systems (include/ffxcuda.h, ffxg_batch_*).
//
// Many small boxes of uneven size (conformer, rotamer or lambda-window energies) are
// launch-bound one at a time: a 96-atom system runs ~150 kernels of a few blocks each.
// A batch keeps one handle per system (its own lists, grids and solver state) and
// captures every system's whole evaluation -- the PCG loop as each system's own
// conditional WHILE node -- as independent branches of ONE CUDA graph, so a batch
// evaluation is one host->device copy of all coordinates, one graph launch, and one
// device->host copy of all gradients.  The branches run concurrently on the device, each
// system stopping its solver on its own convergence test.  LOOP mode evaluates the same
// systems one after another through the single-system path, for comparison.
//
// Results are the single-system results bit for bit: each branch is the graph a
// single-system handle captures for itself, on the same buffers.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ffx_internal.cuh"

using namespace ffx;

struct ffxg_batch {
  std::vector<ffxg_handle *> sys;
  std::vector<int64_t> off;              // first atom of each system; off[n] = total atoms
  int mode = FFXG_BATCH_GRAPH;
  double *d_xyz = nullptr, *d_grad = nullptr;    // [total][3] on the device
  double *h_xyz = nullptr, *h_grad = nullptr;    // pinned mirrors
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};  // by want_grad
  std::vector<int64_t> gen;               // each handle's graph generation at capture
  int64_t graph_builds = 0;
  std::string err;
};

static std::string g_batch_create_error;

static void batch_drop_graphs(ffxg_batch &b) {
  for (cudaGraphExec_t &g : b.exec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static void batch_free(ffxg_batch &b) {
  batch_drop_graphs(b);
  for (ffxg_handle *h : b.sys) ffxg_destroy(h);
  b.sys.clear();
  if (b.d_xyz) cudaFree(b.d_xyz);
  if (b.d_grad) cudaFree(b.d_grad);
  if (b.h_xyz) cudaFreeHost(b.h_xyz);
  if (b.h_grad) cudaFreeHost(b.h_grad);
  if (b.ev_fork) cudaEventDestroy(b.ev_fork);
  if (b.ev_join) cudaEventDestroy(b.ev_join);
  if (b.stream) cudaStreamDestroy(b.stream);
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
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
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
  if (mode != FFXG_BATCH_GRAPH && mode != FFXG_BATCH_LOOP) { b->err = "unknown batch mode"; return FFXG_ERR_BAD_ARG; }
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
  bool graph = b->mode == FFXG_BATCH_GRAPH && batch_graph_ready(*b);
  if (graph && !b->exec[key] && batch_capture(*b, key) != FFXG_OK) graph = false;
  std::vector<char> redo(S, graph ? 0 : 1);
  if (graph) {
    if (cudaGraphLaunch(b->exec[key], b->stream) != cudaSuccess) return fail_cuda();
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail_cuda();
    for (size_t s = 0; s < S; s++) {
      Handle &h = handle_of(b->sys[s]);
      h.want_grad = want_grad != 0;
      h.growths = 0;
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
