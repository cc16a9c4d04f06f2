// graph.cu -- capture a sequence of op_par_loop calls as one CUDA graph.
//
// The reference launches every loop from the host and synchronises after
// each block colour and each reduction (airfoil/res_calc_kernel.cu:230,
// update_kernel.cu:162-165): about 15 host round trips per airfoil
// iteration.  Captured, a whole outer iteration (save_soln + 2 x (adt_calc,
// res_calc, bres_calc, update)) becomes one graph launch; reductions stay on
// the device in their result slots (deferred mode) until op2b_sync().

#include <string>
#include <vector>

#include "loops.h"

namespace op2b {

// A captured kernel that skips reading a dataset because the dataset held
// zeros when the capture began (res after airfoil's update).  A launch at a
// time the dataset may hold other values sets the kernel's parameter to the
// dataset's buffer and, where the skipping kernel is a variant that ignores
// it, the variant that reads it (and writes its zeros) in its place; a later
// launch with the zeros known again puts the captured kernel back.
struct ZeroEntry {
  op_dat dat = nullptr;
  cudaGraphNode_t node = nullptr;  // nullptr: the node could not be identified
  int arg = 0, nparams = 0;
  void *buf = nullptr;
  const void *read_kernel = nullptr;  // nullptr: the captured kernel reads the buffer
  int read_grid = 0;
  bool skipping = true;  // the form the instantiated graph has now
};

struct Graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nkernels = 0;
  std::vector<Runtime::CapturedLoop> loops;
  std::vector<GblRequest> reductions;  // deferred results each launch refreshes
  std::vector<ZeroEntry> zero_entries;
  std::vector<std::pair<int, unsigned char>> zero_effects;  // on the known-zero flags
};

static bool g_prev_deferred = false;
static int g_live_graphs = 0;
static std::vector<ZeroEntry> g_capture_zero_entries;

int live_graphs() { return g_live_graphs; }

void capture_zero_entry(op_dat d, int arg, int nparams, void *buf, const void *read_kernel,
                        int read_grid) {
  ZeroEntry z;
  z.dat = d;
  z.arg = arg;
  z.nparams = nparams;
  z.buf = buf;
  z.read_kernel = read_kernel;
  z.read_grid = read_grid;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t *deps = nullptr;
  const cudaGraphEdgeData *edges = nullptr;
  size_t n = 0;
  if (cudaStreamGetCaptureInfo_v3(rt().stream, &st, nullptr, nullptr, &deps, &edges, &n) ==
          cudaSuccess &&
      st == cudaStreamCaptureStatusActive && n == 1) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(deps[0], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
      z.node = deps[0];
  }
  cudaGetLastError();
  g_capture_zero_entries.push_back(z);
}

// set each recorded kernel to skip or read its dataset as the dataset's
// known-zero flag says now; false (with the error set) when a kernel that
// must read cannot be changed
static bool zero_entries_match(Graph *g) {
  for (ZeroEntry &z : g->zero_entries) {
    const bool zero = dat_known_zero(z.dat);
    if (zero == z.skipping) continue;
    if (!z.node || z.nparams <= z.arg) {
      fail(-1, "op2b error: graph launch: dataset \"%s\" held zeros when the graph was "
               "captured and may not now; capture the graph again\n",
           z.dat->name ? z.dat->name : "");
      return false;
    }
    // the graph's own node holds the captured (skipping) form
    cudaKernelNodeParams kp;
    cudaError_t e = cudaGraphKernelNodeGetParams(z.node, &kp);
    std::vector<void *> args;
    void *ptr = z.buf;
    if (e == cudaSuccess && !zero) {
      args.assign(kp.kernelParams, kp.kernelParams + z.nparams);
      args[z.arg] = &ptr;
      kp.kernelParams = args.data();
      kp.extra = nullptr;
      if (z.read_kernel) {
        kp.func = const_cast<void *>(z.read_kernel);
        kp.gridDim = dim3((unsigned)z.read_grid);
      }
    }
    if (e == cudaSuccess) e = cudaGraphExecKernelNodeSetParams(g->exec, z.node, &kp);
    if (e != cudaSuccess) {
      fail(-1, "op2b error: graph launch: cannot update a kernel for dataset \"%s\": %s\n",
           z.dat->name ? z.dat->name : "", cudaGetErrorString(e));
      return false;
    }
    z.skipping = zero;
  }
  return true;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

static size_t g_pending_mark = 0;

int op2b_capture_begin(int profile) {
  ensure_cuda();
  if (error_pending()) return 0;
  Runtime &R = rt();
  flush_pending();  // loops held back before the capture run outside the graph
  ahead_drop();     // a graph bakes dataset pointers: nothing may be swapped in later
  tile_capture_begin();
  known_zero_capture_begin();
  g_capture_zero_entries.clear();
  deliver_deferred();
  g_pending_mark = red_pending_count();
  R.capture_events.clear();
  R.capture_profile = profile != 0;
  g_prev_deferred = R.gbl_deferred;
  R.gbl_deferred = true;
  cudaError_t e = cudaStreamBeginCapture(R.stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    R.gbl_deferred = g_prev_deferred;
    R.capture_profile = false;
    known_zero_capture_end();
    fail(-1, "op2b error: cannot start graph capture: %s\n", cudaGetErrorString(e));
    return 0;
  }
  return 1;
}

void *op2b_capture_end(void) {
  flush_pending();
  tile_capture_end();  // the graph leaves every dataset in the buffer it found
  Runtime &R = rt();
  Graph *g = new Graph();
  g->zero_effects = known_zero_capture_end();
  g->zero_entries.swap(g_capture_zero_entries);
  cudaError_t e = cudaStreamEndCapture(R.stream, &g->graph);
  R.capture_profile = false;
  R.gbl_deferred = g_prev_deferred;
  g->reductions = red_take_pending_since(g_pending_mark);
  red_reserve_for_graph();
  if (e != cudaSuccess) {
    delete g;
    fail(-1, "op2b error: graph capture failed: %s\n", cudaGetErrorString(e));
    return nullptr;
  }
  g->loops.swap(R.capture_events);
  size_t n = 0;
  OP2B_CUDA(cudaGraphGetNodes(g->graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) OP2B_CUDA(cudaGraphGetNodes(g->graph, nodes.data(), &n));
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    OP2B_CUDA(cudaGraphNodeGetType(nd, &t));
    g->nkernels += (t == cudaGraphNodeTypeKernel);
  }
  e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g->graph);
    delete g;
    fail(-1, "op2b error: graph instantiation failed: %s\n", cudaGetErrorString(e));
    return nullptr;
  }
  g_live_graphs++;
  return g;
}

int op2b_graph_launch(void *h) {
  Graph *g = (Graph *)h;
  if (!g) return (int)cudaErrorInvalidValue;
  if (!zero_entries_match(g)) return -1;
  red_replace_pending(g->reductions);
  const cudaError_t e = cudaGraphLaunch(g->exec, rt().stream);
  if (e == cudaSuccess) known_zero_apply(g->zero_effects);
  return (int)e;
}

int op2b_graph_nloops(void *h) { return h ? (int)((Graph *)h)->loops.size() : -1; }

int op2b_graph_nkernels(void *h) { return h ? ((Graph *)h)->nkernels : -1; }

char const *op2b_graph_loop_name(void *h, int i) {
  Graph *g = (Graph *)h;
  if (!g || i < 0 || i >= (int)g->loops.size()) return "";
  return g->loops[i].name.c_str();
}

int op2b_graph_loop_times(void *h, double *seconds, int n) {
  Graph *g = (Graph *)h;
  if (!g) return -1;
  int k = 0;
  for (auto &l : g->loops) {
    if (k >= n) break;
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(l.stop);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, l.start, l.stop);
    if (e != cudaSuccess) return -(int)e;
    seconds[k++] = ms * 1e-3;
  }
  return k;
}

void op2b_graph_destroy(void *h) {
  Graph *g = (Graph *)h;
  if (!g) return;
  cudaStreamSynchronize(rt().stream);
  for (auto &l : g->loops) {
    cudaEventDestroy(l.start);
    cudaEventDestroy(l.stop);
  }
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  if (g_live_graphs > 0) g_live_graphs--;
}

}  // extern "C"
