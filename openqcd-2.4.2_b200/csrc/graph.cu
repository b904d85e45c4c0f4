// CUDA graphs for launch sequences that repeat with the same arguments: the
// SAP preconditioner (ncy cycles of two colours, each a block-solver launch
// and a boundary launch, with the copies around them) is applied to the same
// few work fields at every GCR step.  The first application with a given set
// of arguments is captured from the stream and instantiated; later ones
// replay the executable graph with one launch.  The key is the byte image of
// everything the captured kernels were given (field pointers, geometry,
// parameters, launch variant), so a replay runs exactly the launches the
// capture saw.
#include "lib.h"
#include <cstring>

namespace qcd {

namespace {
struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec = nullptr;
  unsigned long long last = 0;
};
std::vector<GraphEntry> g_graphs;
unsigned long long g_tick = 0;
// the batched deflated solver with two masses per batch keeps about 80
// graphs alive (SAP sequences, orthogonalisation passes, little-solver
// iterations); two alternating mass pairs need about twice that
const size_t kMaxGraphs = 256;
}  // namespace

void graphs_release() {
  for (auto &e : g_graphs)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  g_graphs.clear();
}

size_t graphs_cached() { return g_graphs.size(); }

int graph_run(Ctx &c, const void *key, size_t keylen, cudaStream_t st, const std::function<int()> &launch) {
  if (!c.use_graphs) return launch();
  const unsigned char *k = (const unsigned char *)key;
  for (auto &e : g_graphs)
    if (e.key.size() == keylen && std::memcmp(e.key.data(), k, keylen) == 0) {
      e.last = ++g_tick;
      return cudaGraphLaunch(e.exec, st) == cudaSuccess ? 0 : fail("graph launch failed");
    }
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return fail("stream capture could not start");
  const int rc = launch();
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);
  if (rc || ce != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    // the sequence did something a capture cannot hold: run it directly
    return rc ? rc : launch();
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    cudaGetLastError();
    return launch();
  }
  if (g_graphs.size() >= kMaxGraphs) {   // drop the least recently used
    size_t old = 0;
    for (size_t i = 1; i < g_graphs.size(); i++)
      if (g_graphs[i].last < g_graphs[old].last) old = i;
    cudaGraphExecDestroy(g_graphs[old].exec);
    g_graphs.erase(g_graphs.begin() + old);
  }
  GraphEntry e;
  e.key.assign(k, k + keylen);
  e.exec = exec;
  e.last = ++g_tick;
  g_graphs.push_back(std::move(e));
  return cudaGraphLaunch(exec, st) == cudaSuccess ? 0 : fail("graph launch failed");
}

}  // namespace qcd
