// engine.cu -- iteration-loop driver (see engine.cuh).
#include <cstring>
#include <vector>

#include "engine.cuh"

// Loop guard, appended to every WHILE body: counts body executions and stops the
// loop with MG_ERR_TIMEOUT once they exceed the run's iteration cap by a margin,
// so a device-side loop always terminates even if a kernel never signals the end.
__global__ void loop_guard_kernel(DevCtl *c, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  const int32_t it = c->body_iters + 1;
  c->body_iters = it;
  if (c->done) {
    cudaGraphSetConditional(h, 0u);
  } else if ((int64_t)it > (int64_t)c->iter_cap + 8) {
    c->status = MG_ERR_TIMEOUT;
    c->done = 1;
    cudaGraphSetConditional(h, 0u);
  }
}

namespace {

struct CachedLoop {
  std::vector<unsigned char> sig;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

struct EngineCache {
  CachedLoop slots[SLOT_COUNT];
};

EngineCache *cache_of(mg_graph *g) {
  if (!g->cache) g->cache = new EngineCache();
  return static_cast<EngineCache *>(g->cache);
}

void drop(CachedLoop &c) {
  if (c.exec) cudaGraphExecDestroy(c.exec);
  if (c.graph) cudaGraphDestroy(c.graph);
  c.exec = nullptr;
  c.graph = nullptr;
  c.sig.clear();
}

mg_status build_loop(mg_graph *g, CachedLoop &c, const LoopBody &body) {
  cudaGraph_t graph = nullptr;
  MG_CUDA_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    mg_set_error("cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(e));
    return MG_ERR_CUDA;
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    mg_set_error("cudaGraphAddNode(while): %s", cudaGetErrorString(e));
    return MG_ERR_CUDA;
  }
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(g->stream, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    mg_set_error("cudaStreamBeginCaptureToGraph: %s", cudaGetErrorString(e));
    return MG_ERR_CUDA;
  }
  body(g->stream, h, 1);
  loop_guard_kernel<<<1, 32, 0, g->stream>>>(g->ctl, h);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(g->stream, &captured);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    cudaGetLastError();
    mg_set_error("cudaStreamEndCapture: %s", cudaGetErrorString(e));
    return MG_ERR_CUDA;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    cudaGetLastError();
    mg_set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
    return MG_ERR_CUDA;
  }
  c.graph = graph;
  c.exec = exec;
  return MG_OK;
}

}  // namespace

void engine_release_cached(mg_graph *g) {
  if (!g->cache) return;
  EngineCache *ec = static_cast<EngineCache *>(g->cache);
  for (auto &c : ec->slots) drop(c);
  delete ec;
  g->cache = nullptr;
}

mg_status fetch_ctl(mg_graph *g) {
  MG_CUDA_TRY(cudaMemcpyAsync(g->ctl_host, g->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, g->stream));
  MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return MG_OK;
}

mg_status run_loop(mg_graph *g, int slot, const void *sig, size_t sig_len, bool use_graph, const LoopBody &body,
                   int64_t max_iters) {
  if (use_graph) {
    CachedLoop &c = cache_of(g)->slots[slot];
    const unsigned char *sb = static_cast<const unsigned char *>(sig);
    bool hit = c.exec && c.sig.size() == sig_len && std::memcmp(c.sig.data(), sb, sig_len) == 0;
    if (!hit) {
      drop(c);
      MG_TRY(build_loop(g, c, body));
      c.sig.assign(sb, sb + sig_len);
    }
    MG_CUDA_TRY(cudaGraphLaunch(c.exec, g->stream));
    return MG_OK;
  }
  for (int64_t it = 0; it < max_iters; it++) {
    g->host_iters = it + 1;
    body(g->stream, 0, 0);
    MG_CUDA_TRY(cudaGetLastError());
    MG_CUDA_TRY(cudaMemcpyAsync(&g->ctl_host->done, &g->ctl->done, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                g->stream));
    MG_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (g->ctl_host->done) return MG_OK;
  }
  mg_set_error("host-driven loop did not finish within %lld iterations", (long long)max_iters);
  return MG_ERR_TIMEOUT;
}
