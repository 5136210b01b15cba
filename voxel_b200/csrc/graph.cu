// The batched edit pipelines as CUDA graphs: a capture records every kernel,
// memset and copy of one edit once; each replay is a single launch, which
// matters for small batches (the serving loop's), where ~40 launches per edit
// would otherwise cost more than the kernels.
#include "graph.cuh"
#include "profile.cuh"

#include <new>

namespace vx::graph {

vx_status capture(const std::function<vx_status(cudaStream_t)> &body, vx_graph **out) {
  if (out == nullptr) return VX_ERR_INVALID_VALUE;
  *out = nullptr;
  cudaStream_t s = nullptr;
  VX_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const uint64_t before = prof::launch_count();
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return from_cuda(e);
  }
  const vx_status st = body(s);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(s, &g);
  cudaStreamDestroy(s);
  const uint64_t kernels = prof::launch_count() - before;
  prof::add_launches(-static_cast<int64_t>(kernels)); // captured, not run
  if (st != VX_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return st != VX_OK ? st : from_cuda(e);
  }
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return from_cuda(e);
  }
  auto *r = new (std::nothrow) vx_graph;
  if (r == nullptr) {
    cudaGraphExecDestroy(ex);
    cudaGraphDestroy(g);
    return VX_ERR_MEMORY_ALLOCATION;
  }
  r->graph = g;
  r->exec = ex;
  r->kernels = kernels;
  *out = r;
  return VX_OK;
}

} // namespace vx::graph

extern "C" {

vx_status vx_graph_launch(vx_graph *graph, vx_stream stream) {
  if (graph == nullptr) return VX_ERR_INVALID_VALUE;
  VX_TRY_CUDA(cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream)));
  vx::prof::add_launches(static_cast<int64_t>(graph->kernels));
  return VX_OK;
}

vx_status vx_graph_kernels(const vx_graph *graph, uint64_t *host_kernels) {
  if (graph == nullptr || host_kernels == nullptr) return VX_ERR_INVALID_VALUE;
  *host_kernels = graph->kernels;
  return VX_OK;
}

vx_status vx_graph_destroy(vx_graph *graph) {
  if (graph == nullptr) return VX_OK;
  cudaGraphExecDestroy(graph->exec);
  cudaGraphDestroy(graph->graph);
  delete graph;
  return VX_OK;
}

} // extern "C"
