// CUDA graphs of the library's stream-ordered pipelines (internal).
#pragma once

#include "common.cuh"

#include <functional>

struct vx_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0; // kernel launches one replay performs
};

namespace vx::graph {

// Records what body() enqueues on a private stream into an executable graph.
// body must not synchronise or allocate (every pipeline captured here is
// stream-ordered by design).
vx_status capture(const std::function<vx_status(cudaStream_t)> &body, vx_graph **out);

} // namespace vx::graph
