// Voxel-list front end shared by the plain (per-call) DAG and SVO paths:
// voxels are sorted by leaf Morton key and OR-reduced into one leaf-mask
// primitive per touched leaf (the reference's build_leaf_masks,
// hash_dag_gpu/detail/build_leaf_masks/pipeline.cuh:81-116).
#pragma once

#include "common.cuh"

namespace vx::plain {
size_t workspace_size(uint32_t count);
vx_status prepare(const vx_voxel *edits, uint32_t count, uint32_t depth,
                  uint32_t op, uint32_t material, void *workspace,
                  const vx_primitive **out_prims, const uint32_t **out_count,
                  cudaStream_t s);
vx_status prepare_leaf_commands(const vx_leaf_command *cmds, uint32_t count, uint32_t depth,
                                uint32_t op, uint32_t material, void *workspace,
                                const vx_primitive **out_prims, const uint32_t **out_count,
                                cudaStream_t s);
} // namespace vx::plain
