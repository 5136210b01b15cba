// voxel_b200_compat.hpp - the reference's C++ call shapes over the C ABI.
//
// Existing callers of yamaatsu1112/voxel's algorithm library include
// <algo/cuda/scan.cuh>, <algo/cuda/sort.cuh>, <algo/svt/hash_dag_gpu.cuh> and
// the GPU SVO headers (<algo/svt/cuda/...>) and call templates such as
//     algo::cuda::scan::exclusive_sum(d_data, n, ws, ws_size, stream);
//     algo::cuda::sort::sort_by_key(keys, sort::value_arrays(vals), n, ws, ws_size, stream);
//     algo::svt::hash_dag_gpu::place_voxel_edits(dag.view(), edits, n, ws, ws_size, stream);
// This header provides the same names and argument meanings, forwarding to
// libvoxel_b200.so; policy template arguments (Config) are accepted and
// ignored, since this library ships one tuned implementation per operation.
// Returns are cudaError_t as in the reference; this library's own codes
// (capacity, timeout) map to cudaErrorMemoryAllocation / cudaErrorLaunchTimeout.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <type_traits>

#include "voxel_b200.h"

namespace vx_compat {
inline cudaError_t to_cuda(vx_status s) {
  if (s == VX_ERR_CAPACITY) return cudaErrorMemoryAllocation;
  if (s == VX_ERR_TIMEOUT) return cudaErrorLaunchTimeout;
  if (s == VX_ERR_NO_DEVICE) return cudaErrorNoDevice;
  return static_cast<cudaError_t>(s);
}
} // namespace vx_compat

namespace algo::cuda::scan {

// cuda/scan/scan.cuh:153-161
template <class T, class... Config>
inline std::size_t required_workspace_size(std::uint32_t count) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "u32 / u64 scans");
  return vx_scan_workspace_size(count);
}

// cuda/scan/scan.cuh:137-151 (Config ignored)
template <class... Config, class T>
inline cudaError_t exclusive_sum(T *d_data, std::uint32_t count, void *ws,
                                 std::size_t ws_size, cudaStream_t stream = nullptr) {
  static_assert(std::is_integral_v<T> && (sizeof(T) == 4 || sizeof(T) == 8),
                "this library scans 32- and 64-bit integers");
  if constexpr (sizeof(T) == 4)
    return vx_compat::to_cuda(vx_scan_exclusive_sum_u32(
        reinterpret_cast<std::uint32_t *>(d_data), count, ws, ws_size, stream));
  else
    return vx_compat::to_cuda(vx_scan_exclusive_sum_u64(
        reinterpret_cast<std::uint64_t *>(d_data), count, ws, ws_size, stream));
}

// cuda/scan/scan.cuh:123-135 (u32)
template <class... Config, class T>
inline cudaError_t inclusive_sum(T *d_data, std::uint32_t count, void *ws,
                                 std::size_t ws_size, cudaStream_t stream = nullptr) {
  static_assert(std::is_integral_v<T> && sizeof(T) == 4, "u32 inclusive scan");
  return vx_compat::to_cuda(vx_scan_inclusive_sum_u32(
      reinterpret_cast<std::uint32_t *>(d_data), count, ws, ws_size, stream));
}

} // namespace algo::cuda::scan

namespace algo::cuda::sort {

// One value array of u32 (cuda/sort/value_arrays.cuh).
template <class V> struct ValueArrays1 {
  V *values;
};
template <class V> inline ValueArrays1<V> value_arrays(V *values) {
  static_assert(sizeof(V) == 4, "u32 payload");
  return ValueArrays1<V>{values};
}

// cuda/sort/sort.cuh:130-167 (KeyBits = all key bits; use vx_sort_pairs_* for
// fewer).
template <class Key, class... Rest>
inline std::size_t required_sort_by_key_workspace_size(std::uint32_t count) {
  return vx_sort_workspace_size(count, sizeof(Key));
}
template <class Key, class... Config>
inline std::size_t required_workspace_size(std::uint32_t count) {
  return vx_sort_workspace_size(count, sizeof(Key));
}

template <class... Config, class Key, class V>
inline cudaError_t sort_by_key(Key *keys, ValueArrays1<V> vals, std::uint32_t count,
                               void *ws, std::size_t ws_size,
                               cudaStream_t stream = nullptr) {
  static_assert(std::is_unsigned_v<Key> && (sizeof(Key) == 4 || sizeof(Key) == 8));
  if constexpr (sizeof(Key) == 4)
    return vx_compat::to_cuda(vx_sort_pairs_u32(
        reinterpret_cast<std::uint32_t *>(keys),
        reinterpret_cast<std::uint32_t *>(vals.values), count, 32, ws, ws_size, stream));
  else
    return vx_compat::to_cuda(vx_sort_pairs_u64(
        reinterpret_cast<std::uint64_t *>(keys),
        reinterpret_cast<std::uint32_t *>(vals.values), count, 64, ws, ws_size, stream));
}

template <class... Config, class Key>
inline cudaError_t sort_keys(Key *keys, std::uint32_t count, void *ws,
                             std::size_t ws_size, cudaStream_t stream = nullptr) {
  static_assert(std::is_unsigned_v<Key> && (sizeof(Key) == 4 || sizeof(Key) == 8));
  if constexpr (sizeof(Key) == 4)
    return vx_compat::to_cuda(vx_sort_pairs_u32(reinterpret_cast<std::uint32_t *>(keys),
                                                nullptr, count, 32, ws, ws_size, stream));
  else
    return vx_compat::to_cuda(vx_sort_pairs_u64(reinterpret_cast<std::uint64_t *>(keys),
                                                nullptr, count, 64, ws, ws_size, stream));
}

} // namespace algo::cuda::sort

namespace algo::svt::hash_dag_gpu {

// hash_dag_gpu/types.cuh:11-15
struct VoxelEdit {
  std::uint32_t x, y, z;
};
static_assert(sizeof(VoxelEdit) == sizeof(vx_voxel));

enum class EditOp { Place, Destroy };

// The view passed to edit calls (hash_dag_gpu/device_view.cuh:14-31): here a
// handle of the resident DAG.
struct DeviceHashDagGpu {
  vx_dag *dag;
};

// hash_dag_gpu/storage.cuh:16-105: RAII owner, non-copyable, non-movable.
// BucketCount / OverflowSlabCount are read as a capacity hint.
template <std::uint32_t BucketCount = 1024, std::uint32_t OverflowSlabCount = 1024>
class HashDagGpu {
public:
  explicit HashDagGpu(std::uint32_t depth = 8,
                      std::uint64_t max_nodes = std::uint64_t(BucketCount) * 31 +
                                                std::uint64_t(OverflowSlabCount) * 31) {
    vx_dag_config cfg{depth, 0, max_nodes < 16 ? 16 : max_nodes, 0};
    status_ = vx_compat::to_cuda(vx_dag_create(&cfg, &dag_));
  }
  ~HashDagGpu() {
    if (dag_) vx_dag_destroy(dag_);
  }
  HashDagGpu(const HashDagGpu &) = delete;
  HashDagGpu &operator=(const HashDagGpu &) = delete;
  HashDagGpu(HashDagGpu &&) = delete;
  HashDagGpu &operator=(HashDagGpu &&) = delete;

  [[nodiscard]] cudaError_t status() const { return status_; }
  [[nodiscard]] DeviceHashDagGpu view() const { return DeviceHashDagGpu{dag_}; }
  cudaError_t reset(cudaStream_t stream = nullptr) {
    return vx_compat::to_cuda(vx_dag_reset(dag_, stream));
  }

private:
  vx_dag *dag_ = nullptr;
  cudaError_t status_ = cudaSuccess;
};

// hash_dag_gpu/edit.cuh:16-61
template <class... Config>
inline std::size_t apply_voxel_edits_workspace_size(std::uint32_t count) {
  return vx_dag_voxel_workspace_size(count);
}

template <class... Config>
inline cudaError_t apply_voxel_edits(DeviceHashDagGpu dag, const VoxelEdit *edits,
                                     std::uint32_t count, EditOp op, void *ws,
                                     std::size_t ws_size, cudaStream_t stream = nullptr) {
  return vx_compat::to_cuda(vx_dag_apply_voxels(
      dag.dag, reinterpret_cast<const vx_voxel *>(edits), count,
      op == EditOp::Place ? VX_EDIT_PLACE : VX_EDIT_DESTROY, ws, ws_size, stream));
}

template <class... Config>
inline cudaError_t place_voxel_edits(DeviceHashDagGpu dag, const VoxelEdit *edits,
                                     std::uint32_t count, void *ws, std::size_t ws_size,
                                     cudaStream_t stream = nullptr) {
  return apply_voxel_edits(dag, edits, count, EditOp::Place, ws, ws_size, stream);
}

template <class... Config>
inline cudaError_t destroy_voxel_edits(DeviceHashDagGpu dag, const VoxelEdit *edits,
                                       std::uint32_t count, void *ws, std::size_t ws_size,
                                       cudaStream_t stream = nullptr) {
  return apply_voxel_edits(dag, edits, count, EditOp::Destroy, ws, ws_size, stream);
}

} // namespace algo::svt::hash_dag_gpu

namespace algo::svt::cuda {

// svt/cuda/voxel/types.cuh, svt/cuda/detail/edit_common.cuh
struct VoxelEdit {
  std::uint32_t x, y, z;
};
static_assert(sizeof(VoxelEdit) == sizeof(vx_voxel));
enum class EditOp { Place, Destroy };

// svt/cuda/terminal/types.cuh:15-31 (same layouts)
using TerminalNodeInput = vx_terminal_node;
using TerminalLeafInput = vx_terminal_leaf;
struct TerminalPlainDepthwiseAllocation {};
struct TerminalCompactAllDepthAllocation {};
struct TerminalDepthwiseRelease {};
struct TerminalFrontierRelease {};
template <class Allocation, class Release> struct TerminalEditConfig {
  using allocation = Allocation;
  using release = Release;
};
using DefaultTerminalEditConfig =
    TerminalEditConfig<TerminalCompactAllDepthAllocation, TerminalFrontierRelease>;

// The view passed to edit calls (svt/cuda/device_view.cuh:11-44): a handle.
struct DeviceGpuSvo {
  vx_svo *svo;
};

// svt/cuda/storage.cuh:12-122: RAII owner of a depth-10 (4096^3) SVO with
// MaxNodeCount nodes and MaxLeafCount leaves; movable, not copyable.
template <std::uint32_t MaxNodeCount = 131072, std::uint32_t MaxLeafCount = 524288>
class GpuSvo {
public:
  GpuSvo() {
    vx_svo_config cfg{10, 0, MaxNodeCount, MaxLeafCount, 0};
    status_ = vx_compat::to_cuda(vx_svo_create(&cfg, &svo_));
  }
  ~GpuSvo() {
    if (svo_) vx_svo_destroy(svo_);
  }
  GpuSvo(const GpuSvo &) = delete;
  GpuSvo &operator=(const GpuSvo &) = delete;
  GpuSvo(GpuSvo &&o) noexcept : svo_(o.svo_), status_(o.status_) { o.svo_ = nullptr; }
  GpuSvo &operator=(GpuSvo &&o) noexcept {
    if (this != &o) {
      if (svo_) vx_svo_destroy(svo_);
      svo_ = o.svo_;
      status_ = o.status_;
      o.svo_ = nullptr;
    }
    return *this;
  }
  [[nodiscard]] cudaError_t status() const { return status_; }
  [[nodiscard]] DeviceGpuSvo view() const { return DeviceGpuSvo{svo_}; }

private:
  vx_svo *svo_ = nullptr;
  cudaError_t status_ = cudaSuccess;
};

// svt/cuda/svo.cuh:17-22
inline cudaError_t reset_svo(DeviceGpuSvo svo, cudaStream_t stream = nullptr) {
  return vx_compat::to_cuda(vx_svo_reset(svo.svo, stream));
}

// svt/cuda/voxel/edit.cuh:38-92 (Config ignored)
template <class... Config>
inline std::size_t apply_voxel_edits_workspace_size(std::uint32_t count) {
  return vx_svo_voxel_workspace_size(count);
}
template <class... Config>
inline cudaError_t place_voxel_edits(DeviceGpuSvo svo, const VoxelEdit *edits,
                                     std::uint32_t count, void *ws, std::size_t ws_size,
                                     cudaStream_t stream = nullptr) {
  return vx_compat::to_cuda(vx_svo_apply_voxels(svo.svo, reinterpret_cast<const vx_voxel *>(edits),
                                                count, VX_EDIT_PLACE, 1, ws, ws_size, stream));
}
template <class... Config>
inline cudaError_t destroy_voxel_edits(DeviceGpuSvo svo, const VoxelEdit *edits,
                                       std::uint32_t count, void *ws, std::size_t ws_size,
                                       cudaStream_t stream = nullptr) {
  return vx_compat::to_cuda(vx_svo_apply_voxels(svo.svo, reinterpret_cast<const vx_voxel *>(edits),
                                                count, VX_EDIT_DESTROY, 0, ws, ws_size, stream));
}

namespace detail {
// svt/cuda/terminal/detail/workspace/edit.cuh:125-134; the request capacity
// is not needed here (inputs become a fixed number of primitives).
template <class Allocation, class Release>
inline std::size_t apply_terminal_edits_workspace_size(std::uint32_t node_count,
                                                       std::uint32_t leaf_count,
                                                       std::uint32_t = 0) {
  return vx_terminal_workspace_size(node_count, leaf_count);
}
template <class Allocation, class Release>
inline cudaError_t apply_terminal_edits(DeviceGpuSvo svo, const TerminalNodeInput *nodes,
                                        std::uint32_t node_count,
                                        const TerminalLeafInput *leaves,
                                        std::uint32_t leaf_count, EditOp op, void *ws,
                                        std::size_t ws_size, cudaStream_t stream = nullptr) {
  return vx_compat::to_cuda(vx_svo_apply_terminal(
      svo.svo, nodes, node_count, leaves, leaf_count,
      op == EditOp::Place ? VX_EDIT_PLACE : VX_EDIT_DESTROY, 1, ws, ws_size, stream));
}
} // namespace detail

// svt/cuda/terminal/detail/pipeline.cuh:200-222
template <class Config = DefaultTerminalEditConfig>
inline cudaError_t place_terminal_edits(DeviceGpuSvo svo, const TerminalNodeInput *nodes,
                                        std::uint32_t node_count,
                                        const TerminalLeafInput *leaves,
                                        std::uint32_t leaf_count, void *ws,
                                        std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::apply_terminal_edits<typename Config::allocation, typename Config::release>(
      svo, nodes, node_count, leaves, leaf_count, EditOp::Place, ws, ws_size, stream);
}
template <class Config = DefaultTerminalEditConfig>
inline cudaError_t destroy_terminal_edits(DeviceGpuSvo svo, const TerminalNodeInput *nodes,
                                          std::uint32_t node_count,
                                          const TerminalLeafInput *leaves,
                                          std::uint32_t leaf_count, void *ws,
                                          std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::apply_terminal_edits<typename Config::allocation, typename Config::release>(
      svo, nodes, node_count, leaves, leaf_count, EditOp::Destroy, ws, ws_size, stream);
}

} // namespace algo::svt::cuda
