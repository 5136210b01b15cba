// voxel_b200_compat.hpp - the reference's C++ call shapes over the C ABI.
//
// Existing callers of yamaatsu1112/voxel's algorithm library include
// <algo/cuda/scan.cuh>, <algo/cuda/sort.cuh> and <algo/svt/hash_dag_gpu.cuh>
// and call templates such as
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
