// voxel_b200_compat.hpp - the reference's C++ call shapes over the C ABI.
//
// Existing callers of yamaatsu1112/voxel's algorithm library include
// <algo/cuda/scan.cuh>, <algo/cuda/sort.cuh>, <algo/svt/hash_dag_gpu.cuh> and
// the GPU SVO headers (<algo/svt/cuda/...>) and call templates such as
//     algo::cuda::scan::exclusive_sum(d_data, n, ws, ws_size, stream);
//     algo::cuda::sort::sort_by_key(keys, sort::value_arrays(vals), n, ws, ws_size, stream);
//     algo::svt::hash_dag_gpu::place_voxel_edits(dag.view(), edits, n, ws, ws_size, stream);
// This header provides the same names and argument meanings, forwarding to
// libvoxel_b200.so.  Policy template arguments (Config) that only choose an
// implementation are accepted and ignored, since this library ships one tuned
// implementation per operation; the ones that change results are honoured
// (RadixSort's KeyBits, default 32 for every key type as in the reference).
// Scans with an operator and float sums use voxel_b200_fused_scan.cuh and
// need nvcc, as the reference's headers do.
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

// ------------------------------------------------------------------ scan --
// The reference's scan configs (cuda/scan/block_based.cuh, global.cuh) as tag
// types so that callers' explicit Config arguments compile; every config runs
// this library's one scan (results are identical by contract).
namespace algo::cuda::scan {

struct DirectSharedLayout {};
struct PaddedSharedLayout {};
struct BlockTileReduction {};
template <class BlockScan> struct ScanThenPropagate { using block_scan = BlockScan; };
template <class BlockScan, class ReducePolicy = BlockTileReduction> struct ReduceThenScan {
  using block_scan = BlockScan;
  using reduce_policy = ReducePolicy;
};
template <class BlockScan> struct DecoupledLookback { using block_scan = BlockScan; };
template <class BlockAlgorithm> struct BlockBased { using block_algorithm = BlockAlgorithm; };
template <int BlockSize = 256, int ItemsPerThread = 2, class Layout = DirectSharedLayout>
struct BlellochBlock {};
template <int BlockSize = 256, int ItemsPerThread = 2> struct HillisSteeleBlock {};
template <int BlockSize = 256, int ItemsPerThread = 4> struct WarpShuffleBlock {};
template <class Algorithm> struct Global { using algorithm = Algorithm; };
template <int BlockSize = 256> struct BlellochGlobal {};
template <int BlockSize = 256> struct HillisSteeleGlobal {};

namespace detail {
using DefaultConfig = BlockBased<DecoupledLookback<WarpShuffleBlock<512, 4>>>;
// Sums of 4- and 8-byte integers run the library's scan (wrapping, so signed
// and unsigned sums agree bit for bit); everything else runs the fused scan
// template (nvcc only).
template <class T>
inline constexpr bool kLibrarySum = std::is_integral_v<T> && (sizeof(T) == 4 || sizeof(T) == 8);
} // namespace detail

} // namespace algo::cuda::scan

#ifdef __CUDACC__
#include "voxel_b200_fused_scan.cuh"
namespace algo::cuda::scan {
namespace detail {
template <class T> struct InPlace {
  T *data;
};
template <class T> struct ReadAt {
  __device__ static T run(std::uint32_t i, const InPlace<T> &in) { return in.data[i]; }
};
template <class T> struct WriteAt {
  __device__ static void run(std::uint32_t i, const InPlace<T> &in, T, T prefix) {
    in.data[i] = prefix;
  }
};
template <bool Inclusive, class Op, class T>
inline cudaError_t op_scan(T *d, std::uint32_t count, void *ws, std::size_t ws_size,
                           cudaStream_t stream) {
  static_assert(std::is_arithmetic_v<T> && (sizeof(T) == 4 || sizeof(T) == 8),
                "scans with an operator take 4- or 8-byte integers or floats");
  if (d == nullptr && count != 0) return cudaErrorInvalidValue;
  return vx::fused::fused_scan<Inclusive, Op, ReadAt<T>, WriteAt<T>>(InPlace<T>{d}, count, ws,
                                                                      ws_size, stream);
}
} // namespace detail
} // namespace algo::cuda::scan
#endif

namespace algo::cuda::scan {

// cuda/scan/scan.cuh:113-135, 153-161: workspace of a scan of count values of
// T with operator Op (either of the two implementations fits in it).
template <class Config, class Op, class T>
inline std::size_t required_workspace_size(std::uint32_t count) {
  static_assert(std::is_integral_v<T> || std::is_floating_point_v<T>,
                "scan only supports integral and floating point types");
  std::size_t n = vx_scan_workspace_size(count);
#ifdef __CUDACC__
  if constexpr (sizeof(T) == 4 || sizeof(T) == 8) {
    const std::size_t f = vx::fused::workspace_size<T>(count);
    n = f > n ? f : n;
  }
#endif
  return n;
}
template <class Config, class T>
inline std::size_t required_workspace_size(std::uint32_t count) {
  return required_workspace_size<Config, void, T>(count);
}
template <class T> inline std::size_t required_workspace_size(std::uint32_t count) {
  return required_workspace_size<detail::DefaultConfig, void, T>(count);
}

namespace detail {
template <bool Inclusive, class T>
inline cudaError_t library_sum(T *d, std::uint32_t count, void *ws, std::size_t ws_size,
                               cudaStream_t stream) {
  if constexpr (sizeof(T) == 4) {
    if constexpr (Inclusive)
      return vx_compat::to_cuda(vx_scan_inclusive_sum_u32(
          reinterpret_cast<std::uint32_t *>(d), count, ws, ws_size, stream));
    else
      return vx_compat::to_cuda(vx_scan_exclusive_sum_u32(
          reinterpret_cast<std::uint32_t *>(d), count, ws, ws_size, stream));
  } else {
    static_assert(!Inclusive, "the library's 64-bit scan is exclusive");
    return vx_compat::to_cuda(vx_scan_exclusive_sum_u64(reinterpret_cast<std::uint64_t *>(d),
                                                        count, ws, ws_size, stream));
  }
}
} // namespace detail

// cuda/scan/scan.cuh:137-151 and 123-135
template <class Config, class T>
inline cudaError_t exclusive_sum(T *d_data, std::uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  static_assert(std::is_integral_v<T> || std::is_floating_point_v<T>,
                "scan only supports integral and floating point types");
  if constexpr (detail::kLibrarySum<T>) {
    return detail::library_sum<false>(d_data, count, ws, ws_size, stream);
  } else {
#ifdef __CUDACC__
    return detail::op_scan<false, vx::fused::Plus<T>, T>(d_data, count, ws, ws_size, stream);
#else
    static_assert(detail::kLibrarySum<T>, "float and 1/2-byte sums need nvcc");
    return cudaErrorInvalidValue;
#endif
  }
}
template <class T>
inline cudaError_t exclusive_sum(T *d_data, std::uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  return exclusive_sum<detail::DefaultConfig, T>(d_data, count, ws, ws_size, stream);
}
template <class Config, class T>
inline cudaError_t inclusive_sum(T *d_data, std::uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  static_assert(std::is_integral_v<T> || std::is_floating_point_v<T>,
                "scan only supports integral and floating point types");
  if constexpr (detail::kLibrarySum<T> && sizeof(T) == 4) {
    return detail::library_sum<true>(d_data, count, ws, ws_size, stream);
  } else {
#ifdef __CUDACC__
    return detail::op_scan<true, vx::fused::Plus<T>, T>(d_data, count, ws, ws_size, stream);
#else
    static_assert(sizeof(T) == 4 && std::is_integral_v<T>, "this inclusive sum needs nvcc");
    return cudaErrorInvalidValue;
#endif
  }
}
template <class T>
inline cudaError_t inclusive_sum(T *d_data, std::uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  return inclusive_sum<detail::DefaultConfig, T>(d_data, count, ws, ws_size, stream);
}

#ifdef __CUDACC__
// cuda/scan/scan.cuh:79-111: in-place scans under any associative Op with
// Op::identity() (Plus, Max, or the caller's own).
template <class Config, class Op, class T>
inline cudaError_t inclusive_scan(T *d_data, std::uint32_t count, void *ws,
                                  std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::op_scan<true, Op, T>(d_data, count, ws, ws_size, stream);
}
template <class Op, class T>
inline cudaError_t inclusive_scan(T *d_data, std::uint32_t count, void *ws,
                                  std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::op_scan<true, Op, T>(d_data, count, ws, ws_size, stream);
}
template <class Config, class Op, class T>
inline cudaError_t exclusive_scan(T *d_data, std::uint32_t count, void *ws,
                                  std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::op_scan<false, Op, T>(d_data, count, ws, ws_size, stream);
}
template <class Op, class T>
inline cudaError_t exclusive_scan(T *d_data, std::uint32_t count, void *ws,
                                  std::size_t ws_size, cudaStream_t stream = nullptr) {
  return detail::op_scan<false, Op, T>(d_data, count, ws, ws_size, stream);
}
#endif

} // namespace algo::cuda::scan

// ------------------------------------------------------------------ sort --
namespace algo::cuda::sort {

// cuda/sort/radix.cuh:15-67: the configs as tags.  Only KeyBits changes what
// a sort computes (the low KeyBits bits of each key order it); the pass
// policy, block size and RadixBits pick an implementation in the reference
// and are accepted and ignored here (this library tunes its own).
struct BucketWiseScan {};
struct FlattenedScan {};
template <class ScanPolicy = BucketWiseScan> struct FlagPrefixSumPass {
  using scan_policy = ScanPolicy;
};
struct SharedAtomicHistogram {};
struct WarpBallotHistogram {};
struct WarpLevelMultiSplitHistogram {};
struct BucketBallotWarpRank {};
struct WarpLevelMultiSplitWarpRank {};
struct WarpBallotBlockHistogram {};
struct SharedAtomicGlobalOffsetsBlockHistogram {};
template <class HistogramPolicy, class WarpRankPolicy, int ItemsPerThread> struct HistogramPass {
  static_assert(ItemsPerThread > 0, "HistogramPass requires ItemsPerThread > 0");
};
template <class BlockHistogramPolicy, class LocalRankPolicy,
          class GlobalOffsetsBlockHistogramPolicy, int ItemsPerThread>
struct OneSweepPass {
  static_assert(ItemsPerThread > 0, "OneSweepPass requires ItemsPerThread > 0");
};
template <class PassPolicy, int BlockSize = 256, int RadixBits = 4, int KeyBits = 32>
struct RadixSort {
  static_assert(BlockSize > 0 && RadixBits > 0 && RadixBits < 32 && KeyBits > 0,
                "RadixSort parameters out of range");
  static_assert(KeyBits % RadixBits == 0,
                "RadixSort requires KeyBits to be a multiple of RadixBits");
  using pass_policy = PassPolicy;
  static constexpr int kBlockSize = BlockSize;
  static constexpr int kRadixBits = RadixBits;
  static constexpr int kKeyBits = KeyBits;
};

// cuda/sort/uint_key.cuh:15-66: a key of Words 32-bit words, word 0 least
// significant.
template <std::size_t Words> struct UIntKey {
  static_assert(Words > 0, "UIntKey requires Words > 0");
  std::uint32_t words[Words]{};
  friend bool operator==(const UIntKey &a, const UIntKey &b) {
    for (std::size_t i = 0; i < Words; ++i)
      if (a.words[i] != b.words[i]) return false;
    return true;
  }
};

// cuda/sort/value_arrays.cuh: any number of value arrays, each permuted with
// the keys.
template <class... Values> struct value_arrays_t;
template <> struct value_arrays_t<> {};
template <class First, class... Rest> struct value_arrays_t<First, Rest...> {
  First *first = nullptr;
  value_arrays_t<Rest...> rest{};
};
inline value_arrays_t<> value_arrays() { return {}; }
template <class First, class... Rest>
value_arrays_t<First, Rest...> value_arrays(First *first, Rest *...rest) {
  return {first, value_arrays(rest...)};
}

namespace detail {

// The reference's default (cuda/sort/sort.cuh:21-24): KeyBits = 32 for every
// key type, so a u64 key is ordered by its low 32 bits unless a RadixSort
// config says otherwise.
using DefaultConfig =
    RadixSort<HistogramPass<SharedAtomicHistogram, WarpLevelMultiSplitWarpRank, 4>, 512, 4>;

template <class Key> struct key_words {
  static constexpr bool kSupported =
      std::is_integral_v<Key> && std::is_unsigned_v<Key> && (sizeof(Key) == 4 || sizeof(Key) == 8);
  static constexpr std::uint32_t kWords = sizeof(Key) / 4;
};
template <std::size_t W> struct key_words<UIntKey<W>> {
  static constexpr bool kSupported = W <= 64;
  static constexpr std::uint32_t kWords = static_cast<std::uint32_t>(W);
};

template <class Config, class Key> constexpr std::uint32_t key_bits() {
  static_assert(key_words<Key>::kSupported,
                "this library sorts u32, u64 and UIntKey<W <= 64> keys");
  static_assert(Config::kKeyBits <= 32 * static_cast<int>(key_words<Key>::kWords),
                "KeyBits exceeds the key's width");
  return static_cast<std::uint32_t>(Config::kKeyBits);
}

inline std::size_t align256(std::size_t v) { return (v + 255) & ~std::size_t(255); }

template <class... Values> constexpr std::size_t max_value_bytes() {
  std::size_t m = 0;
  ((m = sizeof(Values) > m ? sizeof(Values) : m), ...);
  return m;
}

// One u32 payload with a u32 / u64 key: the library's pair sort directly.
template <class Key, class... Values> constexpr bool direct_pairs() {
  if constexpr (sizeof...(Values) == 0) {
    return !std::is_class_v<Key>;
  } else if constexpr (sizeof...(Values) == 1) {
    return !std::is_class_v<Key> && max_value_bytes<Values...>() == 4;
  } else {
    return false;
  }
}

template <class Key, class... Values>
std::size_t sort_workspace(std::uint32_t count) {
  if (count <= 1) return 0;
  if constexpr (direct_pairs<Key, Values...>()) {
    return vx_sort_workspace_size(count, sizeof(Key));
  } else {
    const std::uint32_t words = key_words<Key>::kWords;
    return align256(vx_sort_words_workspace_size(count, words)) +
           align256(sizeof(std::uint32_t) * std::size_t(count)) +
           align256(max_value_bytes<Values...>() * std::size_t(count));
  }
}

inline bool all_valid(value_arrays_t<>) { return true; }
template <class F, class... R> bool all_valid(value_arrays_t<F, R...> v) {
  return v.first != nullptr && all_valid(v.rest);
}

inline cudaError_t permute_values(value_arrays_t<>, const std::uint32_t *, void *, std::uint32_t,
                                  cudaStream_t) {
  return cudaSuccess;
}
template <class F, class... R>
cudaError_t permute_values(value_arrays_t<F, R...> v, const std::uint32_t *perm, void *tmp,
                           std::uint32_t count, cudaStream_t stream) {
  vx_status st = vx_gather(tmp, v.first, perm, count, sizeof(F), stream);
  if (st != VX_OK) return vx_compat::to_cuda(st);
  const cudaError_t e = cudaMemcpyAsync(v.first, tmp, sizeof(F) * std::size_t(count),
                                        cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess) return e;
  return permute_values(v.rest, perm, tmp, count, stream);
}

template <class Config, class Key, class... Values>
cudaError_t sort_impl(Key *keys, value_arrays_t<Values...> vals, std::uint32_t count, void *ws,
                      std::size_t ws_size, cudaStream_t stream) {
  static_assert((std::is_trivially_copyable_v<Values> && ...),
                "sort_by_key requires trivially copyable values");
  constexpr std::uint32_t bits = key_bits<Config, Key>();
  if (keys == nullptr && count != 0) return cudaErrorInvalidValue;
  if (count != 0 && !all_valid(vals)) return cudaErrorInvalidValue;
  if (count <= 1) return cudaSuccess;
  if (ws == nullptr || ws_size < sort_workspace<Key, Values...>(count))
    return cudaErrorInvalidValue;
  if constexpr (direct_pairs<Key, Values...>()) {
    std::uint32_t *v = nullptr;
    if constexpr (sizeof...(Values) == 1) v = reinterpret_cast<std::uint32_t *>(vals.first);
    if constexpr (sizeof(Key) == 4)
      return vx_compat::to_cuda(vx_sort_pairs_u32(reinterpret_cast<std::uint32_t *>(keys), v,
                                                  count, bits, ws, ws_size, stream));
    else
      return vx_compat::to_cuda(vx_sort_pairs_u64(reinterpret_cast<std::uint64_t *>(keys), v,
                                                  count, bits, ws, ws_size, stream));
  } else {
    const std::uint32_t words = key_words<Key>::kWords;
    char *base = static_cast<char *>(ws);
    const std::size_t sort_bytes = align256(vx_sort_words_workspace_size(count, words));
    auto *perm = reinterpret_cast<std::uint32_t *>(base + sort_bytes);
    void *tmp = base + sort_bytes + align256(sizeof(std::uint32_t) * std::size_t(count));
    const vx_status st = vx_sort_words(reinterpret_cast<std::uint32_t *>(keys), words, count,
                                       bits, perm, ws, sort_bytes, stream);
    if (st != VX_OK) return vx_compat::to_cuda(st);
    return permute_values(vals, perm, tmp, count, stream);
  }
}

} // namespace detail

// cuda/sort/sort.cuh:100-167
template <class Config, class Key>
inline std::size_t required_workspace_size(std::uint32_t count) {
  (void)detail::key_bits<Config, Key>();
  return detail::sort_workspace<Key>(count);
}
template <class Key> inline std::size_t required_workspace_size(std::uint32_t count) {
  return required_workspace_size<detail::DefaultConfig, Key>(count);
}
template <class Config, class Key, class... Values>
inline std::size_t required_sort_by_key_workspace_size(std::uint32_t count) {
  (void)detail::key_bits<Config, Key>();
  return detail::sort_workspace<Key, Values...>(count);
}
template <class Key, class... Values>
inline std::size_t required_sort_by_key_workspace_size(std::uint32_t count,
                                                       value_arrays_t<Values...>) {
  return required_sort_by_key_workspace_size<detail::DefaultConfig, Key, Values...>(count);
}

template <class Config, class Key>
inline cudaError_t sort_keys(Key *d_keys, std::uint32_t count, void *ws, std::size_t ws_size,
                             cudaStream_t stream = nullptr) {
  return detail::sort_impl<Config, Key>(d_keys, value_arrays(), count, ws, ws_size, stream);
}
template <class Key>
inline cudaError_t sort_keys(Key *d_keys, std::uint32_t count, void *ws, std::size_t ws_size,
                             cudaStream_t stream = nullptr) {
  return sort_keys<detail::DefaultConfig, Key>(d_keys, count, ws, ws_size, stream);
}
template <class Config, class Key, class... Values>
inline cudaError_t sort_by_key(Key *d_keys, value_arrays_t<Values...> d_values,
                               std::uint32_t count, void *ws, std::size_t ws_size,
                               cudaStream_t stream = nullptr) {
  return detail::sort_impl<Config, Key, Values...>(d_keys, d_values, count, ws, ws_size, stream);
}
template <class Key, class... Values>
inline cudaError_t sort_by_key(Key *d_keys, value_arrays_t<Values...> d_values,
                               std::uint32_t count, void *ws, std::size_t ws_size,
                               cudaStream_t stream = nullptr) {
  return sort_by_key<detail::DefaultConfig, Key, Values...>(d_keys, d_values, count, ws, ws_size,
                                                            stream);
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
