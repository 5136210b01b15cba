/* voxel_b200_fused_scan.cuh - fused transform -> scan -> post-op (nvcc only).
 *
 * One pass over `count` indices: value i = Transform::run(i, input), the
 * inclusive or exclusive scan of the values under an associative Op, and
 * PostScan::run(i, input, value_i, prefix_i) for every index - the shape of
 * the reference's algo::cuda::scan::{inclusive,exclusive}_scan_fused
 * (cuda/scan/fused.cuh:102-269), which callers use for stream compaction,
 * run-length offsets and allocation (counts -> offsets -> writes) without
 * materialising the values.  Header-only: Transform, PostScan and Op are the
 * caller's device types.
 *
 *   struct Op       { __device__ T operator()(T, T) const; static T identity(); }
 *   struct Transform{ __device__ static T run(uint32_t i, const Input &in); }
 *   struct PostScan { __device__ static void run(uint32_t i, const Input &in,
 *                                                T value, T prefix); }
 *
 * Design: 256 threads x 8 items per tile, tiles taken in the order of a
 * global counter (a tile only waits on tiles already taken by running
 * blocks), a warp-parallel decoupled look-back over 32 predecessors per round
 * trip that combines them in index order (Op need only be associative), and a
 * globaltimer bound on every wait (on timeout a status word in the workspace
 * is set and the tile uses the prefix it has).  The workspace holds that
 * status, the tile counter and one record per tile; it is zero bytes when the
 * input fits one tile.
 */
#ifndef VOXEL_B200_FUSED_SCAN_CUH
#define VOXEL_B200_FUSED_SCAN_CUH

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <utility>

namespace vx::fused {

template <class T> struct Plus {
  __host__ __device__ constexpr T operator()(T a, T b) const { return a + b; }
  __host__ __device__ static constexpr T identity() { return T(0); }
};
// Smallest / largest value of an arithmetic type (infinities for floats).
template <class T> __host__ __device__ constexpr T lowest_of() {
  if constexpr (std::is_floating_point_v<T>) {
    if constexpr (sizeof(T) == 4) return -__builtin_huge_valf();
    else return -__builtin_huge_val();
  } else if constexpr (std::is_signed_v<T>) {
    using U = std::make_unsigned_t<T>;
    return static_cast<T>(U(1) << (sizeof(T) * 8 - 1));
  } else {
    return T(0);
  }
}
template <class T> __host__ __device__ constexpr T highest_of() {
  if constexpr (std::is_floating_point_v<T>) {
    if constexpr (sizeof(T) == 4) return __builtin_huge_valf();
    else return __builtin_huge_val();
  } else {
    using U = std::make_unsigned_t<T>;
    return std::is_signed_v<T> ? static_cast<T>(U(~U(0)) >> 1) : static_cast<T>(~U(0));
  }
}
template <class T> struct Max {
  __host__ __device__ constexpr T operator()(T a, T b) const { return a < b ? b : a; }
  __host__ __device__ static constexpr T identity() { return lowest_of<T>(); }
};
template <class T> struct Min {
  __host__ __device__ constexpr T operator()(T a, T b) const { return b < a ? b : a; }
  __host__ __device__ static constexpr T identity() { return highest_of<T>(); }
};

constexpr uint32_t kBlock = 256;
constexpr uint32_t kItems = 8;
constexpr uint32_t kTile = kBlock * kItems;
constexpr uint64_t kWaitNs = 2000000000ull;

template <class Input, class Transform>
using value_t = std::remove_cv_t<std::remove_reference_t<decltype(
    Transform::run(std::declval<uint32_t>(), std::declval<const Input &>()))>>;

// Look-back record of one tile: the aggregate, the inclusive prefix and a
// state word written last (release) and read first (acquire).
template <class T> struct Record {
  T aggregate;
  T inclusive;
  uint32_t state; // 0 not ready, 1 aggregate, 2 inclusive
};

struct Header {
  uint32_t tile_counter;
  uint32_t status; // nonzero after a look-back timed out
};

template <class T> inline size_t workspace_size(uint32_t count) {
  const uint32_t tiles = (count + kTile - 1) / kTile;
  if (tiles <= 1) return 0;
  return 256 + sizeof(Record<T>) * static_cast<size_t>(tiles);
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <class T> __device__ __forceinline__ T shfl_down(T v, uint32_t d) {
  if constexpr (sizeof(T) <= 4) {
    return __shfl_down_sync(0xffffffffu, v, d);
  } else {
    static_assert(sizeof(T) == 8, "4- or 8-byte scan values");
    uint64_t u;
    memcpy(&u, &v, 8);
    u = __shfl_down_sync(0xffffffffu, u, d);
    T r;
    memcpy(&r, &u, 8);
    return r;
  }
}
template <class T> __device__ __forceinline__ T shfl_up(T v, uint32_t d) {
  if constexpr (sizeof(T) <= 4) {
    return __shfl_up_sync(0xffffffffu, v, d);
  } else {
    uint64_t u;
    memcpy(&u, &v, 8);
    u = __shfl_up_sync(0xffffffffu, u, d);
    T r;
    memcpy(&r, &u, 8);
    return r;
  }
}
template <class T> __device__ __forceinline__ T shfl(T v, uint32_t src) {
  if constexpr (sizeof(T) <= 4) {
    return __shfl_sync(0xffffffffu, v, src);
  } else {
    uint64_t u;
    memcpy(&u, &v, 8);
    u = __shfl_sync(0xffffffffu, u, src);
    T r;
    memcpy(&r, &u, 8);
    return r;
  }
}

// Inclusive warp scan in lane order.
template <class Op, class T> __device__ __forceinline__ T warp_inclusive(T v) {
  const uint32_t lane = threadIdx.x & 31u;
  const Op op{};
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const T o = shfl_up(v, d);
    if (lane >= d) v = op(o, v);
  }
  return v;
}

template <class T> __device__ __forceinline__ void publish(Record<T> *r, uint32_t state, T v) {
  if (state == 2) r->inclusive = v;
  else r->aggregate = v;
  __threadfence();
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(&r->state), "r"(state) : "memory");
}

// Called by warp 0: the tile's exclusive prefix (valid in every lane).
template <class Op, class T>
__device__ T lookback(Record<T> *records, uint32_t tile, T aggregate, uint32_t *status) {
  const uint32_t lane = threadIdx.x & 31u;
  const Op op{};
  if (lane == 0) publish(records + tile, tile == 0 ? 2u : 1u, aggregate);
  if (tile == 0) return Op::identity();
  T exclusive = Op::identity(); // combination of the tiles after the window
  int64_t pos = static_cast<int64_t>(tile) - 1;
  const uint64_t t0 = now_ns();
  for (;;) {
    const int64_t p = pos - static_cast<int64_t>(lane); // lane 0 = nearest
    uint32_t st = 2;
    T v = Op::identity();
    if (p >= 0) {
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(st) : "l"(&records[p].state)
                   : "memory");
      __threadfence();
      if (st == 2) v = *(volatile T *)&records[p].inclusive;
      else if (st == 1) v = *(volatile T *)&records[p].aggregate;
    }
    const uint32_t inc = __ballot_sync(0xffffffffu, st == 2);
    const uint32_t nr = __ballot_sync(0xffffffffu, st == 0);
    const uint32_t limit = inc ? (__ffs(inc) - 1u) : 31u;
    const uint32_t range = limit == 31u ? 0xffffffffu : ((1u << (limit + 1u)) - 1u);
    if (nr & range) {
      if (now_ns() - t0 > kWaitNs) {
        if (lane == 0) atomicExch(status, 1u);
        break;
      }
      __nanosleep(32);
      continue;
    }
    // Combine lanes limit..0 in index order (farthest tile on the left).
    T w = lane <= limit ? v : Op::identity();
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const T o = shfl_down(w, d);
      if (lane + d < 32) w = op(o, w);
    }
    exclusive = op(shfl(w, 0), exclusive);
    if (inc) break;
    pos -= 32;
  }
  if (lane == 0) publish(records + tile, 2u, op(exclusive, aggregate));
  return exclusive;
}

template <bool Inclusive, class Op, class T, class Input, class Transform, class PostScan>
__global__ void __launch_bounds__(kBlock)
    fused_scan_kernel(Input input, uint32_t count, Header *hdr, Record<T> *records) {
  __shared__ T s_warp[kBlock / 32];
  __shared__ T s_prefix;
  __shared__ uint32_t s_tile;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const Op op{};
  if (t == 0) s_tile = hdr ? atomicAdd(&hdr->tile_counter, 1u) : blockIdx.x;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = static_cast<uint64_t>(tile) * kTile + static_cast<uint64_t>(t) * kItems;
  // Thread t owns kItems consecutive indices.
  T val[kItems];
  T run = Op::identity();
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    const uint64_t i = base + k;
    val[k] = i < count ? Transform::run(static_cast<uint32_t>(i), input) : Op::identity();
    run = op(run, val[k]);
  }
  const T incl = warp_inclusive<Op>(run);
  if (lane == 31) s_warp[warp] = incl;
  const T up = shfl_up(incl, 1); // every lane shuffles, then lane 0 drops it
  const T thread_excl_in_warp = lane == 0 ? Op::identity() : up;
  __syncthreads();
  if (warp == 0) {
    const T w = lane < kBlock / 32 ? s_warp[lane] : Op::identity();
    const T wi = warp_inclusive<Op>(w);
    const T aggregate = shfl(wi, kBlock / 32 - 1);
    const T wup = shfl_up(wi, 1);
    if (lane < kBlock / 32) s_warp[lane] = lane == 0 ? Op::identity() : wup;
    const T prefix = records ? lookback<Op>(records, tile, aggregate, &hdr->status)
                             : Op::identity();
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  T acc = op(op(s_prefix, s_warp[warp]), thread_excl_in_warp);
#pragma unroll
  for (uint32_t k = 0; k < kItems; ++k) {
    const uint64_t i = base + k;
    const T before = acc;
    acc = op(acc, val[k]);
    if (i < count) PostScan::run(static_cast<uint32_t>(i), input, val[k], Inclusive ? acc : before);
  }
}

template <bool Inclusive, class Op, class Transform, class PostScan, class Input>
cudaError_t fused_scan(Input input, uint32_t count, void *workspace, size_t workspace_bytes,
                       cudaStream_t stream) {
  using T = value_t<Input, Transform>;
  static_assert(std::is_arithmetic_v<T> && (sizeof(T) == 4 || sizeof(T) == 8),
                "fused scan values are 4- or 8-byte integers or floats");
  if (count == 0) return cudaSuccess;
  const uint32_t tiles = (count + kTile - 1) / kTile;
  const size_t need = workspace_size<T>(count);
  if (need != 0 && (workspace == nullptr || workspace_bytes < need)) return cudaErrorInvalidValue;
  Header *hdr = nullptr;
  Record<T> *records = nullptr;
  if (need != 0) {
    hdr = static_cast<Header *>(workspace);
    records = reinterpret_cast<Record<T> *>(static_cast<char *>(workspace) + 256);
    const cudaError_t e = cudaMemsetAsync(workspace, 0, need, stream);
    if (e != cudaSuccess) return e;
  }
  fused_scan_kernel<Inclusive, Op, T, Input, Transform, PostScan>
      <<<tiles, kBlock, 0, stream>>>(input, count, hdr, records);
  return cudaGetLastError();
}

} // namespace vx::fused

// The reference's names (cuda/scan/fused.cuh:219-269, ops.cuh), forwarding to
// the template above, so callers of algo::cuda::scan keep their code.
namespace algo::cuda::scan {

template <class T> using Plus = vx::fused::Plus<T>;
template <class T> using Max = vx::fused::Max<T>;

template <class Op, class ScanValue> std::size_t required_workspace_size_fused(uint32_t count) {
  return vx::fused::workspace_size<ScanValue>(count);
}
template <class ScanValue> std::size_t required_workspace_size_fused(uint32_t count) {
  return vx::fused::workspace_size<ScanValue>(count);
}
template <class Op, class Transform, class PostScan, class Input>
cudaError_t inclusive_scan_fused(Input input, uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  return vx::fused::fused_scan<true, Op, Transform, PostScan>(input, count, ws, ws_size, stream);
}
template <class Op, class Transform, class PostScan, class Input>
cudaError_t exclusive_scan_fused(Input input, uint32_t count, void *ws, std::size_t ws_size,
                                 cudaStream_t stream = nullptr) {
  return vx::fused::fused_scan<false, Op, Transform, PostScan>(input, count, ws, ws_size, stream);
}
template <class Transform, class PostScan, class Input>
cudaError_t inclusive_sum_fused(Input input, uint32_t count, void *ws, std::size_t ws_size,
                                cudaStream_t stream = nullptr) {
  using T = vx::fused::value_t<Input, Transform>;
  return vx::fused::fused_scan<true, Plus<T>, Transform, PostScan>(input, count, ws, ws_size,
                                                                   stream);
}
template <class Transform, class PostScan, class Input>
cudaError_t exclusive_sum_fused(Input input, uint32_t count, void *ws, std::size_t ws_size,
                                cudaStream_t stream = nullptr) {
  using T = vx::fused::value_t<Input, Transform>;
  return vx::fused::fused_scan<false, Plus<T>, Transform, PostScan>(input, count, ws, ws_size,
                                                                    stream);
}

} // namespace algo::cuda::scan

#endif /* VOXEL_B200_FUSED_SCAN_CUH */
