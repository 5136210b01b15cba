// Shared device helpers for the voxel_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/voxel_b200.h"

namespace vx {

constexpr uint32_t kWarp = 32;
constexpr uint32_t kFullMask = 0xffffffffu;

// Device-side error codes written into a status word with atomicCAS so the
// first failure wins (the reference's set_edit_status,
// hash_dag_gpu/detail/edit_common.cuh:96-99).
enum DeviceStatus : uint32_t {
  kDevOk = 0,
  kDevCapacity = 1,   // a table, pool or arena ran out
  kDevTimeout = 2,    // a bounded wait gave up
  kDevInvalid = 3,    // malformed input detected on the device
};

__device__ __forceinline__ void set_status(uint32_t *status, uint32_t code) {
  if (status != nullptr) atomicCAS(status, kDevOk, code);
}

inline vx_status status_from_device(uint32_t code) {
  switch (code) {
  case kDevOk: return VX_OK;
  case kDevCapacity: return VX_ERR_CAPACITY;
  case kDevTimeout: return VX_ERR_TIMEOUT;
  default: return VX_ERR_INVALID_VALUE;
  }
}

inline vx_status from_cuda(cudaError_t e) {
  return e == cudaSuccess ? VX_OK : static_cast<vx_status>(e);
}

#define VX_TRY_CUDA(expr)                                                      \
  do {                                                                         \
    cudaError_t vx_e_ = (expr);                                                \
    if (vx_e_ != cudaSuccess) return ::vx::from_cuda(vx_e_);                   \
  } while (0)

#define VX_TRY(expr)                                                           \
  do {                                                                         \
    vx_status vx_s_ = (expr);                                                  \
    if (vx_s_ != VX_OK) return vx_s_;                                          \
  } while (0)

// Nanosecond wall clock of the GPU, used to bound every spin-wait.
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Every device wait gives up after this long and reports kDevTimeout.
constexpr uint64_t kWaitLimitNs = 2000000000ull; // 2 s

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
// Bring the line holding p into L2 (a hint: no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// atomicSub with acquire-release semantics at GPU scope: this thread's earlier
// stores are visible to whoever observes the new value, and the stores that
// earlier releases of the same word published are visible to this thread's
// later loads.  Returns the old value.
__device__ __forceinline__ uint32_t atomic_sub_acq_rel(uint32_t *p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
               : "=r"(old)
               : "l"(p), "r"(0u - v)
               : "memory");
  return old;
}

// Acquire / release fence at GPU scope: after a relaxed load that observed a
// release store, it makes the writer's earlier stores visible.
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// Streaming 128-bit load that does not allocate in L1 (read-once data).
__device__ __forceinline__ uint4 ld_stream_u4(const uint4 *p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// ---- bulk copies (TMA, 1-D, no multicast) and shared-memory mbarriers ----

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of the barrier to complete, for at most
// kWaitLimitNs; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kWaitLimitNs) return false;
  return true;
}
// Global -> shared bulk copy; src, dst 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ uint32_t lane_id() {
  return threadIdx.x & (kWarp - 1u);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// atomicAdd of v (below 32) to a counter by the lanes that arrive here
// together, as one atomic per warp: each lane gets the counter's old value
// plus the sum of the lanes below it, as from its own atomicAdd.  Counters
// that every insert of a hash table bumps serialise in L2 when each lane
// adds on its own.
__device__ __forceinline__ uint32_t warp_atomic_add_small(uint32_t *ctr, uint32_t v) {
  const uint32_t am = __activemask();
  const uint32_t below = am & lanemask_lt();
  uint32_t prefix = 0, total = 0;
#pragma unroll
  for (uint32_t b = 0; b < 5; ++b) {
    const uint32_t bits = __ballot_sync(am, (v >> b) & 1u);
    prefix += static_cast<uint32_t>(__popc(bits & below)) << b;
    total += static_cast<uint32_t>(__popc(bits)) << b;
  }
  const uint32_t leader = __ffs(am) - 1u;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(ctr, total);
  return __shfl_sync(am, base, leader) + prefix;
}

// atomicAdd of 1 to a 64-bit counter by the lanes that arrive together, as
// one atomic per warp.
__device__ __forceinline__ void warp_count_u64(unsigned long long *ctr) {
  const uint32_t am = __activemask();
  if (lane_id() == __ffs(am) - 1u) atomicAdd(ctr, static_cast<unsigned long long>(__popc(am)));
}

template <class T> __device__ __forceinline__ T warp_inclusive_sum(T v) {
#pragma unroll
  for (uint32_t d = 1; d < kWarp; d <<= 1) {
    const T o = __shfl_up_sync(kFullMask, v, d);
    if (lane_id() >= d) v += o;
  }
  return v;
}

template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (uint32_t d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFullMask, v, d);
  return v;
}

inline uint32_t ceil_div(uint64_t a, uint64_t b) {
  return static_cast<uint32_t>((a + b - 1) / b);
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Number of SMs of the current device (cached per process).
int sm_count();

// Carves typed sub-buffers out of one caller-owned workspace, 256-B aligned.
struct Carver {
  char *base;
  size_t offset = 0;
  explicit Carver(void *p) : base(static_cast<char *>(p)) {}
  template <class T> T *take(size_t count) {
    offset = align_up(offset, 256);
    T *p = reinterpret_cast<T *>(base + offset);
    offset += count * sizeof(T);
    return p;
  }
};

// Size-only twin of Carver.
struct Sizer {
  size_t offset = 0;
  template <class T> void take(size_t count) {
    offset = align_up(offset, 256);
    offset += count * sizeof(T);
  }
};

} // namespace vx
