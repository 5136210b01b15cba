// A user's CUDA code reading this library's structures through
// voxel_b200_device.cuh: built by tests/test_gpu_device_api.py with nvcc,
// launched through the extern "C" functions below.
#include "voxel_b200_device.cuh"

namespace {

__global__ void dag_points(vx_dag_view v, const vx_voxel *pts, uint32_t n, uint8_t *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = vx_dag_get_voxel(v, pts[i].x, pts[i].y, pts[i].z);
}

__global__ void svo_points(vx_svo_view v, const vx_voxel *pts, uint32_t n, uint8_t *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = vx_svo_get_voxel(v, pts[i].x, pts[i].y, pts[i].z);
}

// Every lane of every warp calls the warp-cooperative lookup (inactive past n).
__global__ void slab_contains(vx_slab_set_view v, const uint64_t *keys, uint32_t n,
                              uint32_t *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  const bool found = vx_slab_set_contains_warp(v, active ? keys[i] : 0ull, active);
  if (active) out[i] = found ? 1u : 0u;
}

__global__ void cuckoo_values(vx_cuckoo_view v, const uint64_t *keys, uint32_t n,
                              uint32_t *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t value = VX_HASH_NOT_FOUND_VALUE;
  vx_cuckoo_find(v, keys[i], &value);
  out[i] = value;
}

inline uint32_t blocks(uint32_t n) { return (n + 255u) / 256u; }

} // namespace

extern "C" {
int user_dag_points(const vx_dag_view *v, const vx_voxel *p, uint32_t n, uint8_t *o) {
  dag_points<<<blocks(n), 256>>>(*v, p, n, o);
  return (int)cudaDeviceSynchronize();
}
int user_svo_points(const vx_svo_view *v, const vx_voxel *p, uint32_t n, uint8_t *o) {
  svo_points<<<blocks(n), 256>>>(*v, p, n, o);
  return (int)cudaDeviceSynchronize();
}
int user_slab_contains(const vx_slab_set_view *v, const uint64_t *k, uint32_t n, uint32_t *o) {
  slab_contains<<<blocks(n), 256>>>(*v, k, n, o);
  return (int)cudaDeviceSynchronize();
}
int user_cuckoo_values(const vx_cuckoo_view *v, const uint64_t *k, uint32_t n, uint32_t *o) {
  cuckoo_values<<<blocks(n), 256>>>(*v, k, n, o);
  return (int)cudaDeviceSynchronize();
}
}
