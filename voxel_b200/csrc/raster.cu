// Rasterise sphere / box primitives into voxel lists: the input shape of the
// plain per-call edit path (the reference's voxel sphere generator,
// bench/bench_cuda_svt.cu:37-80, as a GPU kernel).  One block per primitive;
// each thread owns (y, z) rows, whose x-runs are computed in closed form
// (integer square root for spheres), and a block scan places the runs.
#include "common.cuh"
#include "profile.cuh"

namespace vx::raster {

constexpr uint32_t kBlock = 256;

__device__ __forceinline__ int64_t isqrt64(int64_t v) {
  if (v <= 0) return 0;
  int64_t r = static_cast<int64_t>(sqrt(static_cast<double>(v)));
  while (r * r > v) --r;
  while ((r + 1) * (r + 1) <= v) ++r;
  return r;
}

// x-run [x0, x1] (inclusive, clipped) of primitive p on row (y, z); empty if
// x1 < x0.
__device__ __forceinline__ void row_run(const vx_primitive &p, int64_t world,
                                        int64_t y, int64_t z, int64_t &x0,
                                        int64_t &x1) {
  int64_t half;
  if (vx_prim_shape(&p) == VX_SHAPE_SPHERE) {
    const int64_t r = p.r[0], dy = y - p.c[1], dz = z - p.c[2];
    const int64_t rem = r * r - dy * dy - dz * dz;
    if (rem < 0) {
      x0 = 1;
      x1 = 0;
      return;
    }
    half = isqrt64(rem);
  } else {
    int64_t lo, hi;
    vx_prim_axis_range(&p, 0, &lo, &hi);
    x0 = max((int64_t)0, lo);
    x1 = min((int64_t)(world - 1), hi);
    return;
  }
  x0 = max((int64_t)0, (int64_t)p.c[0] - half);
  x1 = min((int64_t)(world - 1), (int64_t)p.c[0] + half);
}

__device__ __forceinline__ void row_range(const vx_primitive &p, int64_t world,
                                          int64_t &y0, int64_t &ny, int64_t &z0,
                                          int64_t &nz) {
  int64_t ylo, yhi, zlo, zhi;
  if (vx_prim_shape(&p) == VX_SHAPE_SPHERE) {
    ylo = (int64_t)p.c[1] - p.r[0];
    yhi = (int64_t)p.c[1] + p.r[0];
    zlo = (int64_t)p.c[2] - p.r[0];
    zhi = (int64_t)p.c[2] + p.r[0];
  } else {
    vx_prim_axis_range(&p, 1, &ylo, &yhi);
    vx_prim_axis_range(&p, 2, &zlo, &zhi);
  }
  y0 = max((int64_t)0, ylo);
  z0 = max((int64_t)0, zlo);
  const int64_t y1 = min((int64_t)(world - 1), yhi);
  const int64_t z1 = min((int64_t)(world - 1), zhi);
  ny = y1 >= y0 ? y1 - y0 + 1 : 0;
  nz = z1 >= z0 ? z1 - z0 + 1 : 0;
}

__global__ void __launch_bounds__(kBlock)
    count_kernel(const vx_primitive *prims, uint32_t n, uint32_t world_exp,
                 uint64_t *counts) {
  const vx_primitive p = prims[blockIdx.x];
  const int64_t world = int64_t(1) << world_exp;
  int64_t y0, ny, z0, nz;
  row_range(p, world, y0, ny, z0, nz);
  uint64_t total = 0;
  for (int64_t row = threadIdx.x; row < ny * nz; row += kBlock) {
    int64_t x0, x1;
    row_run(p, world, y0 + row % ny, z0 + row / ny, x0, x1);
    if (x1 >= x0) total += static_cast<uint64_t>(x1 - x0 + 1);
  }
  total = warp_sum<uint64_t>(total);
  __shared__ uint64_t s[kBlock / kWarp];
  if (lane_id() == 0) s[threadIdx.x / kWarp] = total;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (uint32_t w = 0; w < kBlock / kWarp; ++w) t += s[w];
    counts[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kBlock)
    emit_kernel(const vx_primitive *prims, uint32_t n, uint32_t world_exp,
                const uint64_t *offsets, vx_voxel *out) {
  const vx_primitive p = prims[blockIdx.x];
  const int64_t world = int64_t(1) << world_exp;
  int64_t y0, ny, z0, nz;
  row_range(p, world, y0, ny, z0, nz);
  uint64_t base = offsets[blockIdx.x];
  __shared__ uint64_t s_warp[kBlock / kWarp];
  __shared__ uint64_t s_total;
  const int64_t rows = ny * nz;
  for (int64_t r0 = 0; r0 < rows; r0 += kBlock) {
    const int64_t row = r0 + threadIdx.x;
    int64_t x0 = 1, x1 = 0, y = 0, z = 0;
    if (row < rows) {
      y = y0 + row % ny;
      z = z0 + row / ny;
      row_run(p, world, y, z, x0, x1);
    }
    const uint64_t len = x1 >= x0 ? static_cast<uint64_t>(x1 - x0 + 1) : 0;
    const uint64_t inc = warp_inclusive_sum<uint64_t>(len);
    if (lane_id() == kWarp - 1) s_warp[threadIdx.x / kWarp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t t = 0;
      for (uint32_t w = 0; w < kBlock / kWarp; ++w) {
        const uint64_t v = s_warp[w];
        s_warp[w] = t;
        t += v;
      }
      s_total = t;
    }
    __syncthreads();
    const uint64_t at = base + s_warp[threadIdx.x / kWarp] + inc - len;
    for (uint64_t k = 0; k < len; ++k)
      out[at + k] = vx_voxel{static_cast<uint32_t>(x0 + k), static_cast<uint32_t>(y),
                             static_cast<uint32_t>(z)};
    base += s_total;
    __syncthreads();
  }
}

} // namespace vx::raster

extern "C" {

vx_status vx_rasterize_count(const vx_primitive *prims, uint32_t count,
                             uint32_t world_exp, uint64_t *out_counts,
                             vx_stream stream) {
  if ((prims == nullptr || out_counts == nullptr) && count != 0) return VX_ERR_INVALID_VALUE;
  if (world_exp < 2 || world_exp > 30) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("raster_count", s);
  vx::raster::count_kernel<<<count, vx::raster::kBlock, 0, s>>>(prims, count, world_exp,
                                                                out_counts);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_rasterize(const vx_primitive *prims, uint32_t count,
                       uint32_t world_exp, const uint64_t *offsets,
                       vx_voxel *out, vx_stream stream) {
  if ((prims == nullptr || offsets == nullptr || out == nullptr) && count != 0)
    return VX_ERR_INVALID_VALUE;
  if (world_exp < 2 || world_exp > 30) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("raster_emit", s);
  vx::raster::emit_kernel<<<count, vx::raster::kBlock, 0, s>>>(prims, count, world_exp,
                                                               offsets, out);
  return vx::from_cuda(cudaGetLastError());
}

} // extern "C"
