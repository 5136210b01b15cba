// In-place prefix sums (uint32 / uint64, wrapping), one kernel launch after a
// small memset of the look-back records.  See scan.cuh for the design.
#include "profile.cuh"
#include "scan.cuh"

#include <mutex>

namespace vx {

int sm_count() {
  static int cached = 0;
  if (cached == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 148;
  }
  return cached;
}

namespace scan {

namespace {

template <class T> typename RecordsFor<T>::type make_records(const ScanLayout &ws) {
  typename RecordsFor<T>::type r;
  if constexpr (sizeof(T) == 4) {
    r.rec = ws.rec_a;
  } else {
    r.agg = ws.rec_a;
    r.inc = ws.rec_b;
    r.state = ws.rec_state;
  }
  return r;
}

template <class T, bool Inclusive, bool Vectorised>
__global__ void __launch_bounds__(TileShape<T>::kBlock, 2)
    scan_kernel(T *__restrict__ data, uint32_t count, ScanLayout ws,
                typename RecordsFor<T>::type records) {
  using S = TileShape<T>;
  __shared__ uint32_t s_tile;
  __shared__ T s_warp[S::kWarps][S::kRows];
  __shared__ T s_row_off[S::kRows];
  __shared__ T s_prefix;

  if (threadIdx.x == 0) s_tile = atomicAdd(ws.tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = static_cast<uint64_t>(tile) * S::kTile;
  const uint32_t t = threadIdx.x;
  const uint32_t lane = lane_id();
  const uint32_t warp = t / kWarp;

  T v[S::kRows][S::kPerVec];
  const bool full = base + S::kTile <= count;
  if (Vectorised && full) {
    const uint4 *src = reinterpret_cast<const uint4 *>(data + base);
#pragma unroll
    for (uint32_t r = 0; r < S::kRows; ++r) {
      const uint4 q = ld_stream_u4(src + r * S::kBlock + t);
      const T *qt = reinterpret_cast<const T *>(&q);
#pragma unroll
      for (uint32_t e = 0; e < S::kPerVec; ++e) v[r][e] = qt[e];
    }
  } else {
#pragma unroll
    for (uint32_t r = 0; r < S::kRows; ++r)
#pragma unroll
      for (uint32_t e = 0; e < S::kPerVec; ++e) {
        const uint64_t i =
            base + (static_cast<uint64_t>(r) * S::kBlock + t) * S::kPerVec + e;
        v[r][e] = i < count ? data[i] : T(0);
      }
  }

  // Row sums per thread, then a warp-inclusive scan of each row.
  T sum[S::kRows], incl[S::kRows];
#pragma unroll
  for (uint32_t r = 0; r < S::kRows; ++r) {
    T s = 0;
#pragma unroll
    for (uint32_t e = 0; e < S::kPerVec; ++e) s += v[r][e];
    sum[r] = s;
    incl[r] = warp_inclusive_sum<T>(s);
    if (lane == kWarp - 1) s_warp[warp][r] = incl[r];
  }
  __syncthreads();

  if (warp == 0) {
    T acc = 0;
#pragma unroll
    for (uint32_t r = 0; r < S::kRows; ++r) {
      const T w = lane < S::kWarps ? s_warp[lane][r] : T(0);
      const T wi = warp_inclusive_sum<T>(w);
      if (lane < S::kWarps) s_warp[lane][r] = wi - w; // exclusive warp offset
      if (lane == 0) s_row_off[r] = acc;
      acc += __shfl_sync(kFullMask, wi, S::kWarps - 1);
    }
    const T prefix = warp_lookback<T>(records, tile, acc, ws.status);
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();

  const T tile_prefix = s_prefix;
#pragma unroll
  for (uint32_t r = 0; r < S::kRows; ++r) {
    T run = tile_prefix + s_row_off[r] + s_warp[warp][r] + (incl[r] - sum[r]);
#pragma unroll
    for (uint32_t e = 0; e < S::kPerVec; ++e) {
      const T x = v[r][e];
      if (Inclusive) {
        run += x;
        v[r][e] = run;
      } else {
        v[r][e] = run;
        run += x;
      }
    }
  }

  if (Vectorised && full) {
    uint4 *dst = reinterpret_cast<uint4 *>(data + base);
#pragma unroll
    for (uint32_t r = 0; r < S::kRows; ++r)
      dst[r * S::kBlock + t] = *reinterpret_cast<const uint4 *>(v[r]);
  } else {
#pragma unroll
    for (uint32_t r = 0; r < S::kRows; ++r)
#pragma unroll
      for (uint32_t e = 0; e < S::kPerVec; ++e) {
        const uint64_t i =
            base + (static_cast<uint64_t>(r) * S::kBlock + t) * S::kPerVec + e;
        if (i < count) data[i] = v[r][e];
      }
  }
}

// Tiles for the element size that needs the most records (u64).
uint32_t max_tiles(uint32_t count) {
  return ceil_div(count, TileShape<uint64_t>::kTile) + 1;
}

} // namespace

size_t workspace_size(uint32_t count) {
  if (count == 0) return 0;
  const uint32_t tiles = max_tiles(count);
  Sizer s;
  s.take<uint32_t>(2);        // tile counter, status
  s.take<uint64_t>(tiles);    // packed records / u64 aggregates
  s.take<uint64_t>(tiles);    // u64 inclusive values
  s.take<uint32_t>(tiles);    // u64 record states
  return s.offset;
}

ScanLayout carve(void *workspace, uint32_t count, size_t elem_size) {
  const uint32_t tiles = max_tiles(count);
  Carver c(workspace);
  ScanLayout l;
  uint32_t *hdr = c.take<uint32_t>(2);
  l.tile_counter = hdr;
  l.status = hdr + 1;
  l.rec_a = c.take<uint64_t>(tiles);
  l.rec_b = c.take<uint64_t>(tiles);
  l.rec_state = c.take<uint32_t>(tiles);
  l.clear_bytes = elem_size == 4 ? (reinterpret_cast<char *>(l.rec_a + tiles) -
                                    reinterpret_cast<char *>(hdr))
                                 : c.offset;
  return l;
}

template <class T>
vx_status scan_launch(T *data, uint32_t count, bool inclusive, void *workspace,
                      size_t workspace_bytes, cudaStream_t stream) {
  if (data == nullptr && count != 0) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  if (workspace == nullptr || workspace_bytes < workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  using S = TileShape<T>;
  const ScanLayout ws = carve(workspace, count, sizeof(T));
  VX_TRY_CUDA(cudaMemsetAsync(workspace, 0, ws.clear_bytes, stream));
  const uint32_t tiles = ceil_div(count, S::kTile);
  const bool vec = (reinterpret_cast<uintptr_t>(data) & 15u) == 0;
  const auto records = make_records<T>(ws);
  prof::Scope scope(sizeof(T) == 4 ? "scan_u32" : "scan_u64", stream);
  if (inclusive) {
    if (vec)
      scan_kernel<T, true, true><<<tiles, S::kBlock, 0, stream>>>(data, count, ws, records);
    else
      scan_kernel<T, true, false><<<tiles, S::kBlock, 0, stream>>>(data, count, ws, records);
  } else {
    if (vec)
      scan_kernel<T, false, true><<<tiles, S::kBlock, 0, stream>>>(data, count, ws, records);
    else
      scan_kernel<T, false, false><<<tiles, S::kBlock, 0, stream>>>(data, count, ws, records);
  }
  return from_cuda(cudaGetLastError());
}

template vx_status scan_launch<uint32_t>(uint32_t *, uint32_t, bool, void *,
                                         size_t, cudaStream_t);
template vx_status scan_launch<uint64_t>(uint64_t *, uint32_t, bool, void *,
                                         size_t, cudaStream_t);

} // namespace scan
} // namespace vx

extern "C" {

size_t vx_scan_workspace_size(uint32_t count) {
  return vx::scan::workspace_size(count);
}

vx_status vx_scan_exclusive_sum_u32(uint32_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream) {
  return vx::scan::scan_launch<uint32_t>(data, count, false, workspace,
                                         workspace_bytes,
                                         static_cast<cudaStream_t>(stream));
}

vx_status vx_scan_inclusive_sum_u32(uint32_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream) {
  return vx::scan::scan_launch<uint32_t>(data, count, true, workspace,
                                         workspace_bytes,
                                         static_cast<cudaStream_t>(stream));
}

vx_status vx_scan_exclusive_sum_u64(uint64_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream) {
  return vx::scan::scan_launch<uint64_t>(data, count, false, workspace,
                                         workspace_bytes,
                                         static_cast<cudaStream_t>(stream));
}

} // extern "C"

// ------------------------------------------------- allocation-free variant --
//
// Some callers cannot allocate device memory at the point where they need a
// prefix sum: a frame loop or plugin that owns a fixed device-memory budget,
// or code that must not call cudaMalloc / cudaFree because those calls
// synchronise the device.  This entry point takes no workspace: its look-back
// scratch is one array in this library's own device memory, sized for at
// most kNoAllocMaxCount elements (256 KiB plus a 256-byte header, held on
// every GPU that loads the library until the process exits).

namespace vx::scan {
namespace {

constexpr uint32_t kNoAllocMaxCount = 1u << 28;
constexpr uint32_t kNoAllocTiles =
    (kNoAllocMaxCount + TileShape<uint32_t>::kTile - 1) / TileShape<uint32_t>::kTile;
constexpr size_t kNoAllocHeader = 256; // tile counter, status word

// [0, 256): tile counter and status; then one packed look-back record per tile.
static __device__ __align__(256) unsigned char
    g_noalloc_scratch[kNoAllocHeader + size_t(kNoAllocTiles) * sizeof(uint64_t)];

// Device address of g_noalloc_scratch per device (the symbol's name is only a
// host-side stand-in and must never be handed to a kernel).
void *noalloc_scratch(cudaError_t *err) {
  static std::mutex mu;
  static void *addr[64] = {};
  int dev = 0;
  *err = cudaGetDevice(&dev);
  if (*err != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void *p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (*err != cudaSuccess) return nullptr;
    addr[dev] = p;
  }
  return addr[dev];
}

} // namespace
} // namespace vx::scan

extern "C" {

// Allocation-free exclusive sum (see the block comment above): count must be
// at most 2^28; every call on a device shares one scratch array, so calls that
// may overlap on the GPU (different streams without ordering) race.  The
// first call on each device looks the scratch address up and should come
// before any stream capture.
vx_status vx_scan_exclusive_sum_u32_noalloc(uint32_t *data, uint32_t count,
                                            vx_stream stream) {
  using namespace vx::scan;
  if (data == nullptr && count != 0) return VX_ERR_INVALID_VALUE;
  if (count > kNoAllocMaxCount) return VX_ERR_CAPACITY;
  if (count == 0) return VX_OK;
  cudaError_t err = cudaSuccess;
  char *base = static_cast<char *>(noalloc_scratch(&err));
  if (base == nullptr) return vx::from_cuda(err);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  using S = TileShape<uint32_t>;
  const uint32_t tiles = vx::ceil_div(count, S::kTile);
  ScanLayout ws{};
  ws.tile_counter = reinterpret_cast<uint32_t *>(base);
  ws.status = ws.tile_counter + 1;
  ws.rec_a = reinterpret_cast<uint64_t *>(base + kNoAllocHeader);
  // The previous call's records are still there: clear the part this call uses.
  VX_TRY_CUDA(cudaMemsetAsync(base, 0, kNoAllocHeader + size_t(tiles) * sizeof(uint64_t), s));
  PackedRecords32 records{ws.rec_a};
  vx::prof::Scope scope("scan_u32_noalloc", s);
  if ((reinterpret_cast<uintptr_t>(data) & 15u) == 0)
    scan_kernel<uint32_t, false, true><<<tiles, S::kBlock, 0, s>>>(data, count, ws, records);
  else
    scan_kernel<uint32_t, false, false><<<tiles, S::kBlock, 0, s>>>(data, count, ws, records);
  return vx::from_cuda(cudaGetLastError());
}

} // extern "C"
