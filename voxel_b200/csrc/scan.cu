// In-place prefix sums (uint32 / uint64, wrapping), one kernel launch after a
// small memset of the look-back records.  See scan.cuh for the design.
#include "profile.cuh"
#include "scan.cuh"
#include "tuning.cuh"

#include <cuda.h>

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

// One tile per block, tiles taken in the order of a global counter (a tile
// only waits on tiles already taken by running blocks).  A full, aligned tile
// arrives by one bulk copy; the last, partial tile and unaligned data use
// guarded loads.  Pass 1 reads the rows from shared memory for per-row warp
// totals, warp 0 scans the block and looks back, pass 2 re-reads the rows,
// recomputes each thread's offset inside its warp (cheaper than holding it in
// registers, which bound the resident blocks) and writes the prefix sums
// straight to global memory.
template <class T, bool Inclusive, bool Vectorised, class S = TileShape<T>>
__global__ void __launch_bounds__(S::kBlock, S::kMinBlocks)
    scan_kernel(T *__restrict__ data, uint32_t count, ScanLayout ws,
                typename RecordsFor<T>::type records) {
  constexpr uint32_t kTileBytes = S::kTile * sizeof(T);
  __shared__ __align__(128) T s_data[S::kTile];
  __shared__ uint64_t s_bar;
  __shared__ uint32_t s_tile;
  __shared__ T s_warp[S::kWarps][S::kRows];
  __shared__ T s_row_off[S::kRows];
  __shared__ T s_prefix;

  const uint32_t t = threadIdx.x;
  const uint32_t lane = lane_id();
  const uint32_t warp = t / kWarp;
  if (t == 0) {
    const uint32_t tile = atomicAdd(ws.tile_counter, 1u);
    s_tile = tile;
    if (Vectorised && static_cast<uint64_t>(tile + 1) * S::kTile <= count) {
      mbar_init(&s_bar, 1);
      mbar_arrive_expect_tx(&s_bar, kTileBytes);
      bulk_load(s_data, data + static_cast<uint64_t>(tile) * S::kTile, kTileBytes, &s_bar);
    }
  }
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = static_cast<uint64_t>(tile) * S::kTile;
  const bool bulk = Vectorised && base + S::kTile <= count;
  if (bulk) {
    if (!mbar_wait(&s_bar, 0)) {
      // Never expected: report, let the copy land, give up on this tile.
      if (t == 0) set_status(ws.status, kDevTimeout);
      mbar_wait(&s_bar, 0);
      return;
    }
  } else {
    for (uint32_t i = t; i < S::kTile; i += S::kBlock)
      s_data[i] = base + i < count ? data[base + i] : T(0);
    __syncthreads();
  }
  const uint4 *rows = reinterpret_cast<const uint4 *>(s_data);

  // Pass 1: per-row warp totals.
#pragma unroll 4
  for (uint32_t r = 0; r < S::kRows; ++r) {
    const uint4 q = rows[r * S::kBlock + t];
    const T *qt = reinterpret_cast<const T *>(&q);
    T sum = 0;
#pragma unroll
    for (uint32_t e = 0; e < S::kPerVec; ++e) sum += qt[e];
    sum = warp_sum<T>(sum);
    if (lane == 0) s_warp[warp][r] = sum;
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

  // Pass 2: prefix sums, written straight to global memory.
  const T tile_prefix = s_prefix;
#pragma unroll 4
  for (uint32_t r = 0; r < S::kRows; ++r) {
    uint4 q = rows[r * S::kBlock + t];
    T *qt = reinterpret_cast<T *>(&q);
    T sum = 0;
#pragma unroll
    for (uint32_t e = 0; e < S::kPerVec; ++e) sum += qt[e];
    T run = tile_prefix + s_row_off[r] + s_warp[warp][r] + (warp_inclusive_sum<T>(sum) - sum);
#pragma unroll
    for (uint32_t e = 0; e < S::kPerVec; ++e) {
      const T x = qt[e];
      if (Inclusive) {
        run += x;
        qt[e] = run;
      } else {
        qt[e] = run;
        run += x;
      }
    }
    if (bulk) {
      reinterpret_cast<uint4 *>(data + base)[r * S::kBlock + t] = q;
    } else {
      const uint64_t i0 = base + (static_cast<uint64_t>(r) * S::kBlock + t) * S::kPerVec;
#pragma unroll
      for (uint32_t e = 0; e < S::kPerVec; ++e)
        if (i0 + e < count) data[i0 + e] = qt[e];
    }
  }
}

// Tiles for the element size and tile shape that need the most records (u64
// in the smallest, 8 KB, tile).
uint32_t max_tiles(uint32_t count) {
  return ceil_div(count, TileShape<uint64_t, 64, 24>::kTile) + 1;
}

template <class T, bool Inclusive, bool Vectorised, class S>
void launch_shape(T *data, uint32_t count, const ScanLayout &ws,
                  const typename RecordsFor<T>::type &records, cudaStream_t stream) {
  const uint32_t tiles = ceil_div(count, S::kTile);
  scan_kernel<T, Inclusive, Vectorised, S><<<tiles, S::kBlock, 0, stream>>>(data, count, ws,
                                                                            records);
}

// Tile shape from the "scan.tile_kb" knob (32, 16 or 8 KB tiles).
template <class T, bool Inclusive, bool Vectorised>
void launch_tuned(T *data, uint32_t count, const ScanLayout &ws,
                  const typename RecordsFor<T>::type &records, cudaStream_t stream) {
  switch (tune::get(tune::kScanTileKb)) {
  case 8:
    launch_shape<T, Inclusive, Vectorised, TileShape<T, 64, 24>>(data, count, ws, records,
                                                                 stream);
    break;
  case 16:
    launch_shape<T, Inclusive, Vectorised, TileShape<T, 128, 12>>(data, count, ws, records,
                                                                  stream);
    break;
  default:
    launch_shape<T, Inclusive, Vectorised, TileShape<T>>(data, count, ws, records, stream);
  }
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
  const ScanLayout ws = carve(workspace, count, sizeof(T));
  VX_TRY_CUDA(cudaMemsetAsync(workspace, 0, ws.clear_bytes, stream));
  const bool vec = (reinterpret_cast<uintptr_t>(data) & 15u) == 0;
  const auto records = make_records<T>(ws);
  prof::Scope scope(sizeof(T) == 4 ? "scan_u32" : "scan_u64", stream);
  if (inclusive) {
    if (vec)
      launch_tuned<T, true, true>(data, count, ws, records, stream);
    else
      launch_tuned<T, true, false>(data, count, ws, records, stream);
  } else {
    if (vec)
      launch_tuned<T, false, true>(data, count, ws, records, stream);
    else
      launch_tuned<T, false, false>(data, count, ws, records, stream);
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

// Unique id of the calling thread's current CUDA context (0 when there is
// none or the driver entry points are unavailable).  Context ids are never
// reused within a process, so a context created again after a device reset
// gets a new id even when its handle value repeats.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (get_current == nullptr || get_id == nullptr) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_noalloc_scratch in the current context (the symbol's
// name is only a host-side stand-in and must never be handed to a kernel).
// The address is looked up with cudaGetSymbolAddress once per context and
// cached under the context's unique id, so a device reset (which unloads the
// module) is followed by a fresh lookup instead of a dangling address.  When
// the context id cannot be read, the address is looked up on every call.
void *noalloc_scratch(cudaError_t *err) {
  static std::mutex mu;
  static unsigned long long cached_ctx = 0;
  static void *cached_addr = nullptr;
  *err = cudaSuccess;
  unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(mu);
  if (ctx != 0 && ctx == cached_ctx && cached_addr != nullptr) return cached_addr;
  void *p = nullptr;
  *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (*err != cudaSuccess) return nullptr;
  if (ctx == 0) ctx = current_context_id(); // the lookup may have created the context
  cached_ctx = ctx;
  cached_addr = ctx != 0 ? p : nullptr;
  return p;
}

} // namespace
} // namespace vx::scan

extern "C" {

// Allocation-free exclusive sum (see the block comment above): count must be
// at most 2^28; every call on a device shares one scratch array, so calls that
// may overlap on the GPU (different streams without ordering) race.  The
// first call in each CUDA context looks the scratch address up and should
// come before any stream capture; vx_scan_noalloc_status reads the status
// word this call leaves behind.
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

// Status of the most recent allocation-free scan on the current device:
// synchronises the stream, then reads the device status word that the scan
// kernel leaves in the shared scratch (VX_ERR_TIMEOUT when a look-back wait
// gave up, in which case that call's prefix sums are not valid).  Every call
// of the allocation-free scan clears the word first, so this reports the last
// call that ran before the read; with calls that overlap on the GPU the word
// belongs to whichever wrote it last.
vx_status vx_scan_noalloc_status(vx_stream stream) {
  using namespace vx::scan;
  cudaError_t err = cudaSuccess;
  char *base = static_cast<char *>(noalloc_scratch(&err));
  if (base == nullptr) return vx::from_cuda(err);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t code = 0;
  VX_TRY_CUDA(cudaMemcpyAsync(&code, base + sizeof(uint32_t), sizeof(code),
                              cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  return vx::status_from_device(code);
}

} // extern "C"
