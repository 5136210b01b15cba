// A user's fused scans (voxel_b200_fused_scan.cuh), built by
// tests/test_gpu_fused_scan.py with nvcc and launched through the extern "C"
// functions below; every launcher takes a workspace of the size the
// matching *_ws function reports.
#include "voxel_b200_fused_scan.cuh"

namespace {

struct Compact {  // keep the multiples of 3, in order
  const uint32_t *x;
  uint32_t *out;
};
struct KeepFlag {
  __device__ static uint32_t run(uint32_t i, const Compact &in) { return in.x[i] % 3u == 0u; }
};
struct Scatter {
  __device__ static void run(uint32_t i, const Compact &in, uint32_t keep, uint32_t at) {
    if (keep) in.out[at] = in.x[i];
  }
};

struct Signed {
  const int32_t *x;
  int32_t *out;
};
struct Value {
  __device__ static int32_t run(uint32_t i, const Signed &in) { return in.x[i]; }
};
struct Store {
  __device__ static void run(uint32_t i, const Signed &in, int32_t, int32_t prefix) {
    in.out[i] = prefix;
  }
};

struct Words {
  const uint64_t *w;
  uint64_t *out;
};
struct Popc {
  __device__ static uint64_t run(uint32_t i, const Words &in) { return __popcll(in.w[i]); }
};
struct StoreU64 {
  __device__ static void run(uint32_t i, const Words &in, uint64_t, uint64_t prefix) {
    in.out[i] = prefix;
  }
};

struct Reals {
  const double *x;
  double *out;
};
struct Real {
  __device__ static double run(uint32_t i, const Reals &in) { return in.x[i]; }
};
struct StoreReal {
  __device__ static void run(uint32_t i, const Reals &in, double, double prefix) {
    in.out[i] = prefix;
  }
};

} // namespace

namespace scan = algo::cuda::scan;

extern "C" {
size_t compact_ws(uint32_t n) { return scan::required_workspace_size_fused<uint32_t>(n); }
int compact(const uint32_t *x, uint32_t *out, uint32_t n, void *ws, size_t ws_bytes) {
  int e = (int)scan::exclusive_sum_fused<KeepFlag, Scatter>(Compact{x, out}, n, ws, ws_bytes);
  return e ? e : (int)cudaDeviceSynchronize();
}
size_t max_ws(uint32_t n) { return scan::required_workspace_size_fused<scan::Max<int32_t>, int32_t>(n); }
int running_max(const int32_t *x, int32_t *out, uint32_t n, void *ws, size_t ws_bytes) {
  int e = (int)scan::inclusive_scan_fused<scan::Max<int32_t>, Value, Store>(Signed{x, out}, n, ws,
                                                                             ws_bytes);
  return e ? e : (int)cudaDeviceSynchronize();
}
size_t popc_ws(uint32_t n) { return scan::required_workspace_size_fused<uint64_t>(n); }
int popc_offsets(const uint64_t *w, uint64_t *out, uint32_t n, void *ws, size_t ws_bytes) {
  int e = (int)scan::exclusive_sum_fused<Popc, StoreU64>(Words{w, out}, n, ws, ws_bytes);
  return e ? e : (int)cudaDeviceSynchronize();
}
size_t real_ws(uint32_t n) { return scan::required_workspace_size_fused<double>(n); }
int real_sums(const double *x, double *out, uint32_t n, void *ws, size_t ws_bytes) {
  int e = (int)scan::inclusive_sum_fused<Real, StoreReal>(Reals{x, out}, n, ws, ws_bytes);
  return e ? e : (int)cudaDeviceSynchronize();
}
}
