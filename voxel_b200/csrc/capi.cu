// Library-wide C ABI helpers: version, status names, workspace status.
#include "common.cuh"

extern "C" {

uint32_t vx_version(void) { return 0x000100u; }

const char *vx_status_string(vx_status status) {
  switch (status) {
  case VX_OK: return "ok";
  case VX_ERR_INVALID_VALUE: return "invalid value";
  case VX_ERR_MEMORY_ALLOCATION: return "memory allocation failed";
  case VX_ERR_TIMEOUT: return "a bounded device wait timed out";
  case VX_ERR_CAPACITY: return "capacity exceeded (node pool, table or arena full)";
  case VX_ERR_NO_DEVICE: return "no CUDA device";
  case VX_ERR_IO: return "file could not be read or written";
  default: return cudaGetErrorString(static_cast<cudaError_t>(status));
  }
}

// Scan and sort leave a device status word at byte offset 4 of their
// workspace (0 = ok, otherwise a device status code).  This reads it after
// synchronising the stream.
vx_status vx_workspace_status(const void *workspace, vx_stream stream) {
  if (workspace == nullptr) return VX_ERR_INVALID_VALUE;
  uint32_t code = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  VX_TRY_CUDA(cudaMemcpyAsync(&code, static_cast<const char *>(workspace) + 4,
                              sizeof(code), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  return vx::status_from_device(code);
}

} // extern "C"

// ------------------------------------------------------------ profiling --

#include "profile.cuh"
#include "tuning.cuh"

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace vx::prof {
namespace {

struct Pair {
  cudaEvent_t start, stop;
};

struct Registry {
  std::mutex mu;
  bool on = false;
  std::map<std::string, std::vector<Pair>> launches;
  std::map<std::string, cudaEvent_t> open;
};

Registry &reg() {
  static Registry r;
  return r;
}

} // namespace

bool enabled() { return reg().on; }

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void add_launches(int64_t n) {
  g_launches.fetch_add(static_cast<uint64_t>(n), std::memory_order_relaxed);
}

void record(const char *name, cudaStream_t stream, bool start) {
  // Inside a stream capture (a CUDA graph being built) nothing is timed.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return;
  Registry &r = reg();
  std::lock_guard<std::mutex> lock(r.mu);
  cudaEvent_t ev;
  if (cudaEventCreate(&ev) != cudaSuccess) return;
  cudaEventRecord(ev, stream);
  if (start) {
    r.open[name] = ev;
  } else {
    auto it = r.open.find(name);
    if (it == r.open.end()) {
      cudaEventDestroy(ev);
      return;
    }
    r.launches[name].push_back(Pair{it->second, ev});
    r.open.erase(it);
  }
}

} // namespace vx::prof

extern "C" {

void vx_profile_enable(uint32_t on) { vx::prof::reg().on = on != 0; }

// Kernels this library has launched in this process (every launch site
// counts, whether or not timing is enabled).
uint64_t vx_profile_launches(void) { return vx::prof::g_launches.load(); }

void vx_profile_reset(void) {
  auto &r = vx::prof::reg();
  std::lock_guard<std::mutex> lock(r.mu);
  for (auto &kv : r.launches)
    for (auto &p : kv.second) {
      cudaEventDestroy(p.start);
      cudaEventDestroy(p.stop);
    }
  r.launches.clear();
  for (auto &kv : r.open) cudaEventDestroy(kv.second);
  r.open.clear();
}

// Total milliseconds and launch count recorded for one kernel name since the
// last reset (synchronises on the recorded events).
vx_status vx_profile_query(const char *name, double *host_total_ms,
                           uint64_t *host_launches) {
  auto &r = vx::prof::reg();
  std::lock_guard<std::mutex> lock(r.mu);
  double total = 0.0;
  uint64_t n = 0;
  auto it = r.launches.find(name);
  if (it != r.launches.end()) {
    for (auto &p : it->second) {
      VX_TRY_CUDA(cudaEventSynchronize(p.stop));
      float ms = 0.f;
      VX_TRY_CUDA(cudaEventElapsedTime(&ms, p.start, p.stop));
      total += ms;
      ++n;
    }
  }
  if (host_total_ms) *host_total_ms = total;
  if (host_launches) *host_launches = n;
  return VX_OK;
}

} // extern "C"

extern "C" {

// Seeded primitive list for a benchmark configuration, written to host memory
// (the generator of vx_workload.h; no device work).
vx_status vx_generate_primitives(const vx_edit_mix *mix, uint64_t seed,
                                 uint64_t stream, uint64_t count,
                                 vx_primitive *host_out) {
  if (mix == nullptr || (host_out == nullptr && count != 0) || mix->world_exp < 3 ||
      mix->r_max < mix->r_min || mix->material_max < mix->material_min)
    return VX_ERR_INVALID_VALUE;
  vx_generate_primitives_host(mix, seed, stream, count, host_out);
  return VX_OK;
}

} // extern "C"

// ---------------------------------------------------------------- tuning --

namespace vx::tune {
namespace {
struct Knob {
  const char *name;
  int64_t def;
  int64_t allowed[6];
  uint32_t n_allowed;
};
// Defaults = the autotuner's choice on B200 (voxel_b200/tuning/NVIDIA_B200.json).
constexpr Knob kKnobs[kKnobCount] = {
    {"sort.items_u32", 16, {12, 16}, 2},
    {"sort.items_u64", 10, {8, 10}, 2},
    {"sort.early_counts", 0, {0, 1}, 2},
    {"sort.rank_ballots", 0, {0, 1}, 2},
    {"edit.big_item", 32, {16, 32, 64, 128, 256, 512}, 6},
    {"edit.blocks_per_sm", 32, {2, 4, 8, 16, 32}, 5},
    {"edit.leafparent_blocks", 5, {4, 5, 6}, 3},
    {"serve.blocks_per_sm", 4, {2, 4, 8, 16, 32}, 5},
    {"edit.leafparent_lanes", 4, {2, 4, 8}, 3},
    {"edit.small_max_prims", 256, {0, 64, 256, 1024, 4096}, 5},
    {"edit.small_blocks_per_sm", 1, {1, 2, 4}, 3},
    {"edit.small_max_voxels", 16384, {0, 4096, 16384, 65536}, 4},
    {"sort.radix_bits", 8, {6, 7, 8}, 3},
    {"scan.tile_kb", 32, {8, 16, 32}, 3},
    {"edit.leafparent_prefetch", 1, {0, 1}, 2},
};
std::atomic<int64_t> g_values[kKnobCount] = {{16}, {10}, {0}, {0}, {32}, {32}, {5}, {4}, {4},
                                             {256}, {1}, {16384}, {8}, {32}, {1}};

int find(const char *name) {
  if (name == nullptr) return -1;
  for (uint32_t i = 0; i < kKnobCount; ++i)
    if (std::strcmp(kKnobs[i].name, name) == 0) return static_cast<int>(i);
  return -1;
}
} // namespace

int64_t get(Id id) { return g_values[id].load(std::memory_order_relaxed); }

} // namespace vx::tune

extern "C" {

uint32_t vx_tuning_count(void) { return vx::tune::kKnobCount; }

const char *vx_tuning_name(uint32_t index) {
  return index < vx::tune::kKnobCount ? vx::tune::kKnobs[index].name : nullptr;
}

vx_status vx_tuning_options(const char *name, int64_t *host_values, uint32_t capacity,
                            uint32_t *host_count) {
  const int i = vx::tune::find(name);
  if (i < 0 || host_count == nullptr) return VX_ERR_INVALID_VALUE;
  const auto &k = vx::tune::kKnobs[i];
  *host_count = k.n_allowed;
  if (host_values != nullptr)
    for (uint32_t j = 0; j < k.n_allowed && j < capacity; ++j) host_values[j] = k.allowed[j];
  return VX_OK;
}

vx_status vx_tuning_get(const char *name, int64_t *host_value) {
  const int i = vx::tune::find(name);
  if (i < 0 || host_value == nullptr) return VX_ERR_INVALID_VALUE;
  *host_value = vx::tune::g_values[i].load();
  return VX_OK;
}

vx_status vx_tuning_set(const char *name, int64_t value) {
  const int i = vx::tune::find(name);
  if (i < 0) return VX_ERR_INVALID_VALUE;
  const auto &k = vx::tune::kKnobs[i];
  for (uint32_t j = 0; j < k.n_allowed; ++j)
    if (k.allowed[j] == value) {
      vx::tune::g_values[i].store(value);
      return VX_OK;
    }
  return VX_ERR_INVALID_VALUE;
}

vx_status vx_tuning_reset(void) {
  for (uint32_t i = 0; i < vx::tune::kKnobCount; ++i)
    vx::tune::g_values[i].store(vx::tune::kKnobs[i].def);
  return VX_OK;
}

} // extern "C"
