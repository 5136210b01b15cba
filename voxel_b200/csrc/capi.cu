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

#include <atomic>
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

void record(const char *name, cudaStream_t stream, bool start) {
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
