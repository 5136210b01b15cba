// Kernel launch counting and optional per-kernel CUDA-event timing inside
// the library.  Disabled by
// default (each guard is then one branch); when enabled with
// vx_profile_enable(1), every launch site wrapped in a ProfileScope records an
// event pair on the launching stream, and vx_profile_query() sums the elapsed
// times per kernel name.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vx::prof {

bool enabled();
void record(const char *name, cudaStream_t stream, bool start);
void count_launch();
uint64_t launch_count();
void add_launches(int64_t n); // graph replays add, captures take back

struct Scope {
  const char *name;
  cudaStream_t stream;
  bool on;
  Scope(const char *n, cudaStream_t s) : name(n), stream(s), on(enabled()) {
    count_launch();
    if (on) record(name, stream, true);
  }
  ~Scope() {
    if (on) record(name, stream, false);
  }
};

} // namespace vx::prof
