// Single-pass prefix sum with decoupled look-back (Merrill & Garland 2016,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back"), written for
// sm_100a: 128-bit coalesced row loads, a dynamic tile id so that a tile only
// ever waits on tiles that are already resident, a warp-parallel look-back
// over 32 predecessors at a time, and a globaltimer bound on every wait.
//
// Replaces the reference's BlockBased<DecoupledLookback<WarpShuffleBlock<512,4>>>
// (cuda/scan/block_based/decoupled_lookback.cuh:116-221), whose look-back is a
// single thread with an unbounded spin (:99-102), and its fused variant
// (cuda/scan/fused.cuh:102-159), which assumes in-order block scheduling.
#pragma once

#include "common.cuh"

namespace vx::scan {

// Look-back record states.
constexpr uint32_t kNotReady = 0, kAggregate = 1, kInclusive = 2;

// u32 sums pack state and value into one 64-bit word, so one relaxed load
// observes both atomically.
struct PackedRecords32 {
  uint64_t *rec;
  __device__ void publish(uint32_t tile, uint32_t state, uint32_t value) const {
    st_relaxed_u64(rec + tile, (static_cast<uint64_t>(state) << 62) | value);
  }
  __device__ void read(int64_t tile, uint32_t &state, uint32_t &value) const {
    if (tile < 0) {
      state = kInclusive;
      value = 0;
      return;
    }
    const uint64_t r = ld_relaxed_u64(rec + tile);
    state = static_cast<uint32_t>(r >> 62);
    value = static_cast<uint32_t>(r);
  }
};

// u64 sums keep the value beside a state word: value first, then a release
// store of the state; readers acquire the state before reading the value.
struct SplitRecords64 {
  uint64_t *agg;
  uint64_t *inc;
  uint32_t *state;
  __device__ void publish(uint32_t tile, uint32_t s, uint64_t value) const {
    st_relaxed_u64((s == kInclusive ? inc : agg) + tile, value);
    st_release_u32(state + tile, s);
  }
  __device__ void read(int64_t tile, uint32_t &s, uint64_t &value) const {
    if (tile < 0) {
      s = kInclusive;
      value = 0;
      return;
    }
    s = ld_acquire_u32(state + tile);
    value = s == kInclusive ? ld_relaxed_u64(inc + tile)
                            : (s == kAggregate ? ld_relaxed_u64(agg + tile) : 0);
  }
};

template <class T> struct RecordsFor;
template <> struct RecordsFor<uint32_t> { using type = PackedRecords32; };
template <> struct RecordsFor<uint64_t> { using type = SplitRecords64; };

// Warp-parallel look-back, called by one full warp.  Publishes the tile's
// aggregate, accumulates predecessors 32 at a time until an inclusive record
// is found, publishes the inclusive prefix and returns the exclusive prefix
// (valid in every lane).  On timeout sets *status and returns a partial sum.
template <class T, class Records>
__device__ T warp_lookback(const Records &records, uint32_t tile, T aggregate,
                           uint32_t *status) {
  const uint32_t lane = lane_id();
  if (tile == 0) {
    if (lane == 0) records.publish(0, kInclusive, aggregate);
    return T(0);
  }
  if (lane == 0) records.publish(tile, kAggregate, aggregate);
  T exclusive = 0;
  int64_t pos = static_cast<int64_t>(tile) - 1;
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t s;
    T v;
    records.read(pos - static_cast<int64_t>(lane), s, v);
    const uint32_t inc_mask = __ballot_sync(kFullMask, s == kInclusive);
    const uint32_t wait_mask = __ballot_sync(kFullMask, s == kNotReady);
    const uint32_t limit = inc_mask ? (__ffs(inc_mask) - 1u) : 31u;
    const uint32_t range = limit == 31u ? kFullMask : ((1u << (limit + 1u)) - 1u);
    if (wait_mask & range) {
      if (global_ns() - t0 > kWaitLimitNs) {
        if (lane == 0) set_status(status, kDevTimeout);
        break;
      }
      __nanosleep(32);
      continue;
    }
    exclusive += warp_sum<T>(lane <= limit ? v : T(0));
    if (inc_mask) break;
    pos -= kWarp;
  }
  if (lane == 0) records.publish(tile, kInclusive, exclusive + aggregate);
  return exclusive;
}

// Block-wide scan tile geometry: kBlock threads, each owning kRows 16-byte
// vectors; row r of the tile is the contiguous range of kBlock vectors
// [r * kBlock, (r + 1) * kBlock), so every row load is fully coalesced.
template <class T> struct TileShape {
  static constexpr uint32_t kBlock = 512;
  static constexpr uint32_t kRows = 4;
  static constexpr uint32_t kPerVec = 16 / sizeof(T);
  static constexpr uint32_t kTile = kBlock * kRows * kPerVec;
  static constexpr uint32_t kWarps = kBlock / kWarp;
};

struct ScanLayout {
  uint32_t *tile_counter;
  uint32_t *status;
  uint64_t *rec_a;
  uint64_t *rec_b;
  uint32_t *rec_state;
  size_t clear_bytes; // bytes from the workspace start to clear per call
};

size_t workspace_size(uint32_t count);
ScanLayout carve(void *workspace, uint32_t count, size_t elem_size);

template <class T>
vx_status scan_launch(T *data, uint32_t count, bool inclusive, void *workspace,
                      size_t workspace_bytes, cudaStream_t stream);

} // namespace vx::scan
