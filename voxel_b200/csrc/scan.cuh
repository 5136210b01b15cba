// Single-pass prefix sum with decoupled look-back (Merrill & Garland 2016,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back"), written for
// sm_100a: each tile arrives in shared memory by one bulk copy (TMA), a
// dynamic tile id makes a tile only ever wait on tiles that are already
// resident, a warp-parallel look-back reads 64 predecessors per round trip,
// and a globaltimer bound limits every wait.
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
// aggregate, then reads the records of the previous 32 * R tiles at once
// (lane l, row j reads distance l + 32 j: R coalesced loads in flight per
// lane), accumulates back to the nearest inclusive record, publishes the
// inclusive prefix and returns the exclusive prefix (valid in every lane).
// A window wider than one warp matters because with hundreds of tiles
// resident the nearest inclusive record can be far back, and each window
// costs one round trip to L2.  On timeout sets *status and returns a partial
// sum.
template <class T, uint32_t R = 2, class Records>
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
    uint32_t st[R];
    T v[R];
#pragma unroll
    for (uint32_t j = 0; j < R; ++j)
      records.read(pos - static_cast<int64_t>(lane + kWarp * j), st[j], v[j]);
    // Nearest inclusive record: first row with one, first lane in it.
    int32_t first_row = -1;
    uint32_t limit = 31;
    bool wait = false;
#pragma unroll
    for (uint32_t j = 0; j < R; ++j) {
      const uint32_t inc = __ballot_sync(kFullMask, st[j] == kInclusive);
      const uint32_t nr = __ballot_sync(kFullMask, st[j] == kNotReady);
      if (first_row < 0) {
        const uint32_t lim = inc ? (__ffs(inc) - 1u) : 31u;
        const uint32_t range = lim == 31u ? kFullMask : ((1u << (lim + 1u)) - 1u);
        wait = wait || (nr & range) != 0;
        if (inc) {
          first_row = static_cast<int32_t>(j);
          limit = lim;
        }
      }
    }
    if (wait) {
      if (global_ns() - t0 > kWaitLimitNs) {
        if (lane == 0) set_status(status, kDevTimeout);
        break;
      }
      __nanosleep(32);
      continue;
    }
    T part = 0;
#pragma unroll
    for (uint32_t j = 0; j < R; ++j) {
      const bool in = first_row < 0 || static_cast<int32_t>(j) < first_row ||
                      (static_cast<int32_t>(j) == first_row && lane <= limit);
      part += in ? v[j] : T(0);
    }
    exclusive += warp_sum<T>(part);
    if (first_row >= 0) break;
    pos -= static_cast<int64_t>(kWarp * R);
  }
  if (lane == 0) records.publish(tile, kInclusive, exclusive + aggregate);
  return exclusive;
}

// Tile geometry: 256 threads x 8 rows of 16-byte vectors (a 32 KB tile);
// row r of the tile is the contiguous range of kBlock vectors [r * kBlock,
// (r + 1) * kBlock) and thread t owns vector t of every row.  The tile is
// staged in shared memory by one bulk copy and scanned from there in two
// passes, so a thread keeps only a few registers.  What bounds the bandwidth
// is the bytes in flight per SM while tiles wait for their loads and
// look-backs: registers would hold 128 KB of tiles per SM, shared memory
// holds six 32 KB tiles.  Without the look-back this pipeline streams at
// ~91 % of a device copy; the look-back chain (each tile waits for the
// aggregates of all tiles before it) costs the rest.  Measured alternatives
// on B200 (2^28 u32): 64 KB tiles x 3 per SM 0.63 ms, 128 KB x 1 0.72 ms,
// 32 KB x 4 0.82 ms, this shape 0.61 ms; 512 threads x 4 rows held in
// registers (2 per SM) 0.93 ms.
// The "scan.tile_kb" knob offers two smaller tiles of the same 8 rows with
// more of them resident (16 KB: 128 threads, 12 blocks / SM; 8 KB: 64
// threads, 24 blocks / SM): about as many bytes staged per SM, but a tile
// that waits for its predecessors' aggregates holds less of it.  On B200
// they are slower (2^28 u32, median of 10: 32 KB 0.578 ms, 16 KB 0.598 ms,
// 8 KB 0.672 ms; 2^27 u64: 0.755 / 0.815 / 0.924 ms): twice or four times
// the tiles means as many more look-backs, each a round trip to L2.
template <class T, uint32_t Block = 256, uint32_t MinBlocks = 6> struct TileShape {
  static constexpr uint32_t kBlock = Block;
  static constexpr uint32_t kRows = 8;
  static constexpr uint32_t kMinBlocks = MinBlocks;
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
