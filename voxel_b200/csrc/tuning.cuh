// Launch-shape knobs read at launch time (process-wide; an autotuner sets
// them per device through vx_tuning_set).  Every allowed value is a correct
// configuration; the knobs only trade speed.
#pragma once

#include <cstdint>

namespace vx::tune {

enum Id : uint32_t {
  kSortItemsU32,    // partition items per thread, u32 keys: 12 or 16
  kSortItemsU64,    // partition items per thread, u64 keys: 8 or 10
  kSortEarlyCounts, // publish tile digit counts before ranking: 0 or 1
  kSortRankBallots, // rank keys with per-bit ballots (1) or shared-memory atomic OR (0)
  kEditBigItem,     // items with more primitives go to the block-per-item expansion
  kEditBlocksPerSm, // grid of the edit pipelines' item kernels, in blocks per SM
  kEditLeafparentBlocks, // resident blocks the DAG leaf-parent kernel is built for
  kServeBlocksPerSm, // grid of the serving loop's edit graphs, in blocks per SM
  kEditLeafparentLanes, // threads per item in the DAG leaf-parent kernel: 2, 4 or 8
  kEditSmallMaxPrims, // batches of at most this many primitives run as one cooperative kernel
  kEditSmallBlocksPerSm, // resident blocks per SM of that kernel
  kEditSmallMaxVoxels, // voxel lists / leaf commands of at most this length run that way
  kSortRadixBits,   // radix digit width in bits: 6, 7 or 8 (passes = key bits / width)
  kScanTileKb,      // prefix-sum tile in KB: 32 (256 threads), 16 (128) or 8 (64)
  kEditLeafparentPrefetch, // DAG leaf-parent kernel prefetches the next item's old node: 0 or 1
  kKnobCount
};

int64_t get(Id id);

} // namespace vx::tune
