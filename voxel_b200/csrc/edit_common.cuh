// Shared pieces of the batched edit pipelines (Hash DAG and SVO).
//
// Both structures are edited by the same top-down, level-synchronous
// expansion.  A work item is one octree cell that at least one primitive
// touches but does not decide completely.  It carries the cell, the ref of the
// structure that was there before (or a uniform constant), and the ordered
// list of primitive indices that still matter inside it.  For each of its 8
// children the expansion finds the last primitive that covers the child
// entirely: every earlier primitive is overwritten there, so the child starts
// from that primitive's uniform value, and only later primitives that cut the
// child partially travel down.  Children that no primitive touches keep their
// old subtree (copy-on-write).  The result is exactly sequential application
// of the primitives in array order.
#pragma once

#include "common.cuh"

namespace vx::edit {

// Internal primitive shapes beyond the public sphere / box.
constexpr uint32_t kShapeLeafMask = 2; // c = leaf origin, r[0..1] = mask lo/hi
constexpr uint32_t kShapeTerrain = 3;  // c = {seed, scale, caves}

constexpr uint32_t kBlock = 256;

struct Cell {
  uint32_t x, y, z; // cell index at its level
};

__host__ __device__ __forceinline__ uint64_t pack_cell(uint32_t x, uint32_t y,
                                                       uint32_t z) {
  return static_cast<uint64_t>(x) | (static_cast<uint64_t>(y) << 21) |
         (static_cast<uint64_t>(z) << 42);
}
__host__ __device__ __forceinline__ Cell unpack_cell(uint64_t p) {
  return Cell{static_cast<uint32_t>(p & 0x1fffff),
              static_cast<uint32_t>((p >> 21) & 0x1fffff),
              static_cast<uint32_t>((p >> 42) & 0x1fffff)};
}
__host__ __device__ __forceinline__ uint64_t child_cell(uint64_t p, uint32_t c) {
  const Cell k = unpack_cell(p);
  return pack_cell(2 * k.x + (c & 1u), 2 * k.y + ((c >> 1) & 1u),
                   2 * k.z + ((c >> 2) & 1u));
}

// Classify primitive p against the voxel cube [o, o + n)^3.  Kernels that
// only ever see sphere / box / leaf-mask primitives instantiate Terrain =
// false and carry none of the terrain generator's code.
template <bool Terrain>
__device__ __forceinline__ uint32_t classify(const vx_primitive &p,
                                             uint32_t world_exp, int64_t ox,
                                             int64_t oy, int64_t oz, int64_t n) {
  const uint32_t shape = vx_prim_shape(&p);
  if (Terrain && shape == kShapeTerrain) {
    const vx_terrain t{static_cast<uint32_t>(p.c[0]), static_cast<uint32_t>(p.c[1]),
                       static_cast<uint32_t>(p.c[2]), world_exp};
    return vx_terrain_classify(&t, static_cast<uint32_t>(ox),
                               static_cast<uint32_t>(oy),
                               static_cast<uint32_t>(oz), static_cast<uint32_t>(n));
  }
  if (shape == kShapeLeafMask) {
    const int64_t lx = p.c[0], ly = p.c[1], lz = p.c[2];
    if (lx < ox || lx >= ox + n || ly < oy || ly >= oy + n || lz < oz ||
        lz >= oz + n)
      return VX_CELL_EMPTY;
    return VX_CELL_MIXED;
  }
  return vx_prim_classify(&p, ox, oy, oz, n);
}

// Voxels of the 4^3 leaf at o that the primitive covers.
template <bool Terrain>
__device__ __forceinline__ uint64_t leaf_mask(const vx_primitive &p,
                                              uint32_t world_exp, int64_t ox,
                                              int64_t oy, int64_t oz) {
  const uint32_t shape = vx_prim_shape(&p);
  if (Terrain && shape == kShapeTerrain) {
    const vx_terrain t{static_cast<uint32_t>(p.c[0]), static_cast<uint32_t>(p.c[1]),
                       static_cast<uint32_t>(p.c[2]), world_exp};
    return vx_terrain_leaf_mask(&t, static_cast<uint32_t>(ox),
                                static_cast<uint32_t>(oy), static_cast<uint32_t>(oz));
  }
  if (shape == kShapeLeafMask) {
    if (p.c[0] != ox || p.c[1] != oy || p.c[2] != oz) return 0;
    return static_cast<uint64_t>(p.r[0]) | (static_cast<uint64_t>(p.r[1]) << 32);
  }
  return vx_prim_leaf_mask(&p, ox, oy, oz);
}

// One work item of the top-down expansion (32 bytes).
struct Item {
  uint64_t cell;
  uint32_t old;        // ref (DAG) or slot word (SVO) of the previous content
  uint32_t pstart;     // first pair of this item in its level's pair array
  uint32_t pcount;     // number of pairs
  uint32_t child_base; // first child item at the next level
  uint32_t masks;      // child_mask | const_mask << 8 | const_full << 16
  uint32_t result;     // rebuilt ref / slot word
};
static_assert(sizeof(Item) == 32, "Item is 32 bytes");

// Per-edit device bookkeeping (one per structure).
struct Header {
  uint32_t root;
  uint32_t status;
  uint32_t prim_count;          // primitives of the current submission
  uint32_t pad0;
  uint32_t item_off[16];        // first item of each level
  uint32_t item_count[16];      // items of each level
  uint32_t pair_count[16];      // pairs of each level
  uint64_t node_count[16];      // items inserted per table (DAG)
  uint32_t pool_used[16];       // words used per level pool (DAG)
  uint32_t big_count[16];       // items deferred to the block-per-item path
};

struct Arena {
  Item *items;
  uint32_t *pairs[2];
  uint32_t *big;       // indices of items with long primitive lists
  uint32_t item_cap;
  uint32_t pair_cap;
  uint32_t big_cap;
};

// Items with more primitives than this are expanded by a whole block.
constexpr uint32_t kBigItem = 64;

} // namespace vx::edit
