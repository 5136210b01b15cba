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
#include "voxel_b200_device.cuh"

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

// Exact sphere tests in 32-bit arithmetic for radii below 2^14: a distance
// that decides anything is at most r (+3 inside a leaf), so every square and
// every sum of three squares stays below 2^31.  Larger radii take the 64-bit
// definitions of vx_workload.h; both give identical results.
constexpr int64_t kFastRadius = int64_t(1) << 14;

// Cells lie in [0, 2^16] per axis (depth <= 14); a centre clamped to
// [-2^16, 2^18] keeps every outcome (a clamped centre is still more than
// 2^14 > r away from every cell), so the differences fit in 32 bits.
__device__ __forceinline__ uint32_t sphere_classify32(const vx_primitive &p, int64_t ox,
                                                      int64_t oy, int64_t oz, int64_t n) {
  const int32_t r = static_cast<int32_t>(p.r[0]);
  const int32_t lo[3] = {static_cast<int32_t>(ox), static_cast<int32_t>(oy),
                         static_cast<int32_t>(oz)};
  const int32_t n1 = static_cast<int32_t>(n) - 1;
  uint32_t near2 = 0, far2 = 0;
  bool far_in = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int32_t c = max(-(1 << 16), min(1 << 18, p.c[a]));
    const int32_t a0 = lo[a], a1 = lo[a] + n1;
    const int32_t d = c < a0 ? a0 - c : (c > a1 ? c - a1 : 0);
    if (d > r) return VX_CELL_EMPTY;
    near2 += static_cast<uint32_t>(d) * static_cast<uint32_t>(d);
    const int32_t f = max(abs(c - a0), abs(c - a1));
    if (f > r) far_in = false;
    else far2 += static_cast<uint32_t>(f) * static_cast<uint32_t>(f);
  }
  const uint32_t r2 = static_cast<uint32_t>(r) * static_cast<uint32_t>(r);
  if (near2 > r2) return VX_CELL_EMPTY;
  return (far_in && far2 <= r2) ? VX_CELL_FULL : VX_CELL_MIXED;
}

// Sphere mask of the leaf at o; the caller has classified the leaf MIXED, so
// every coordinate difference is within r + 3 of the centre.
__device__ __forceinline__ uint64_t sphere_leaf_mask32(const vx_primitive &p, int64_t ox,
                                                       int64_t oy, int64_t oz) {
  const int32_t r = static_cast<int32_t>(p.r[0]);
  const int32_t r2 = r * r;
  const int32_t dx0 = static_cast<int32_t>(ox - p.c[0]);
  const int32_t dy0 = static_cast<int32_t>(oy - p.c[1]);
  const int32_t dz0 = static_cast<int32_t>(oz - p.c[2]);
  int32_t dx2[4], dy2[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dx2[i] = (dx0 + i) * (dx0 + i);
    dy2[i] = (dy0 + i) * (dy0 + i);
  }
  uint64_t m = 0;
#pragma unroll
  for (int z = 0; z < 4; ++z) {
    const int32_t rz = r2 - (dz0 + z) * (dz0 + z);
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int32_t ry = rz - dy2[y];
      const uint32_t bits = (dx2[0] <= ry ? 1u : 0u) | (dx2[1] <= ry ? 2u : 0u) |
                            (dx2[2] <= ry ? 4u : 0u) | (dx2[3] <= ry ? 8u : 0u);
      m |= static_cast<uint64_t>(ry >= 0 ? bits : 0u) << (4 * y + 16 * z);
    }
  }
  return m;
}

// The same mask for radii up to kFloatMaskRadius, in single precision: the
// caller has classified the leaf MIXED, so every coordinate difference is at
// most r + 3 and every value below is an integer under 2^22 in magnitude,
// which each single-precision operation (contracted or not) keeps exact.  A
// voxel is inside when sx <= r^2 - sy - sz, i.e. when sx - (r^2 + 1 - sy -
// sz) is negative; an exact zero is +0, so the sign bit is the voxel's bit.
// The sign bits of a row's four voxels are gathered by byte permutes and one
// multiply (bits 7, 15, 23, 31 land in bits 28-31 with no carries into
// them), which moves most of the work off the integer pipe.
constexpr uint32_t kFloatMaskRadius = 1024;

__device__ __forceinline__ uint64_t sphere_leaf_mask_f32(const vx_primitive &p, int64_t ox,
                                                        int64_t oy, int64_t oz) {
  const float r = static_cast<float>(p.r[0]);
  const float fx = static_cast<float>(static_cast<int32_t>(ox - p.c[0]));
  const float fy = static_cast<float>(static_cast<int32_t>(oy - p.c[1]));
  const float fz = static_cast<float>(static_cast<int32_t>(oz - p.c[2]));
  float sx[4], sy[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float a = fx + static_cast<float>(i), b = fy + static_cast<float>(i);
    sx[i] = a * a;
    sy[i] = b * b;
  }
  const float r2p1 = r * r + 1.0f;
  uint32_t half[2] = {0u, 0u};
#pragma unroll
  for (int z = 0; z < 4; ++z) {
    const float c = fz + static_cast<float>(z);
    const float tz = r2p1 - c * c;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const float t = tz - sy[y];
      const uint32_t d01 = __byte_perm(__float_as_uint(sx[0] - t), __float_as_uint(sx[1] - t), 0x0073);
      const uint32_t d23 = __byte_perm(__float_as_uint(sx[2] - t), __float_as_uint(sx[3] - t), 0x0073);
      const uint32_t w = __byte_perm(d01, d23, 0x5410); // byte x = the top byte of voxel x's value
      const uint32_t row = ((w & 0x80808080u) * 0x00204081u) >> 28;
      half[z >> 1] |= row << (4 * y + 16 * (z & 1));
    }
  }
  return (static_cast<uint64_t>(half[1]) << 32) | half[0];
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
  if (shape == VX_SHAPE_SPHERE && p.r[0] < kFastRadius)
    return sphere_classify32(p, ox, oy, oz, n);
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
  if (shape == VX_SHAPE_SPHERE && p.r[0] <= kFloatMaskRadius)
    return sphere_leaf_mask_f32(p, ox, oy, oz);
  if (shape == VX_SHAPE_SPHERE && p.r[0] < kFastRadius)
    return sphere_leaf_mask32(p, ox, oy, oz);
  return vx_prim_leaf_mask(&p, ox, oy, oz);
}

// One work item of the top-down expansion (32 bytes).  Two fields change
// meaning over an edit: `pstart`, once the item is expanded, counts its child
// items that have not finished yet, and `result`, until the item is rebuilt,
// holds its parent's item index (kNoParent for the root), so that a
// bottom-up build can run without level barriers: the last child to finish
// rebuilds its parent.
struct Item {
  uint64_t cell;
  uint32_t old;        // ref (DAG) or slot word (SVO) of the previous content
  uint32_t pstart;     // first pair of this item in its level's pair array; then pending children
  uint32_t pcount;     // number of pairs
  uint32_t child_base; // first child item at the next level
  uint32_t masks;      // child_mask | const_mask << 8 | const_full << 16
  uint32_t result;     // parent index until rebuilt, then the rebuilt ref / slot word
};
constexpr uint32_t kNoParent = 0xffffffffu;

// Item reads on a climb (another SM wrote the item or its children's
// results in this launch): from L2, never from this SM's L1.
__device__ __forceinline__ Item load_item_l2(const Item *p) {
  const uint4 a = __ldcg(reinterpret_cast<const uint4 *>(p));
  const uint4 b = __ldcg(reinterpret_cast<const uint4 *>(p) + 1);
  Item it;
  it.cell = static_cast<uint64_t>(a.x) | (static_cast<uint64_t>(a.y) << 32);
  it.old = a.z;
  it.pstart = a.w;
  it.pcount = b.x;
  it.child_base = b.y;
  it.masks = b.z;
  it.result = b.w;
  return it;
}
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
  uint32_t pool_mark[16];       // pool_used before this edit's inserts (DAG)
};

struct Arena {
  Item *items;
  uint32_t *pairs[2];
  uint32_t *big;       // indices of items with long primitive lists
  uint32_t item_cap;
  uint32_t pair_cap;
  uint32_t big_cap;
};

// Items with more primitives than EditCtx::big_item (the tuning knob
// "edit.big_item", 32 by default) are expanded by a whole block.  They are
// listed when they are emitted (the level above's expansion, or the init of
// the root), so that a level's short and long lists can be expanded side by
// side; the big buffer's two halves alternate by level, so level l + 1's
// list fills while level l's is read.
__device__ __forceinline__ uint32_t *big_list(const Arena &a, uint32_t l) {
  return a.big + (l & 1u) * (a.big_cap / 2u);
}


// init_kernel's root_old value meaning "the root stored in the header".
constexpr uint32_t kUseHeaderRoot = 0xfffffffeu;

// Device-side edit context shared by the DAG and SVO pipelines.
struct EditCtx {
  Header *hdr;
  Arena a;
  const vx_primitive *prims;
  const uint32_t *d_prim_count; // device count (NULL: use host_prim_count)
  uint32_t host_prim_count;
  uint32_t depth;
  uint32_t big_item; // longer primitive lists go to expand_big_kernel
};

// List item `idx` of level l (its index within the level) for the
// block-per-item expansion when its primitive list is long and level l is
// expanded at all (levels below depth - 1).
__device__ __forceinline__ void note_big(const EditCtx &x, uint32_t l, uint32_t idx,
                                         uint32_t pcount) {
  if (pcount <= x.big_item || l + 1 >= x.depth) return;
  const uint32_t slot = atomicAdd(&x.hdr->big_count[l], 1u);
  if (slot < x.a.big_cap / 2u) big_list(x.a, l)[slot] = idx;
  else set_status(&x.hdr->status, kDevCapacity);
}

// A tree Policy supplies:
//   static constexpr bool kItemsForConst  - also create a (primitive-free)
//       child item where a primitive covers the child entirely, so the
//       rebuild sees its constant value in the child item's `old`;
//   child(l, old, c)                      - content of child c of `old` at level l;
//   classify<Terrain>(prim, world_exp, ox, oy, oz, n);
//   const_value(prim, oz, n)              - the content a fully covering
//       primitive leaves in the cube at height oz of side n (1 = full);
//   replaced(l, old, c)                   - child c of `old` is overwritten
//       by a fully covering primitive (its subtree is dropped).

// The blocks a pipeline stage runs on: its own launch (blockIdx / gridDim), or
// the whole grid of the single cooperative kernel that runs every stage of a
// small edit in a row.
struct Blocks {
  uint32_t id, count;
};
__device__ __forceinline__ Blocks launch_blocks() { return Blocks{blockIdx.x, gridDim.x}; }

// True on every thread of the block when the edit's status is no longer ok.
// Block-uniform, so a stage that returns on it never leaves part of a block
// at a barrier.
__device__ __forceinline__ bool edit_failed(const Header *h) {
  return __syncthreads_or(ld_relaxed_u32(&h->status) != kDevOk) != 0;
}

__device__ __forceinline__ void init_body(EditCtx x, uint32_t root_old, Blocks blk) {
  Header *h = x.hdr;
  // With a device-side count, host_prim_count is the capacity of the list.
  const uint32_t dn = x.d_prim_count ? *x.d_prim_count : 0u;
  if (x.d_prim_count && dn > x.host_prim_count) {
    if (blk.id == 0 && threadIdx.x == 0) set_status(&h->status, kDevInvalid);
    return;
  }
  const uint32_t n = x.d_prim_count ? dn : x.host_prim_count;
  if (blk.id == 0 && threadIdx.x == 0) {
    for (uint32_t l = 0; l < 16; ++l) {
      h->item_off[l] = 0;
      h->item_count[l] = 0;
      h->pair_count[l] = 0;
      h->big_count[l] = 0;
    }
    h->prim_count = n;
    const uint32_t ok = h->status == kDevOk && n <= x.a.pair_cap;
    if (h->status == kDevOk && n > x.a.pair_cap) h->status = kDevCapacity;
    if (ok) {
      h->item_count[0] = 1;
      h->pair_count[0] = n;
      Item it{};
      it.cell = 0;
      it.old = root_old == kUseHeaderRoot ? h->root : root_old;
      it.pstart = 0;
      it.pcount = n;
      it.result = kNoParent;
      x.a.items[0] = it;
      note_big(x, 0, 0, n);
    }
  }
  if (n > x.a.pair_cap) return;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < n; i += static_cast<uint64_t>(blk.count) * blockDim.x)
    x.a.pairs[0][i] = static_cast<uint32_t>(i);
}

static __global__ void init_kernel(EditCtx x, uint32_t root_old) {
  init_body(x, root_old, launch_blocks());
}

// ------------------------------------------- plain voxel lists, small edits --
//
// Inside the single cooperative kernel of a small edit, a voxel list (one op
// for every voxel) becomes its leaf-mask primitives without a sort: voxels
// are aggregated into a hash table of {leaf key + 1, mask} slots (atomicCAS
// claims a slot and lists it, atomicOr sets the voxel's bit), then primitive
// i is written from the i-th listed slot.  One op for all voxels makes the
// order of the primitives irrelevant.  Stages: clear, aggregate, fill (the
// last beside the edit's init, which only needs the count), each followed by
// a grid-wide barrier.
struct PlainPrep {
  const vx_voxel *edits;
  uint32_t count;       // voxels
  uint32_t op, material;
  ulonglong2 *slots;    // {packed leaf coordinates + 1 (0 = free), mask}
  uint32_t nslots;
  uint32_t *order;      // used slots in the order they were claimed
  vx_primitive *prims;  // out: one leaf-mask primitive per touched leaf
  uint32_t *nprims;     // out: their number (the edit's device-side count)
};

// The prep's table and primitive list carved from a plain-path workspace;
// false when they do not fit it.
inline bool plain_prep_layout(void *ws, size_t ws_bytes, const vx_voxel *edits, uint32_t count,
                              uint32_t op, uint32_t material, PlainPrep *out) {
  Carver c(ws);
  PlainPrep p{};
  p.edits = edits;
  p.count = count;
  p.op = op;
  p.material = material;
  p.nslots = count + count / 2u + 1u; // distinct leaves <= count: load <= 2/3
  p.slots = c.take<ulonglong2>(p.nslots);
  p.order = c.take<uint32_t>(count);
  p.prims = c.take<vx_primitive>(count);
  p.nprims = c.take<uint32_t>(1);
  if (c.offset > ws_bytes) return false;
  *out = p;
  return true;
}

__device__ __forceinline__ void plain_prep_clear(const PlainPrep &p, Blocks blk) {
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < p.nslots;
       i += static_cast<uint64_t>(blk.count) * blockDim.x)
    p.slots[i] = make_ulonglong2(0ull, 0ull);
  if (blk.id == 0 && threadIdx.x == 0) *p.nprims = 0;
}

__device__ __forceinline__ void plain_prep_aggregate(const PlainPrep &p, uint32_t depth,
                                                     Blocks blk) {
  const uint32_t side_exp = depth + 2;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < p.count;
       i += static_cast<uint64_t>(blk.count) * blockDim.x) {
    const vx_voxel v = p.edits[i];
    if ((v.x >> side_exp) | (v.y >> side_exp) | (v.z >> side_exp)) continue; // outside: ignored
    const uint64_t key = (static_cast<uint64_t>(v.x >> 2) | (static_cast<uint64_t>(v.y >> 2) << 21) |
                          (static_cast<uint64_t>(v.z >> 2) << 42)) + 1ull;
    const uint64_t bit = 1ull << ((v.x & 3u) + 4u * (v.y & 3u) + 16u * (v.z & 3u));
    uint32_t pos = vx_reduce_hash(vx_mix64(key), p.nslots);
    for (uint32_t probe = 0; probe < p.nslots; ++probe) {
      const unsigned long long old =
          atomicCAS(reinterpret_cast<unsigned long long *>(&p.slots[pos].x), 0ull, key);
      if (old == 0ull || old == key) {
        if (old == 0ull) p.order[atomicAdd(p.nprims, 1u)] = pos; // distinct leaves <= count
        atomicOr(reinterpret_cast<unsigned long long *>(&p.slots[pos].y), bit);
        break;
      }
      pos = pos + 1u == p.nslots ? 0u : pos + 1u;
    }
  }
}

__device__ __forceinline__ void plain_prep_fill(const PlainPrep &p, Blocks blk) {
  const uint32_t n = *p.nprims;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(blk.count) * blockDim.x) {
    const ulonglong2 e = p.slots[p.order[i]];
    const uint64_t k = e.x - 1ull;
    vx_primitive pr{};
    pr.c[0] = static_cast<int32_t>((k & 0x1fffffull) * 4u);
    pr.c[1] = static_cast<int32_t>(((k >> 21) & 0x1fffffull) * 4u);
    pr.c[2] = static_cast<int32_t>(((k >> 42) & 0x1fffffull) * 4u);
    pr.r[0] = static_cast<uint32_t>(e.y);
    pr.r[1] = static_cast<uint32_t>(e.y >> 32);
    pr.flags = vx_make_flags(kShapeLeafMask, p.op, p.material);
    p.prims[i] = pr;
  }
}

// Top-down expansion of level l into level l + 1 (l + 1 < depth).  Eight
// lanes per work item, one per child cell: lane c walks the item's ordered
// primitive list once, remembering the last primitive that covers child c
// entirely (which resets the count of partial ones before it) and counting the
// partial ones after it; a second walk writes those to the child's list.
// Output space for a block's 32 items is taken with one atomicAdd per counter.
template <class Policy, bool Terrain>
__device__ __forceinline__ void expand_body(EditCtx x, Policy pol, uint32_t l, Blocks blk) {
  Header *h = x.hdr;
  // the level's counts load beside the status (one round trip, not two)
  const uint32_t W = h->item_count[l];
  const uint32_t base = h->item_off[l];
  if (edit_failed(h)) return;
  const uint32_t depth = x.depth;
  const uint32_t next_base = base + W;
  if (blk.id == 0 && threadIdx.x == 0) h->item_off[l + 1] = next_base;
  const uint32_t *in_pairs = x.a.pairs[l & 1u];
  uint32_t *out_pairs = x.a.pairs[(l + 1) & 1u];
  const int64_t csize = int64_t(4) << (depth - l - 1); // child cell size
  const uint32_t world_exp = depth + 2;
  constexpr uint32_t kGroups = kBlock / 8;
  static_assert(kGroups == kWarp, "one warp scans the groups' counts");

  __shared__ uint32_t s_items[kGroups], s_pairs[kGroups];
  __shared__ uint32_t s_item_base, s_pair_base;
  __shared__ bool s_room;
  // the group's current chunk of its item's list: pair values and primitives
  __shared__ uint32_t s_pidx[kGroups][8];
  __shared__ vx_primitive s_prim[kGroups][8];
  const uint32_t group = threadIdx.x >> 3, c = threadIdx.x & 7u;
  const uint32_t gshift = (lane_id() >> 3) * 8u; // this group's byte in a ballot
  const uint32_t gmask = 0xffu << gshift;        // this group's lanes

  for (uint64_t tile = blk.id; tile * kGroups < W; tile += blk.count) {
    const uint32_t wi = static_cast<uint32_t>(tile * kGroups) + group;
    const bool have = wi < W;
    Item it{};
    if (have) it = x.a.items[base + wi];
    // Long lists were listed for expand_big (one block per item) when the
    // item was emitted.
    const bool big = have && it.pcount > x.big_item;
    if (big) it.pcount = 0;
    const Cell cell = unpack_cell(it.cell);
    const int64_t ox = int64_t(2 * cell.x + (c & 1u)) * csize;
    const int64_t oy = int64_t(2 * cell.y + ((c >> 1) & 1u)) * csize;
    const int64_t oz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * csize;
    // The child's previous content, read before the list walk so that the
    // two chains of loads overlap (unused when a primitive covers the child).
    const uint32_t old_child = have && !big ? pol.child(l, it.old, c) : 0u;
    int32_t last_full = -1;
    uint32_t cnt = 0;
    // Bit k: the list's k-th primitive cuts this child partially and comes
    // after every primitive that covers it (kept for lists of up to 32).
    uint32_t partial = 0;
    // Eight primitives at a time: each lane of the group loads one pair and
    // its primitive (two rounds of independent loads per chunk instead of two
    // dependent loads per primitive), then every lane walks the chunk for its
    // own child.  pcount is the same on the group's lanes, so they pass the
    // group barriers together.
    // (A terrain build's items hold its one primitive: walked in place.)
    for (uint32_t k = 0; Terrain && k < it.pcount; ++k) {
      const uint32_t p = in_pairs[it.pstart + k];
      const uint32_t cls = pol.template classify<Terrain>(x.prims[p], world_exp, ox, oy, oz, csize);
      if (cls == VX_CELL_FULL) {
        last_full = static_cast<int32_t>(p);
        cnt = 0;
        partial = 0;
      } else if (cls == VX_CELL_MIXED) {
        ++cnt;
        if (k < 32u) partial |= 1u << k;
      }
    }
    for (uint32_t k0 = 0; !Terrain && k0 < it.pcount; k0 += 8) {
      if (k0 + c < it.pcount) {
        const uint32_t p = in_pairs[it.pstart + k0 + c];
        s_pidx[group][c] = p;
        s_prim[group][c] = x.prims[p];
      }
      __syncwarp(gmask);
      const uint32_t m = min(8u, it.pcount - k0);
      for (uint32_t j = 0; j < m; ++j) {
        const uint32_t k = k0 + j;
        const uint32_t cls =
            pol.template classify<Terrain>(s_prim[group][j], world_exp, ox, oy, oz, csize);
        if (cls == VX_CELL_FULL) {
          last_full = static_cast<int32_t>(s_pidx[group][j]);
          cnt = 0;
          partial = 0;
        } else if (cls == VX_CELL_MIXED) {
          ++cnt;
          if (k < 32u) partial |= 1u << k;
        }
      }
      __syncwarp(gmask); // the chunk is overwritten next
    }
    // Prefix sums over the 8 lanes of the group.
    uint32_t inc_items =
                 (cnt != 0 || (Policy::kItemsForConst && last_full >= 0)) ? 1u : 0u,
             inc_pairs = cnt;
#pragma unroll
    for (uint32_t d = 1; d < 8; d <<= 1) {
      const uint32_t a = __shfl_up_sync(kFullMask, inc_items, d, 8);
      const uint32_t b = __shfl_up_sync(kFullMask, inc_pairs, d, 8);
      if (c >= d) {
        inc_items += a;
        inc_pairs += b;
      }
    }
    const uint32_t group_items = __shfl_sync(kFullMask, inc_items, 7, 8);
    const uint32_t group_pairs = __shfl_sync(kFullMask, inc_pairs, 7, 8);
    const uint32_t const_val =
        last_full >= 0 ? pol.const_value(x.prims[last_full], oz, csize) : 0u;
    const bool full_add = last_full >= 0 && const_val == 1u;
    const bool has_item = cnt != 0 || (Policy::kItemsForConst && last_full >= 0);
    const uint32_t child_mask = (__ballot_sync(kFullMask, has_item) >> gshift) & 0xffu;
    const uint32_t const_mask = (__ballot_sync(kFullMask, last_full >= 0) >> gshift) & 0xffu;
    const uint32_t const_full = (__ballot_sync(kFullMask, full_add) >> gshift) & 0xffu;
    if (c == 0) {
      s_items[group] = have && !big ? group_items : 0u;
      s_pairs[group] = have && !big ? group_pairs : 0u;
    }
    __syncthreads();
    if (threadIdx.x < kWarp) { // one group per lane: exclusive offsets by shuffles
      const uint32_t a = s_items[threadIdx.x], b = s_pairs[threadIdx.x];
      const uint32_t ia = warp_inclusive_sum(a), ib = warp_inclusive_sum(b);
      s_items[threadIdx.x] = ia - a;
      s_pairs[threadIdx.x] = ib - b;
      const uint32_t ti = __shfl_sync(kFullMask, ia, kWarp - 1);
      const uint32_t tp = __shfl_sync(kFullMask, ib, kWarp - 1);
      if (threadIdx.x == 0) {
        s_item_base = ti ? atomicAdd(&h->item_count[l + 1], ti) : 0;
        s_pair_base = tp ? atomicAdd(&h->pair_count[l + 1], tp) : 0;
        // this tile's own room (an overflow elsewhere fails the edit at the
        // next stage; writing within the buffers meanwhile is harmless)
        bool room = true;
        if (ti && static_cast<uint64_t>(next_base) + s_item_base + ti > x.a.item_cap) room = false;
        if (tp && static_cast<uint64_t>(s_pair_base) + tp > x.a.pair_cap) room = false;
        if (!room) set_status(&h->status, kDevCapacity);
        s_room = room;
      }
    }
    __syncthreads();
    const bool room = s_room;
    const uint32_t item_off = s_item_base + s_items[group];
    const uint32_t pair_off = s_pair_base + s_pairs[group];
    __syncthreads(); // s_* are reused by the next tile
    if (!have || big || !room) continue;
    if (last_full >= 0) pol.replaced(l, it.old, c);

    if (has_item) {
      const uint32_t my_pairs = pair_off + inc_pairs - cnt;
      Item ci{};
      ci.cell = child_cell(it.cell, c);
      ci.old = last_full >= 0 ? const_val : old_child;
      ci.pstart = my_pairs;
      ci.pcount = cnt;
      ci.result = static_cast<uint32_t>(base + wi);
      x.a.items[next_base + item_off + inc_items - 1] = ci;
      note_big(x, l + 1, item_off + inc_items - 1, cnt);
      uint32_t j = 0;
      if (it.pcount <= 32u) {
        // The child's list is the set bits of `partial`: independent loads
        // of the pairs, no second classification.
        for (uint32_t bits = partial; bits != 0u; bits &= bits - 1u)
          out_pairs[my_pairs + j++] = in_pairs[it.pstart + __ffs(bits) - 1u];
      } else {
        for (uint32_t k = 0; k < it.pcount && j < cnt; ++k) {
          const uint32_t p = in_pairs[it.pstart + k];
          if (static_cast<int32_t>(p) <= last_full) continue;
          if (pol.template classify<Terrain>(x.prims[p], world_exp, ox, oy, oz, csize) == VX_CELL_MIXED)
            out_pairs[my_pairs + j++] = p;
        }
      }
    }
    if (c == 0) {
      x.a.items[base + wi].child_base = next_base + item_off;
      x.a.items[base + wi].masks = child_mask | (const_mask << 8) | (const_full << 16);
      x.a.items[base + wi].pstart = __popc(child_mask); // the pairs were read above
    }
  }
}

template <class Policy, bool Terrain>
__global__ void __launch_bounds__(kBlock)
    expand_kernel(EditCtx x, Policy pol, uint32_t l) {
  expand_body<Policy, Terrain>(x, pol, l, launch_blocks());
}

// Expansion of the long-list items of level l: one block of Threads
// threads per item.  Three walks over the list: the last fully-covering
// primitive per child (block max), the partial primitives after it per child
// (block sum), then an order-preserving block-wide compaction of those into
// each child's list.  The root of a batch carries every primitive and is
// expanded by one block alone, so edits use a wide block (kBigBlock); the
// terrain generator's classification needs more registers than a wide
// block leaves a thread, so terrain builds use kBlock.  Lists of up to
// kBigCache primitives are classified once: walk 1 keeps each primitive's
// per-child MIXED bits in shared memory for walks 2 and 3.
constexpr uint32_t kBigBlock = 512;
constexpr uint32_t kBigCache = 32768;

template <class Policy, bool Terrain, uint32_t Threads, uint32_t Cache>
__device__ __forceinline__ void expand_big_body(EditCtx x, Policy pol, uint32_t l, Blocks blk) {
  Header *h = x.hdr;
  // the level's counts and this block's first listed item load beside the
  // status (the list is read past its count only within its buffer)
  const uint32_t nbig = min(h->big_count[l], x.a.big_cap / 2u);
  const uint32_t *bigs = big_list(x.a, l);
  const uint32_t base = h->item_off[l];
  const uint32_t next_base = base + h->item_count[l];
  uint32_t first_wi = blk.id < x.a.big_cap / 2u ? bigs[blk.id] : 0u;
  if (edit_failed(h)) return;
  const uint32_t depth = x.depth;
  const uint32_t *in_pairs = x.a.pairs[l & 1u];
  uint32_t *out_pairs = x.a.pairs[(l + 1) & 1u];
  const int64_t csize = int64_t(4) << (depth - l - 1);
  const uint32_t world_exp = depth + 2;
  constexpr uint32_t kWarps = Threads / kWarp;
  static_assert(kWarps <= kWarp, "one warp scans the warps' counts");
  __shared__ int32_t s_last[8];
  __shared__ uint32_t s_cnt[8], s_start[8], s_const[8], s_cm;
  __shared__ uint32_t s_warp[8][kWarps], s_total[8];
  __shared__ uint32_t s_item_base, s_pair_base;
  __shared__ bool s_room;
  __shared__ uint8_t s_mixed[Cache];
  const uint32_t t = threadIdx.x, lane = lane_id(), warp = t / kWarp;

  for (uint32_t b = blk.id; b < nbig; b += blk.count) {
    const uint32_t wi = b == blk.id ? first_wi : bigs[b];
    const Item it = x.a.items[base + wi];
    const Cell cell = unpack_cell(it.cell);
    const bool cached = it.pcount <= Cache; // block-uniform
    // child t's previous content, loaded beside the walks (used unless a
    // primitive covers the child)
    const uint32_t old_child = t < 8 ? pol.child(l, it.old, t) : 0u;
    if (t < 8) {
      s_last[t] = -1;
      s_cnt[t] = 0;
    }
    __syncthreads();
    // Walk 1: last FULL per child (and the MIXED bits, when cached).
    int32_t last[8];
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) last[c] = -1;
    for (uint32_t k = t; k < it.pcount; k += Threads) {
      const uint32_t p = in_pairs[it.pstart + k];
      const vx_primitive pr = x.prims[p];
      uint32_t mixed = 0;
#pragma unroll
      for (uint32_t c = 0; c < 8; ++c) {
        const int64_t ox = int64_t(2 * cell.x + (c & 1u)) * csize;
        const int64_t oy = int64_t(2 * cell.y + ((c >> 1) & 1u)) * csize;
        const int64_t oz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * csize;
        const uint32_t cls = pol.template classify<Terrain>(pr, world_exp, ox, oy, oz, csize);
        if (cls == VX_CELL_FULL) last[c] = max(last[c], static_cast<int32_t>(p));
        else if (cls == VX_CELL_MIXED) mixed |= 1u << c;
      }
      if (cached) s_mixed[k] = static_cast<uint8_t>(mixed);
    }
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) {
      const int32_t m = __reduce_max_sync(kFullMask, last[c]);
      if (lane == 0 && m >= 0) atomicMax(&s_last[c], m);
    }
    __syncthreads();
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) last[c] = s_last[c];
    // Walk 2: partial primitives after the last full one.
    uint32_t cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t k = t; k < it.pcount; k += Threads) {
      const uint32_t p = in_pairs[it.pstart + k];
      if (cached) { // each thread reads back the bits it wrote in walk 1
        const uint32_t mixed = s_mixed[k];
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c)
          cnt[c] += (static_cast<int32_t>(p) > last[c] && ((mixed >> c) & 1u)) ? 1u : 0u;
        continue;
      }
      const vx_primitive pr = x.prims[p];
#pragma unroll
      for (uint32_t c = 0; c < 8; ++c) {
        if (static_cast<int32_t>(p) <= last[c]) continue;
        const int64_t ox = int64_t(2 * cell.x + (c & 1u)) * csize;
        const int64_t oy = int64_t(2 * cell.y + ((c >> 1) & 1u)) * csize;
        const int64_t oz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * csize;
        if (pol.template classify<Terrain>(pr, world_exp, ox, oy, oz, csize) == VX_CELL_MIXED) ++cnt[c];
      }
    }
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) {
      const uint32_t v = __reduce_add_sync(kFullMask, cnt[c]);
      if (lane == 0 && v) atomicAdd(&s_cnt[c], v);
    }
    __syncthreads();
    if (t == 0) {
      uint32_t ni = 0, np = 0, cm = 0, km = 0, kf = 0;
      for (uint32_t c = 0; c < 8; ++c) {
        s_start[c] = np;
        const int64_t coz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * csize;
        s_const[c] = s_last[c] >= 0 ? pol.const_value(x.prims[s_last[c]], coz, csize) : 0u;
        if (s_cnt[c] || (Policy::kItemsForConst && s_last[c] >= 0)) {
          cm |= 1u << c;
          ++ni;
          np += s_cnt[c];
        }
        if (s_last[c] >= 0) {
          km |= 1u << c;
          if (s_const[c] == 1u) kf |= 1u << c;
        }
      }
      s_cm = cm;
      s_item_base = ni ? atomicAdd(&h->item_count[l + 1], ni) : 0;
      s_pair_base = np ? atomicAdd(&h->pair_count[l + 1], np) : 0;
      // this item's own room (an overflow elsewhere fails the edit at the
      // next stage; writing within the buffers meanwhile is harmless)
      bool room = true;
      if (ni && static_cast<uint64_t>(next_base) + s_item_base + ni > x.a.item_cap) room = false;
      if (np && static_cast<uint64_t>(s_pair_base) + np > x.a.pair_cap) room = false;
      if (!room) set_status(&h->status, kDevCapacity);
      x.a.items[base + wi].child_base = next_base + s_item_base;
      x.a.items[base + wi].masks = cm | (km << 8) | (kf << 16);
      x.a.items[base + wi].pstart = __popc(cm); // every thread holds its own copy of it
      s_room = room;
    }
    __syncthreads();
    const bool room = s_room; // block-uniform: it guards barriers below
    if (room && t < 8 && s_last[t] >= 0) pol.replaced(l, it.old, t);
    if (room && t < 8 && ((s_cm >> t) & 1u)) {
      const uint32_t k = __popc(s_cm & ((1u << t) - 1u));
      Item ci{};
      ci.cell = child_cell(it.cell, t);
      ci.old = s_last[t] >= 0 ? s_const[t] : old_child;
      ci.pstart = s_pair_base + s_start[t];
      ci.pcount = s_cnt[t];
      ci.result = static_cast<uint32_t>(base + wi);
      x.a.items[next_base + s_item_base + k] = ci;
      note_big(x, l + 1, s_item_base + k, s_cnt[t]);
    }
    // Walk 3: order-preserving compaction, one Threads-pair chunk at a time.
    uint32_t run[8];
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) run[c] = s_pair_base + s_start[c];
    for (uint32_t k0 = 0; k0 < it.pcount && room; k0 += Threads) {
      const uint32_t k = k0 + t;
      uint32_t take = 0, p = 0;
      if (k < it.pcount && cached) {
        p = in_pairs[it.pstart + k];
        const uint32_t mixed = s_mixed[k];
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c)
          if (static_cast<int32_t>(p) > last[c] && ((mixed >> c) & 1u)) take |= 1u << c;
      } else if (k < it.pcount) {
        p = in_pairs[it.pstart + k];
        const vx_primitive pr = x.prims[p];
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c) {
          if (static_cast<int32_t>(p) <= last[c]) continue;
          const int64_t ox = int64_t(2 * cell.x + (c & 1u)) * csize;
          const int64_t oy = int64_t(2 * cell.y + ((c >> 1) & 1u)) * csize;
          const int64_t oz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * csize;
          if (pol.template classify<Terrain>(pr, world_exp, ox, oy, oz, csize) == VX_CELL_MIXED)
            take |= 1u << c;
        }
      }
      uint32_t ballots[8];
#pragma unroll
      for (uint32_t c = 0; c < 8; ++c) {
        ballots[c] = __ballot_sync(kFullMask, (take >> c) & 1u);
        if (lane == 0) s_warp[c][warp] = __popc(ballots[c]);
      }
      __syncthreads();
      if (warp == 0) { // exclusive offsets of the warps, per child, by shuffles
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c) {
          const uint32_t v = lane < kWarps ? s_warp[c][lane] : 0u;
          const uint32_t inc = warp_inclusive_sum(v);
          if (lane < kWarps) s_warp[c][lane] = inc - v;
          if (lane == kWarp - 1) s_total[c] = inc;
        }
      }
      __syncthreads();
#pragma unroll
      for (uint32_t c = 0; c < 8; ++c) {
        if ((take >> c) & 1u)
          out_pairs[run[c] + s_warp[c][warp] + __popc(ballots[c] & lanemask_lt())] = p;
        run[c] += s_total[c];
      }
      __syncthreads();
    }
    __syncthreads();
  }
}

template <class Policy, bool Terrain, uint32_t Threads = Terrain ? kBlock : kBigBlock>
__global__ void __launch_bounds__(Threads)
    expand_big_kernel(EditCtx x, Policy pol, uint32_t l) {
  expand_big_body<Policy, Terrain, Threads, kBigCache>(x, pol, l, launch_blocks());
}

} // namespace vx::edit
