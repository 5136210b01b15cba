// Pointer sparse voxel octree on one B200: in-place batched / plain edits,
// terrain builds, queries, counters, canonical dump.
//
// Layout (the reference GpuSvo, svt/cuda/storage.cuh:12-122 and
// device_view.cuh:11-44): nodes are 8 u32 child words — bits 0-29 child
// index, bit 30 child present, bit 31 filled when absent (svt/cuda/config.cuh:
// 36-42); node 0 is the root and always exists.  Leaves are u64 masks
// (bit = x + 4y + 16z).  With materials each leaf also owns 64 material bytes
// and an absent filled child keeps its material in bits 0-7; a region
// collapses only when occupancy and material are both uniform.  Without
// materials the structure is exactly the reference's: a node or leaf exists
// iff its region is not uniform (svo.hpp:26-91, GPU collapse
// svt/cuda/voxel/detail/collapse/kernels.cuh:12-94).
//
// Edits use the shared top-down expansion (edit_common.cuh); the rebuild then
// updates nodes in place bottom-up: a changed region that stays non-uniform
// reuses its node / leaf, a new one takes an index from the free-list
// snapshot first and the bump counter after (the reference's rank -> index
// rule, svt/cuda/voxel/detail/allocation/materialize_common.cuh:72-84), and a
// region that became uniform detaches its old subtree.  Detached subtrees are
// reclaimed by a reachability pass that rebuilds the free lists.  Before any
// write the edit checks that the worst-case allocation fits; if not it
// reports VX_ERR_CAPACITY and changes nothing.
#include <cooperative_groups.h>

#include "edit_common.cuh"
#include "voxel_b200_device.cuh"
#include "plain.cuh"
#include "graph.cuh"
#include "profile.cuh"
#include "tuning.cuh"

#include <algorithm>
#include <new>
#include <vector>

namespace vx::svo {

using namespace vx::edit;

constexpr uint32_t kChild = 1u << 30, kFilled = 1u << 31, kIndex = kChild - 1u;
constexpr uint32_t kMaxDepth = 12;

struct Counters {
  uint32_t node_count, leaf_count, free_node_count, free_leaf_count;
  uint32_t base_node_count, base_leaf_count, base_free_nodes, base_free_leaves;
  uint32_t taken_nodes, taken_leaves;
  uint32_t detached;   // some subtree became unreachable since the last collection
  uint32_t gc_needed;  // the collection stages run (gate read by every block)
  uint32_t gc_count[kMaxDepth + 1];
};

struct Tables {
  uint32_t depth;
  uint32_t materials;
  uint32_t *nodes;
  uint64_t *leaves;
  uint8_t *mats;
  uint32_t *free_nodes;
  uint32_t *free_leaves;
  uint8_t *node_mark;
  uint8_t *leaf_mark;
  uint32_t *front[2];
  uint32_t max_nodes, max_leaves;
  Counters *ctr;
  Header *hdr;
};

__device__ __forceinline__ uint32_t word_value(uint32_t w, bool mats) {
  return (w & kFilled) ? (mats ? (w & 0xffu) : 1u) : 0u;
}
__device__ __forceinline__ uint32_t uniform_word(uint32_t v, bool mats) {
  return v ? (kFilled | (mats ? v : 0u)) : 0u;
}

// Material an add primitive writes at height z (terrain: its height band).
__device__ __forceinline__ uint32_t prim_material(const vx_primitive &p, uint32_t world_exp,
                                                  uint32_t z) {
  if (vx_prim_shape(&p) == kShapeTerrain) {
    const vx_terrain t{static_cast<uint32_t>(p.c[0]), static_cast<uint32_t>(p.c[1]),
                       static_cast<uint32_t>(p.c[2]), world_exp};
    return vx_terrain_material(&t, z);
  }
  const uint32_t m = vx_prim_material(&p);
  return m ? m : 1u;
}

struct SvoTree {
  Tables t;
  static constexpr bool kItemsForConst = true;
  __device__ uint32_t child(uint32_t, uint32_t old, uint32_t c) const {
    if (old & kChild) return t.nodes[static_cast<size_t>(old & kIndex) * 8u + c];
    return old; // a uniform region's children hold the same value
  }
  // A materialised child overwritten by a covering primitive leaves its
  // subtree unreachable: flag it for a later collection.
  __device__ void replaced(uint32_t l, uint32_t old, uint32_t c) const {
    if ((old & kChild) && (child(l, old, c) & kChild)) atomicOr(&t.ctr->detached, 1u);
  }
  template <bool Terrain>
  __device__ uint32_t classify(const vx_primitive &p, uint32_t world_exp, int64_t ox,
                               int64_t oy, int64_t oz, int64_t n) const {
    const uint32_t c = vx::edit::classify<Terrain>(p, world_exp, ox, oy, oz, n);
    if (Terrain && t.materials && c == VX_CELL_FULL && vx_prim_shape(&p) == kShapeTerrain) {
      // solid terrain is uniform only inside one material band
      const int64_t band = 8 * static_cast<int64_t>(p.c[1]);
      if (oz / band != (oz + n - 1) / band) return VX_CELL_MIXED;
    }
    return c;
  }
  __device__ uint32_t const_value(const vx_primitive &p, int64_t oz, int64_t) const {
    if (vx_prim_op(&p) != VX_OP_ADD) return 0u;
    return uniform_word(prim_material(p, t.depth + 2, static_cast<uint32_t>(oz)),
                        t.materials != 0);
  }
};

__device__ __forceinline__ uint32_t alloc_node(const Tables &t) {
  const uint32_t r = warp_atomic_add_small(&t.ctr->taken_nodes, 1u);
  const uint32_t bf = t.ctr->base_free_nodes;
  return r < bf ? t.free_nodes[bf - 1u - r] : t.ctr->base_node_count + (r - bf);
}
__device__ __forceinline__ uint32_t alloc_leaf(const Tables &t) {
  const uint32_t r = warp_atomic_add_small(&t.ctr->taken_leaves, 1u);
  const uint32_t bf = t.ctr->base_free_leaves;
  return r < bf ? t.free_leaves[bf - 1u - r] : t.ctr->base_leaf_count + (r - bf);
}

// The word a rebuilt cell leaves in its parent: uniform when all 8 children
// are the same uniform word (never for the root), else a node, reused or new.
__device__ uint32_t finish_node(const Tables &t, uint32_t old, const uint32_t (&child)[8],
                                bool is_root) {
  bool uni = (child[0] & kChild) == 0u;
#pragma unroll
  for (uint32_t c = 1; c < 8; ++c) uni = uni && child[c] == child[0];
  if (uni && !is_root) {
    if (old & kChild) atomicOr(&t.ctr->detached, 1u);
    return child[0];
  }
  const uint32_t idx = is_root ? 0u : ((old & kChild) ? (old & kIndex) : alloc_node(t));
  uint4 *dst = reinterpret_cast<uint4 *>(t.nodes + static_cast<size_t>(idx) * 8u);
  dst[0] = make_uint4(child[0], child[1], child[2], child[3]);
  dst[1] = make_uint4(child[4], child[5], child[6], child[7]);
  // A materialised child keeps the fill of the uniform region it replaced in
  // bit 31, as the reference does (make_child_data, svt/cuda/detail/
  // node_ops.cuh:24-28; SVO::set_voxel, svo.hpp:54-58); a reused one keeps its.
  return kChild | idx | (old & kFilled);
}

__device__ __forceinline__ void begin_body(Tables t) {
  Counters *c = t.ctr;
  c->base_node_count = c->node_count;
  c->base_leaf_count = c->leaf_count;
  c->base_free_nodes = c->free_node_count;
  c->base_free_leaves = c->free_leaf_count;
  c->taken_nodes = 0;
  c->taken_leaves = 0;
}
__global__ void begin_kernel(Tables t) { begin_body(t); }

// Worst case before any write: every item below the root may need a node and
// every leaf child of the last level a leaf.
// Nodes and leaves the edit may need (every item below the root a node, 8
// leaves per leaf-parent item) against what the free lists and the unused
// tail hold.
__device__ __forceinline__ bool edit_fits(const Tables &t) {
  const Header *h = t.hdr;
  uint64_t nodes = 0;
  for (uint32_t l = 1; l < t.depth; ++l) nodes += h->item_count[l];
  const uint64_t leaves = 8ull * h->item_count[t.depth - 1];
  const Counters *c = t.ctr;
  const uint64_t avail_nodes = c->base_free_nodes + uint64_t(t.max_nodes - c->base_node_count);
  const uint64_t avail_leaves = c->base_free_leaves + uint64_t(t.max_leaves - c->base_leaf_count);
  return nodes <= avail_nodes && leaves <= avail_leaves;
}

// Garbage is collected lazily: only when an edit would not fit in the room
// left does the collection run, before the edit allocates anything (the
// edit has only read the tree so far, so marking from the current root
// keeps everything it reads).  A capacity error follows only if the edit
// still does not fit after it.
__device__ __forceinline__ void check_capacity_body(Tables t) {
  Header *h = t.hdr;
  t.ctr->gc_needed = 0;
  if (h->status != kDevOk) return;
  if (!edit_fits(t)) {
    if (t.ctr->detached) t.ctr->gc_needed = 1;
    else h->status = kDevCapacity;
  }
}
__global__ void check_capacity_kernel(Tables t) { check_capacity_body(t); }

__device__ void finish_upwards(const EditCtx &x, const Tables &t, uint32_t parent, uint32_t l);

// Climb: after storing an item's word, finish its ancestors (the single
// cooperative kernel's bottom-up build, without level barriers).
template <bool Terrain, bool Climb = false>
__device__ __forceinline__ void leafparent_body(EditCtx x, Tables t, Blocks blk) {
  Header *h = x.hdr;
  const SvoTree pol{t};
  const uint32_t l = t.depth - 1;
  const uint32_t W = h->item_count[l]; // loaded beside the status
  const uint32_t base = h->item_off[l];
  if (edit_failed(h)) return;
  const uint32_t *pairs = x.a.pairs[l & 1u];
  const uint32_t world_exp = t.depth + 2;
  const bool mats = t.materials != 0;
  const uint32_t lane = lane_id();
  // one item per 8 lanes: its group's chunk of primitives
  __shared__ vx_primitive s_prim[kBlock / 8][8];
  const uint32_t group = threadIdx.x >> 3;
  const uint32_t gmask = 0xffu << (lane & ~7u);
  const uint64_t total = static_cast<uint64_t>(W) * 8u;
  const uint64_t stride = static_cast<uint64_t>(blk.count) * blockDim.x;
  for (uint64_t g0 = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x - lane;
       g0 < total; g0 += stride) {
    const uint64_t g = g0 + lane;
    const bool have = g < total;
    const uint32_t wi = static_cast<uint32_t>(g >> 3), c = lane & 7u;
    uint32_t result = 0;
    Item it{};
    if (have) {
      it = x.a.items[base + wi];
      const Cell cell = unpack_cell(it.cell);
      const int64_t ox = int64_t(2 * cell.x + (c & 1u)) * 4;
      const int64_t oy = int64_t(2 * cell.y + ((c >> 1) & 1u)) * 4;
      const int64_t oz = int64_t(2 * cell.z + ((c >> 2) & 1u)) * 4;
      const uint32_t oc = pol.child(l, it.old, c);
      // The leaf's previous content: for edits loaded beside the primitives
      // (a covering primitive overwrites all of it, so loading it in any case
      // changes nothing); a terrain build, whose classification needs the
      // registers, loads it at its first partial primitive.
      uint64_t mask = 0;
      uint32_t v[16]; // 64 material bytes, 4 per word; word w holds z = w >> 2
      auto load_old = [&]() {
        if (oc & kChild) {
          const uint32_t li = oc & kIndex;
          mask = t.leaves[li];
          if (mats) {
            const uint4 *src = reinterpret_cast<const uint4 *>(t.mats + static_cast<size_t>(li) * 64u);
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
              const uint4 u = src[q];
              v[4 * q] = u.x;
              v[4 * q + 1] = u.y;
              v[4 * q + 2] = u.z;
              v[4 * q + 3] = u.w;
            }
          }
        } else {
          const uint32_t val = word_value(oc, mats);
          mask = val ? ~0ull : 0ull;
          if (mats)
#pragma unroll
            for (uint32_t w = 0; w < 16; ++w) v[w] = val * 0x01010101u;
        }
      };
      if (!Terrain) load_old();
      bool loaded = !Terrain, touched = false;
      // One primitive's effect on this lane's leaf.
      auto apply = [&](const vx_primitive &pr) {
        const uint32_t cls = pol.template classify<Terrain>(pr, world_exp, ox, oy, oz, 4);
        if (cls == VX_CELL_EMPTY) return;
        const bool add = vx_prim_op(&pr) == VX_OP_ADD;
        if (!loaded && cls == VX_CELL_MIXED) load_old();
        loaded = true;
        touched = true;
        const uint64_t m = cls == VX_CELL_FULL ? ~0ull : leaf_mask<Terrain>(pr, world_exp, ox, oy, oz);
        mask = add ? (mask | m) : (mask & ~m);
        if (mats) {
#pragma unroll
          for (uint32_t w = 0; w < 16; ++w) {
            const uint32_t nib = static_cast<uint32_t>(m >> (4 * w)) & 0xfu;
            if (!nib) continue;
            const uint32_t bm = ((nib & 1u) ? 0xffu : 0u) | ((nib & 2u) ? 0xff00u : 0u) |
                                ((nib & 4u) ? 0xff0000u : 0u) | ((nib & 8u) ? 0xff000000u : 0u);
            const uint32_t val =
                add ? prim_material(pr, world_exp, static_cast<uint32_t>(oz) + (w >> 2)) : 0u;
            v[w] = (v[w] & ~bm) | ((val * 0x01010101u) & bm);
          }
        }
      };
      // A terrain build's items hold its single primitive, read in place; an
      // edit's primitives come eight at a time, staged in shared memory by the
      // item's eight lanes (independent loads, not two dependent ones per
      // primitive).
      for (uint32_t k = 0; Terrain && k < it.pcount; ++k) apply(x.prims[pairs[it.pstart + k]]);
      for (uint32_t k0 = 0; !Terrain && k0 < it.pcount; k0 += 8) {
        if (k0 + c < it.pcount) s_prim[group][c] = x.prims[pairs[it.pstart + k0 + c]];
        __syncwarp(gmask);
        const uint32_t m = min(8u, it.pcount - k0);
        for (uint32_t j = 0; j < m; ++j) apply(s_prim[group][j]);
        __syncwarp(gmask); // the chunk is overwritten next
      }
      if (!touched) {
        result = oc;
      } else {
        bool uni;
        uint32_t uval;
        if (mats) {
          uni = true;
#pragma unroll
          for (uint32_t w = 1; w < 16; ++w) uni = uni && v[w] == v[0];
          uni = uni && v[0] == (v[0] & 0xffu) * 0x01010101u;
          uval = v[0] & 0xffu;
        } else {
          uni = mask == 0 || mask == ~0ull;
          uval = mask ? 1u : 0u;
        }
        if (uni) {
          if (oc & kChild) atomicOr(&t.ctr->detached, 1u);
          result = uniform_word(uval, mats);
        } else {
          const uint32_t li = (oc & kChild) ? (oc & kIndex) : alloc_leaf(t);
          t.leaves[li] = mask;
          if (mats) {
            uint4 *dst = reinterpret_cast<uint4 *>(t.mats + static_cast<size_t>(li) * 64u);
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q)
              dst[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
          }
          result = kChild | li | (oc & kFilled);
        }
      }
    }
    uint32_t child[8];
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k)
      child[k] = __shfl_sync(kFullMask, result, (lane & ~7u) + k);
    if (have && c == 0) {
      x.a.items[base + wi].result = finish_node(t, it.old, child, l == 0);
      if (Climb) finish_upwards(x, t, it.result, l); // it.result: the parent's index
    }
  }
}

template <bool Terrain>
__global__ void __launch_bounds__(kBlock) leafparent_kernel(EditCtx x, Tables t) {
  leafparent_body<Terrain>(x, t, launch_blocks());
}

// The rebuilt word of one item at inner level l from its children's results
// (Climb: read from L2, other SMs wrote them in this launch).
template <bool Climb = false>
__device__ __forceinline__ uint32_t build_item(const EditCtx &x, const Tables &t, uint32_t l,
                                               const Item &it) {
  const uint32_t cm = it.masks & 0xffu;
  uint32_t child[8];
  if (it.old & kChild) {
    const uint4 *src = reinterpret_cast<const uint4 *>(t.nodes + static_cast<size_t>(it.old & kIndex) * 8u);
    const uint4 a = src[0], b = src[1];
    child[0] = a.x; child[1] = a.y; child[2] = a.z; child[3] = a.w;
    child[4] = b.x; child[5] = b.y; child[6] = b.z; child[7] = b.w;
  } else {
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) child[c] = it.old;
  }
  uint32_t k = 0;
#pragma unroll
  for (uint32_t c = 0; c < 8; ++c)
    if (cm & (1u << c)) {
      const uint32_t *r = &x.a.items[it.child_base + k++].result;
      child[c] = Climb ? __ldcg(r) : *r;
    }
  return finish_node(t, it.old, child, l == 0);
}

__device__ __forceinline__ void build_body(EditCtx x, Tables t, uint32_t l, Blocks blk) {
  Header *h = x.hdr;
  const uint32_t W = h->item_count[l]; // loaded beside the status
  const uint32_t base = h->item_off[l];
  if (edit_failed(h)) return;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < W; i += static_cast<uint64_t>(blk.count) * blockDim.x)
    x.a.items[base + i].result = build_item(x, t, l, x.a.items[base + i]);
}

// Bottom-up without level barriers (the single cooperative kernel): an item
// at level l has just stored its word; count it off its parent's pending
// children with one acquire-release decrement, and when it was the last one
// rebuild the parent and go on up.  A node is rewritten in place only when
// all of its children are done, as in the level-by-level build.
__device__ void finish_upwards(const EditCtx &x, const Tables &t, uint32_t parent, uint32_t l) {
  while (parent != kNoParent) {
    // The parent's own fields were written by its expansion, stages ago:
    // read them while the decrement is in flight (only the children's
    // results need its acquire).
    const Item it = load_item_l2(&x.a.items[parent]);
    if (atomic_sub_acq_rel(&x.a.items[parent].pstart, 1u) != 1u) return;
    --l;
    x.a.items[parent].result = build_item<true>(x, t, l, it);
    parent = it.result; // the grandparent, stored there until now
  }
}

// Items below the leaf-parent level with no child items rebuild at once and
// start their own climb.
__device__ __forceinline__ void rebuild_childless_body(EditCtx x, Tables t, Blocks blk) {
  Header *h = x.hdr;
  // every level's counts in one round trip
  __shared__ uint32_t s_w[kMaxDepth], s_base[kMaxDepth];
  if (threadIdx.x < kMaxDepth) {
    s_w[threadIdx.x] = h->item_count[threadIdx.x];
    s_base[threadIdx.x] = h->item_off[threadIdx.x];
  }
  if (edit_failed(h)) return; // (its barrier also publishes s_w, s_base)
  for (uint32_t l = 0; l + 1 < t.depth; ++l) {
    const uint32_t W = s_w[l];
    const uint32_t base = s_base[l];
    for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         i < W; i += static_cast<uint64_t>(blk.count) * blockDim.x) {
      const Item it = x.a.items[base + i];
      if (it.masks & 0xffu) continue;
      x.a.items[base + i].result = build_item<true>(x, t, l, it);
      finish_upwards(x, t, it.result, l);
    }
  }
}

__global__ void __launch_bounds__(kBlock) build_kernel(EditCtx x, Tables t, uint32_t l) {
  build_body(x, t, l, launch_blocks());
}

__device__ __forceinline__ void finalize_body(Tables t) {
  Counters *c = t.ctr;
  if (t.hdr->status != kDevOk) return;
  const uint32_t tn = c->taken_nodes, tl = c->taken_leaves;
  if (tn <= c->base_free_nodes) {
    c->free_node_count = c->base_free_nodes - tn;
  } else {
    c->free_node_count = 0;
    c->node_count = c->base_node_count + (tn - c->base_free_nodes);
  }
  if (tl <= c->base_free_leaves) {
    c->free_leaf_count = c->base_free_leaves - tl;
  } else {
    c->free_leaf_count = 0;
    c->leaf_count = c->base_leaf_count + (tl - c->base_free_leaves);
  }
}
__global__ void finalize_kernel(Tables t) { finalize_body(t); }

// ------------------------------------------------------------------- GC --

__device__ __forceinline__ void gc_clear_body(Tables t, Blocks blk) {
  Counters *c = t.ctr;
  if (!c->gc_needed) return;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < c->node_count; i += static_cast<uint64_t>(blk.count) * blockDim.x)
    t.node_mark[i] = 0;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < c->leaf_count; i += static_cast<uint64_t>(blk.count) * blockDim.x)
    t.leaf_mark[i] = 0;
  if (blk.id == 0 && threadIdx.x == 0) {
    for (uint32_t l = 0; l <= kMaxDepth; ++l) c->gc_count[l] = 0;
    c->gc_count[0] = 1;
    t.front[0][0] = 0; // the root
  }
}
__global__ void gc_clear_kernel(Tables t) { gc_clear_body(t, launch_blocks()); }

__device__ __forceinline__ void gc_level_body(Tables t, uint32_t l, Blocks blk) {
  Counters *c = t.ctr;
  if (!c->gc_needed) return;
  const uint32_t n = c->gc_count[l];
  const uint32_t *front = t.front[l & 1u];
  uint32_t *next = t.front[(l + 1) & 1u];
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(blk.count) * blockDim.x) {
    const uint32_t node = front[i];
    t.node_mark[node] = 1;
    for (uint32_t k = 0; k < 8; ++k) {
      const uint32_t w = t.nodes[static_cast<size_t>(node) * 8u + k];
      if (!(w & kChild)) continue;
      if (l + 1 < t.depth) next[atomicAdd(&c->gc_count[l + 1], 1u)] = w & kIndex;
      else t.leaf_mark[w & kIndex] = 1;
    }
  }
}
__global__ void gc_level_kernel(Tables t, uint32_t l) { gc_level_body(t, l, launch_blocks()); }

__device__ __forceinline__ void gc_zero_free_body(Tables t) {
  Counters *c = t.ctr;
  if (!c->gc_needed) return;
  c->free_node_count = 0;
  c->free_leaf_count = 0;
}
__global__ void gc_zero_free_kernel(Tables t) { gc_zero_free_body(t); }

__device__ __forceinline__ void gc_rebuild_body(Tables t, Blocks blk) {
  Counters *c = t.ctr;
  if (!c->gc_needed) return;
  const uint32_t nn = c->node_count, nl = c->leaf_count;
  for (uint64_t i = 1 + blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < nn;
       i += static_cast<uint64_t>(blk.count) * blockDim.x)
    if (!t.node_mark[i]) t.free_nodes[atomicAdd(&c->free_node_count, 1u)] = static_cast<uint32_t>(i);
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < nl;
       i += static_cast<uint64_t>(blk.count) * blockDim.x)
    if (!t.leaf_mark[i]) t.free_leaves[atomicAdd(&c->free_leaf_count, 1u)] = static_cast<uint32_t>(i);
}
__global__ void gc_rebuild_kernel(Tables t) { gc_rebuild_body(t, launch_blocks()); }

// After a collection inside an edit: the free lists are the edit's starting
// point; the edit fails only if it still does not fit.
__device__ __forceinline__ void gc_recheck_body(Tables t) {
  Counters *c = t.ctr;
  if (!c->gc_needed) return;
  c->gc_needed = 0;
  c->detached = 0;
  c->base_free_nodes = c->free_node_count;
  c->base_free_leaves = c->free_leaf_count;
  if (t.hdr->status == kDevOk && !edit_fits(t)) t.hdr->status = kDevCapacity;
}
__global__ void gc_recheck_kernel(Tables t) { gc_recheck_body(t); }

// vx_svo_collect: a collection on request, between edits.
__global__ void gc_request_kernel(Tables t) { t.ctr->gc_needed = t.ctr->detached; }
__global__ void gc_end_kernel(Tables t) {
  if (t.ctr->gc_needed) t.ctr->detached = 0;
  t.ctr->gc_needed = 0;
}

// A whole edit, collection included, in one cooperative launch: the stages
// of run_pipeline separated by grid-wide barriers instead of kernel
// boundaries, for small batches, where ~30 launches cost more than the work
// (the plain per-call path).  Long primitive lists are expanded with a
// 256-thread block and a 4 KiB classification cache.  Requires every block of
// the grid to be resident (cudaLaunchCooperativeKernel checks it).
constexpr uint32_t kSmallBigCache = 4096;

// With Plain, the edit's input is a voxel list (one op and material): the
// first stages turn it into leaf-mask primitives (PlainPrep) in place of the
// sort-based preparation of the multi-launch path.
// One block per SM runs it, so it may take up to 255 registers (the
// default cap for 256-thread blocks, 128, made it spill).
template <bool Plain>
__global__ void __maxnreg__(255) small_edit_kernel(EditCtx e, Tables t, PlainPrep prep,
                                                            uint32_t *status_out) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const Blocks blk = launch_blocks();
  const SvoTree pol{t};
  const bool lead = blk.id == 0 && threadIdx.x == 0;
  if (Plain) {
    plain_prep_clear(prep, blk);
    grid.sync();
    plain_prep_aggregate(prep, t.depth, blk);
    grid.sync();
    plain_prep_fill(prep, blk); // beside init: both need only the final count
  }
  if (lead) begin_body(t);
  init_body(e, kChild, blk);
  grid.sync();
  for (uint32_t l = 0; l + 1 < t.depth; ++l) {
    // Short and long lists of level l side by side, one barrier per level:
    // the long ones were listed when level l was emitted (their count is
    // final at the barrier before, the same in every block) and go to the
    // blocks from the last one down, the short ones from block 0 up.
    expand_body<SvoTree, false>(e, pol, l, blk);
    if (t.hdr->big_count[l] != 0)
      expand_big_body<SvoTree, false, kBlock, kSmallBigCache>(e, pol, l,
                                                          Blocks{blk.count - 1u - blk.id, blk.count});
    grid.sync();
  }
  // Every block reaches the capacity verdict of check_capacity_body from the
  // same final counts, so the common case (the edit fits) needs no barrier.
  __shared__ uint32_t s_verdict; // 0 fits, 1 collect first, 2 no room
  if (threadIdx.x == 0) {
    uint32_t v = 0;
    if (t.hdr->status == kDevOk && !edit_fits(t)) v = t.ctr->detached ? 1u : 2u;
    s_verdict = v;
  }
  __syncthreads();
  const uint32_t verdict = s_verdict;
  if (lead) t.ctr->gc_needed = verdict == 1u; // no other block reads it before a barrier
  if (verdict == 1u) {
    grid.sync(); // gc_needed, read by every collection stage
    gc_clear_body(t, blk);
    grid.sync();
    for (uint32_t l = 0; l < t.depth; ++l) {
      gc_level_body(t, l, blk);
      grid.sync();
    }
    if (lead) gc_zero_free_body(t);
    grid.sync();
    gc_rebuild_body(t, blk);
    grid.sync();
    if (lead) gc_recheck_body(t);
    grid.sync();
  }
  // The bottom-up build without level barriers: the leaf-parent items and
  // the childless items of the levels above finish their ancestors, each
  // item rebuilt by the last of its children to finish.
  if (verdict != 2u) {
    leafparent_body<false, true>(e, t, blk);
    rebuild_childless_body(e, t, blk);
  }
  grid.sync();
  if (lead) {
    // written after the barrier: every block has read the status by then
    if (verdict == 2u) t.hdr->status = kDevCapacity;
    finalize_body(t);
    if (status_out) *status_out = t.hdr->status; // the caller's mapped host word
  }
}

__global__ void reset_kernel(Tables t) {
#pragma unroll
  for (uint32_t c = 0; c < 8; ++c) t.nodes[c] = 0;
  Counters *c = t.ctr;
  c->node_count = 1;
  c->leaf_count = 0;
  c->free_node_count = 0;
  c->free_leaf_count = 0;
  c->detached = 0;
  c->gc_needed = 0;
  t.hdr->status = kDevOk;
}

__global__ void query_kernel(vx_svo_view v, const vx_voxel *pts, uint32_t n, uint8_t *out) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const vx_voxel p = pts[i];
  out[i] = vx_svo_get_voxel(v, p.x, p.y, p.z);
}

} // namespace vx::svo

// ================================================================ handle ==

struct vx_svo {
  vx::svo::Tables t{};
  vx::edit::Arena a{};
  void *arena_mem = nullptr;
  vx_primitive *tmp_prim = nullptr;
  uint32_t *host_status = nullptr; // pinned word for status reads (allocated on first use)
  uint32_t *status_alias = nullptr; // its device address, when mapped at creation
};

namespace vx::svo {

// The single cooperative launch of small_edit_kernel, on as many blocks as
// are resident at once (at most the edit.small_blocks_per_sm knob per SM).
// Resident blocks per SM of small_edit_kernel<plain or not>, queried once
// (at SVO creation, so never first inside a stream capture).
int g_small_resident[2] = {-1, -1};
inline const void *small_kernel(bool plain) {
  return plain ? reinterpret_cast<const void *>(&small_edit_kernel<true>)
               : reinterpret_cast<const void *>(&small_edit_kernel<false>);
}
vx_status query_small_residency() {
  for (int plain = 0; plain < 2; ++plain) {
    if (g_small_resident[plain] >= 0) continue;
    int n = 0;
    VX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, small_kernel(plain != 0),
                                                              kBlock, 0));
    g_small_resident[plain] = n;
  }
  return VX_OK;
}

// status_out: a mapped host word the kernel's last act writes the status to.
vx_status run_small(const EditCtx &e, const Tables &t, cudaStream_t s,
                    const PlainPrep *prep = nullptr, uint32_t *status_out = nullptr) {
  VX_TRY(query_small_residency());
  const int per_sm = g_small_resident[prep ? 1 : 0];
  if (per_sm < 1) return VX_ERR_INVALID_VALUE;
  const int want = static_cast<int>(tune::get(tune::kEditSmallBlocksPerSm));
  const uint32_t grid = static_cast<uint32_t>(sm_count()) *
                        static_cast<uint32_t>(std::max(1, std::min(per_sm, want)));
  EditCtx ec = e;
  Tables tc = t;
  PlainPrep pp = prep ? *prep : PlainPrep{};
  void *args[] = {&ec, &tc, &pp, &status_out};
  prof::Scope sc("svo_small_edit", s);
  VX_TRY_CUDA(cudaLaunchCooperativeKernel(small_kernel(prep != nullptr), dim3(grid),
                                          dim3(kBlock), args, 0, s));
  return VX_OK;
}

// Small edits (by the edit.small_max_* knobs) run as one cooperative kernel:
// a batch of primitives by its count, a voxel list or leaf commands by its
// length.
inline bool small_batch(uint32_t n, bool voxel_list) {
  return n <= static_cast<uint32_t>(tune::get(voxel_list ? tune::kEditSmallMaxVoxels
                                                         : tune::kEditSmallMaxPrims));
}

// The collection stages as kernels, each leaving at once unless gc_needed is
// set: by the capacity check inside an edit (ended by gc_recheck_kernel), or
// by gc_request_kernel when a caller asks (ended by gc_end_kernel).
vx_status launch_collection(const Tables &t, uint32_t grid, cudaStream_t s, bool on_request) {
  prof::Scope sc("svo_gc", s);
  if (on_request) gc_request_kernel<<<1, 1, 0, s>>>(t);
  gc_clear_kernel<<<grid, kBlock, 0, s>>>(t);
  for (uint32_t l = 0; l < t.depth; ++l) gc_level_kernel<<<grid, kBlock, 0, s>>>(t, l);
  gc_zero_free_kernel<<<1, 1, 0, s>>>(t);
  gc_rebuild_kernel<<<grid, kBlock, 0, s>>>(t);
  if (on_request) gc_end_kernel<<<1, 1, 0, s>>>(t);
  else gc_recheck_kernel<<<1, 1, 0, s>>>(t);
  return from_cuda(cudaGetLastError());
}

vx_status run_pipeline(vx_svo *v, const vx_primitive *prims, const uint32_t *d_count,
                       uint32_t host_count, cudaStream_t s, bool terrain,
                       int small = -1 /* -1: by host_count as a primitive batch */) {
  const Tables &t = v->t;
  const EditCtx e{t.hdr, v->a, prims, d_count, host_count, t.depth,
                  static_cast<uint32_t>(tune::get(tune::kEditBigItem))};
  const SvoTree pol{t};
  const uint32_t depth = t.depth;
  const uint32_t grid = static_cast<uint32_t>(sm_count()) *
                        static_cast<uint32_t>(tune::get(tune::kEditBlocksPerSm));
  if (!terrain && (small < 0 ? small_batch(host_count, false) : small != 0))
    return run_small(e, t, s);
  {
    prof::Scope sc("svo_init", s);
    begin_kernel<<<1, 1, 0, s>>>(t);
    init_kernel<<<std::min<uint32_t>(grid, ceil_div(std::max(host_count, 1u), kBlock) + 1),
                  kBlock, 0, s>>>(e, kChild);
  }
  VX_TRY_CUDA(cudaGetLastError());
  for (uint32_t l = 0; l + 1 < depth; ++l) {
    {
      prof::Scope sc("svo_expand", s);
      if (terrain) expand_kernel<SvoTree, true><<<grid, kBlock, 0, s>>>(e, pol, l);
      else expand_kernel<SvoTree, false><<<grid, kBlock, 0, s>>>(e, pol, l);
    }
    VX_TRY_CUDA(cudaGetLastError());
    {
      prof::Scope sc("svo_expand_big", s);
      if (terrain) expand_big_kernel<SvoTree, true><<<sm_count() * 2, kBlock, 0, s>>>(e, pol, l);
      else expand_big_kernel<SvoTree, false><<<sm_count(), kBigBlock, 0, s>>>(e, pol, l);
    }
    VX_TRY_CUDA(cudaGetLastError());
  }
  {
    prof::Scope sc("svo_check_capacity", s);
    check_capacity_kernel<<<1, 1, 0, s>>>(t);
  }
  VX_TRY(launch_collection(t, grid, s, false));
  {
    prof::Scope sc("svo_leafparent", s);
    if (terrain) leafparent_kernel<true><<<grid, kBlock, 0, s>>>(e, t);
    else leafparent_kernel<false><<<grid, kBlock, 0, s>>>(e, t);
  }
  VX_TRY_CUDA(cudaGetLastError());
  for (uint32_t r = depth - 1; r > 0; --r) {
    prof::Scope sc("svo_build", s);
    build_kernel<<<grid, kBlock, 0, s>>>(e, t, r - 1);
    VX_TRY_CUDA(cudaGetLastError());
  }
  {
    prof::Scope sc("svo_finalize", s);
    finalize_kernel<<<1, 1, 0, s>>>(t);
  }
  return from_cuda(cudaGetLastError());
}

// The device status, read through a pinned word (a copy into pageable
// memory goes through a staging buffer); a failed status is cleared.
vx_status read_status(vx_svo *v, cudaStream_t s) {
  if (v->host_status == nullptr &&
      cudaHostAlloc(reinterpret_cast<void **>(&v->host_status), sizeof(uint32_t),
                    cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError(); // not fatal: read through a stack word instead
    v->host_status = nullptr;
  }
  uint32_t stack_code = 0;
  uint32_t *code = v->host_status ? v->host_status : &stack_code;
  VX_TRY_CUDA(cudaMemcpyAsync(code, &v->t.hdr->status, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  const uint32_t c = *code;
  if (c != kDevOk) {
    VX_TRY_CUDA(cudaMemsetAsync(&v->t.hdr->status, 0, sizeof(uint32_t), s));
    VX_TRY_CUDA(cudaStreamSynchronize(s));
  }
  return status_from_device(c);
}

// The status a small kernel wrote into the mapped host word (set to
// kStatusUnset before the launch): after the kernel there is no copy to
// wait for.  A word the kernel did not write falls back to read_status.
constexpr uint32_t kStatusUnset = 0xffffffffu;
vx_status read_written_status(vx_svo *v, cudaStream_t s) {
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  const uint32_t c = *reinterpret_cast<volatile uint32_t *>(v->host_status);
  if (c == kStatusUnset) return read_status(v, s);
  if (c != kDevOk) {
    VX_TRY_CUDA(cudaMemsetAsync(&v->t.hdr->status, 0, sizeof(uint32_t), s));
    VX_TRY_CUDA(cudaStreamSynchronize(s));
  }
  return status_from_device(c);
}

} // namespace vx::svo

using namespace vx::svo;

extern "C" {

vx_status vx_svo_create(const vx_svo_config *cfg, vx_svo **out) {
  if (cfg == nullptr || out == nullptr || cfg->depth < 1 || cfg->depth > kMaxDepth ||
      cfg->max_nodes < 1 || cfg->max_leaves < 1 || cfg->max_nodes > kIndex ||
      cfg->max_leaves > kIndex)
    return VX_ERR_INVALID_VALUE;
  int devs = 0;
  if (cudaGetDeviceCount(&devs) != cudaSuccess || devs == 0) return VX_ERR_NO_DEVICE;
  auto *v = new (std::nothrow) vx_svo;
  if (v == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  Tables &t = v->t;
  t.depth = cfg->depth;
  t.materials = cfg->materials ? 1u : 0u;
  t.max_nodes = cfg->max_nodes;
  t.max_leaves = cfg->max_leaves;
  auto fail = [&](cudaError_t e) {
    vx_svo_destroy(v);
    return vx::from_cuda(e);
  };
  cudaError_t e;
  if (vx_status qs = vx::svo::query_small_residency(); qs != VX_OK) {
    vx_svo_destroy(v);
    return qs;
  }
  const size_t nn = cfg->max_nodes, nl = cfg->max_leaves;
  if ((e = cudaMalloc(&t.nodes, nn * 32)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.leaves, nl * 8)) != cudaSuccess) return fail(e);
  if (t.materials && (e = cudaMalloc(&t.mats, nl * 64)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.free_nodes, nn * 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.free_leaves, nl * 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.node_mark, nn)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.leaf_mark, nl)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.front[0], nn * 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.front[1], nn * 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.ctr, sizeof(Counters))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&t.hdr, sizeof(vx::edit::Header))) != cudaSuccess) return fail(e);
  // the status word, mapped so that a small kernel can write it directly
  if (cudaHostAlloc(reinterpret_cast<void **>(&v->host_status), sizeof(uint32_t),
                    cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void **>(&v->status_alias), v->host_status,
                               0) != cudaSuccess) {
    cudaGetLastError(); // not fatal: statuses are then copied
    v->status_alias = nullptr;
  }
  if ((e = cudaMalloc(&v->tmp_prim, sizeof(vx_primitive))) != cudaSuccess) return fail(e);
  const uint64_t arena = cfg->arena_bytes ? cfg->arena_bytes : (256ull << 20);
  if ((e = cudaMalloc(&v->arena_mem, arena)) != cudaSuccess) return fail(e);
  const uint64_t big_bytes = std::min<uint64_t>(arena / 64, 4ull << 20) / 256 * 256;
  const uint64_t item_bytes = (arena - big_bytes) / 10 * 6 / 256 * 256;
  const uint64_t pair_bytes = (arena - big_bytes - item_bytes) / 2 / 256 * 256;
  char *base = static_cast<char *>(v->arena_mem);
  v->a.items = reinterpret_cast<vx::edit::Item *>(base);
  v->a.item_cap = static_cast<uint32_t>(std::min<uint64_t>(item_bytes / sizeof(vx::edit::Item), 0xffffffffull));
  v->a.pairs[0] = reinterpret_cast<uint32_t *>(base + item_bytes);
  v->a.pairs[1] = reinterpret_cast<uint32_t *>(base + item_bytes + pair_bytes);
  v->a.pair_cap = static_cast<uint32_t>(std::min<uint64_t>(pair_bytes / 4, 0xffffffffull));
  v->a.big = reinterpret_cast<uint32_t *>(base + item_bytes + 2 * pair_bytes);
  v->a.big_cap = static_cast<uint32_t>(big_bytes / 4);
  if ((e = cudaMemset(t.hdr, 0, sizeof(vx::edit::Header))) != cudaSuccess) return fail(e);
  if ((e = cudaMemset(t.ctr, 0, sizeof(Counters))) != cudaSuccess) return fail(e);
  const vx_status st = vx_svo_reset(v, nullptr);
  if (st != VX_OK) {
    vx_svo_destroy(v);
    return st;
  }
  if ((e = cudaStreamSynchronize(nullptr)) != cudaSuccess) return fail(e);
  *out = v;
  return VX_OK;
}

vx_status vx_svo_destroy(vx_svo *v) {
  if (v == nullptr) return VX_ERR_INVALID_VALUE;
  Tables &t = v->t;
  cudaFree(t.nodes);
  cudaFree(t.leaves);
  cudaFree(t.mats);
  cudaFree(t.free_nodes);
  cudaFree(t.free_leaves);
  cudaFree(t.node_mark);
  cudaFree(t.leaf_mark);
  cudaFree(t.front[0]);
  cudaFree(t.front[1]);
  cudaFree(t.ctr);
  cudaFree(t.hdr);
  cudaFree(v->tmp_prim);
  if (v->host_status) cudaFreeHost(v->host_status);
  cudaFree(v->arena_mem);
  delete v;
  return VX_OK;
}

// reset_svo (svt/cuda/svo.cuh:17-22): root = all empty, counters {1,0,0,0}.
vx_status vx_svo_reset(vx_svo *v, vx_stream stream) {
  if (v == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("svo_reset", s);
  reset_kernel<<<1, 1, 0, s>>>(v->t);
  return vx::from_cuda(cudaGetLastError());
}

size_t vx_svo_voxel_workspace_size(uint32_t count) {
  return vx::plain::workspace_size(count);
}

vx_status vx_svo_apply_voxels(vx_svo *v, const vx_voxel *edits, uint32_t count,
                              uint32_t op, uint32_t material, void *workspace,
                              size_t workspace_bytes, vx_stream stream) {
  if (v == nullptr || (edits == nullptr && count != 0) || op > 1 || material > 255)
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  if (workspace == nullptr || workspace_bytes < vx_svo_voxel_workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const vx_primitive *prims = nullptr;
  const uint32_t *n = nullptr;
  const uint32_t mat = op == VX_EDIT_PLACE ? (material ? material : 1u) : 0u;
  PlainPrep prep;
  if (small_batch(count, true) &&
      plain_prep_layout(workspace, workspace_bytes, edits, count, op, mat, &prep)) {
    // one cooperative launch: voxels -> leaf masks -> the edit and collection
    const EditCtx e{v->t.hdr, v->a, prep.prims, prep.nprims, count, v->t.depth,
                    static_cast<uint32_t>(vx::tune::get(vx::tune::kEditBigItem))};
    if (v->status_alias == nullptr) {
      VX_TRY(run_small(e, v->t, s, &prep));
      return read_status(v, s);
    }
    *reinterpret_cast<volatile uint32_t *>(v->host_status) = kStatusUnset;
    VX_TRY(run_small(e, v->t, s, &prep, v->status_alias));
    return read_written_status(v, s);
  }
  VX_TRY(vx::plain::prepare(edits, count, v->t.depth, op, mat, workspace, &prims, &n, s));
  VX_TRY(run_pipeline(v, prims, n, count, s, false, small_batch(count, true)));
  return read_status(v, s);
}

vx_status vx_svo_apply_leaf_commands(vx_svo *v, const vx_leaf_command *cmds, uint32_t count,
                                     uint32_t op, uint32_t material, void *workspace,
                                     size_t workspace_bytes, vx_stream stream) {
  if (v == nullptr || (cmds == nullptr && count != 0) || op > 1 || material > 255)
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  if (workspace == nullptr || workspace_bytes < vx_leaf_command_workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const vx_primitive *prims = nullptr;
  const uint32_t *n = nullptr;
  const uint32_t mat = op == VX_EDIT_PLACE ? (material ? material : 1u) : 0u;
  VX_TRY(vx::plain::prepare_leaf_commands(cmds, count, v->t.depth, op, mat, workspace, &prims,
                                          &n, s));
  VX_TRY(run_pipeline(v, prims, n, count, s, false, small_batch(count, true)));
  return read_status(v, s);
}

uint32_t vx_svo_depth(const vx_svo *v) { return v ? v->t.depth : 0; }

vx_status vx_svo_device_view(const vx_svo *v, vx_svo_view *out) {
  if (v == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  *out = vx_svo_view{v->t.depth, v->t.materials, v->t.nodes, v->t.leaves, v->t.mats};
  return VX_OK;
}

vx_status vx_svo_apply_primitives(vx_svo *v, const vx_primitive *prims,
                                  uint32_t count, vx_stream stream) {
  if (v == nullptr || (prims == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  return run_pipeline(v, prims, nullptr, count, static_cast<cudaStream_t>(stream), false);
}

vx_status vx_svo_graph_primitives(vx_svo *v, const vx_primitive *prims,
                                  const uint32_t *device_count, uint32_t capacity,
                                  vx_graph **out) {
  if (v == nullptr || out == nullptr || prims == nullptr || capacity == 0)
    return VX_ERR_INVALID_VALUE;
  return vx::graph::capture(
      [&](cudaStream_t s) { return run_pipeline(v, prims, device_count, capacity, s, false); },
      out);
}

vx_status vx_svo_status(vx_svo *v, vx_stream stream) {
  if (v == nullptr) return VX_ERR_INVALID_VALUE;
  return read_status(v, static_cast<cudaStream_t>(stream));
}

vx_status vx_svo_build_terrain(vx_svo *v, const vx_terrain *terrain, vx_stream stream) {
  if (v == nullptr || terrain == nullptr || terrain->scale == 0) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx_primitive p{};
  p.c[0] = static_cast<int32_t>(terrain->seed);
  p.c[1] = static_cast<int32_t>(terrain->scale);
  p.c[2] = static_cast<int32_t>(terrain->caves);
  p.flags = vx_make_flags(vx::edit::kShapeTerrain, VX_OP_ADD, 0);
  VX_TRY(vx_svo_reset(v, stream));
  VX_TRY_CUDA(cudaMemcpyAsync(v->tmp_prim, &p, sizeof(p), cudaMemcpyHostToDevice, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  return run_pipeline(v, v->tmp_prim, nullptr, 1, s, true);
}

vx_status vx_svo_query(const vx_svo *v, const vx_voxel *pts, uint32_t count,
                       uint8_t *out, vx_stream stream) {
  if (v == nullptr || ((pts == nullptr || out == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("svo_query", s);
  vx_svo_view view;
  VX_TRY(vx_svo_device_view(v, &view));
  query_kernel<<<vx::ceil_div(count, kBlock), kBlock, 0, s>>>(view, pts, count, out);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_svo_collect(vx_svo *v, vx_stream stream) {
  if (v == nullptr) return VX_ERR_INVALID_VALUE;
  const uint32_t grid = static_cast<uint32_t>(vx::sm_count()) *
                        static_cast<uint32_t>(vx::tune::get(vx::tune::kEditBlocksPerSm));
  return launch_collection(v->t, grid, static_cast<cudaStream_t>(stream), true);
}

vx_status vx_svo_get_counters(const vx_svo *v, vx_svo_counters *host, vx_stream stream) {
  if (v == nullptr || host == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Counters c;
  VX_TRY_CUDA(cudaMemcpyAsync(&c, v->t.ctr, sizeof(c), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  // live counts (GpuSvoCounters: allocated high-water and free-stack sizes)
  host->node_count = c.node_count;
  host->leaf_count = c.leaf_count;
  host->free_node_count = c.free_node_count;
  host->free_leaf_count = c.free_leaf_count;
  return VX_OK;
}

vx_status vx_svo_export_canonical(const vx_svo *v, uint32_t *host_node_count,
                                  uint32_t *host_leaf_count, uint32_t *host_nodes,
                                  uint32_t nodes_capacity, uint64_t *host_leaves,
                                  uint8_t *host_materials, uint32_t leaves_capacity,
                                  vx_stream stream) {
  if (v == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Tables &t = v->t;
  Counters c;
  VX_TRY_CUDA(cudaMemcpyAsync(&c, t.ctr, sizeof(c), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> nodes(static_cast<size_t>(c.node_count) * 8);
  std::vector<uint64_t> leaves(c.leaf_count);
  std::vector<uint8_t> mats(t.materials ? static_cast<size_t>(c.leaf_count) * 64 : 0);
  VX_TRY_CUDA(cudaMemcpyAsync(nodes.data(), t.nodes, nodes.size() * 4, cudaMemcpyDeviceToHost, s));
  if (c.leaf_count) {
    VX_TRY_CUDA(cudaMemcpyAsync(leaves.data(), t.leaves, leaves.size() * 8, cudaMemcpyDeviceToHost, s));
    if (t.materials)
      VX_TRY_CUDA(cudaMemcpyAsync(mats.data(), t.mats, mats.size(), cudaMemcpyDeviceToHost, s));
  }
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  // DFS pre-order: node ids on first visit, leaves in visit order.
  std::vector<uint32_t> out_nodes;
  std::vector<uint64_t> out_leaves;
  std::vector<uint8_t> out_mats;
  struct Frame {
    uint32_t node, depth, c, id;
    uint32_t rec[8];
  };
  std::vector<Frame> st;
  auto open = [&](uint32_t node, uint32_t depth) {
    Frame f{};
    f.node = node;
    f.depth = depth;
    f.id = static_cast<uint32_t>(out_nodes.size() / 8);
    out_nodes.resize(out_nodes.size() + 8, 0);
    st.push_back(f);
  };
  open(0, 0);
  while (!st.empty()) {
    Frame &f = st.back();
    if (f.c == 8) {
      std::copy(f.rec, f.rec + 8, out_nodes.begin() + static_cast<size_t>(f.id) * 8);
      const uint32_t id = f.id;
      st.pop_back();
      if (!st.empty()) {
        Frame &p = st.back();
        p.rec[p.c] = kChild | id; // bit 31 of a present child is a don't-care
        ++p.c;
      }
      continue;
    }
    const uint32_t w = nodes[static_cast<size_t>(f.node) * 8 + f.c];
    if (!(w & kChild)) {
      f.rec[f.c++] = w;
    } else if (f.depth + 1 < t.depth) {
      open(w & kIndex, f.depth + 1); // completes when popped
    } else {
      const uint32_t li = w & kIndex;
      f.rec[f.c++] = kChild | static_cast<uint32_t>(out_leaves.size());
      out_leaves.push_back(leaves[li]);
      if (t.materials) out_mats.insert(out_mats.end(), &mats[static_cast<size_t>(li) * 64],
                                       &mats[static_cast<size_t>(li) * 64] + 64);
    }
  }
  const uint32_t nn = static_cast<uint32_t>(out_nodes.size() / 8);
  const uint32_t nl = static_cast<uint32_t>(out_leaves.size());
  if (host_node_count) *host_node_count = nn;
  if (host_leaf_count) *host_leaf_count = nl;
  if (host_nodes) {
    if (nn > nodes_capacity) return VX_ERR_INVALID_VALUE;
    std::copy(out_nodes.begin(), out_nodes.end(), host_nodes);
  }
  if (host_leaves) {
    if (nl > leaves_capacity) return VX_ERR_INVALID_VALUE;
    std::copy(out_leaves.begin(), out_leaves.end(), host_leaves);
  }
  if (host_materials && t.materials) std::copy(out_mats.begin(), out_mats.end(), host_materials);
  return VX_OK;
}

} // extern "C"
