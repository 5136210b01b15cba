// Hash DAG resident on one B200: hash-consed per-level tables, batched
// primitive edits, the plain per-call voxel-list path, terrain builds,
// queries and a canonical dump.
//
// Storage (one table per level):
//   inner level l < depth: a word pool holding items
//       [child_mask | fill_mask << 8, child refs of child_mask in order]
//     (the reference's canonical item, hash_dag_gpu/detail/node.cuh:266-289)
//     and an open-addressing index of 64-bit slots {tag, ref}; ref = word
//     offset + 2.  An insert reserves an empty slot with the busy marker,
//     appends the item to the pool and publishes {tag, ref} with a release
//     store; readers that meet a busy slot with their tag wait (bounded).
//   leaf level: an open-addressing set of the 64-bit masks themselves;
//     ref = slot + 2.  Masks 0 and ~0 are never stored: refs 0 and 1 are the
//     empty / full subtree of any level (hash_dag_gpu/config.cuh:30-37).
// Structural sharing is by content: two equal subtrees of a level always
// have the same ref, so an edit copies only the paths it changes.
#include "edit_common.cuh"
#include "voxel_b200_device.cuh"
#include "graph.cuh"
#include "profile.cuh"
#include "tuning.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <cstdio>
#include <cmath>
#include <new>
#include <vector>

namespace vx::dag {

using namespace vx::edit;

constexpr uint32_t kEmptyRef = 0, kFullRef = 1;
constexpr uint32_t kBusy = 0xffffffffu;
constexpr uint32_t kMaxDepth = 14;
constexpr uint32_t kMaxProbes = 1u << 16;

struct Tables {
  uint32_t depth;
  uint32_t *pool[kMaxDepth];
  uint64_t *index[kMaxDepth];
  uint64_t pool_cap[kMaxDepth];
  uint64_t index_mask[kMaxDepth];
  uint64_t *leaves;
  uint64_t leaf_mask;
  Header *hdr;
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// Hash of an item's n words, fed one word at a time: each word is folded in
// by an xor, a multiply by an odd constant and a rotation (a bijection of
// the state for every word, so items that differ in one word never
// collide), and splitmix64's finaliser spreads the state over all 64 bits.
struct WordHash {
  uint64_t h;
  __device__ __forceinline__ explicit WordHash(uint32_t n) : h(0x243f6a8885a308d3ull ^ n) {}
  __device__ __forceinline__ void add(uint32_t w) {
    const uint64_t x = (h ^ w) * 0x9fb21c651e98df25ull;
    h = (x << 29) | (x >> 35);
  }
  __device__ __forceinline__ uint64_t finish() const { return mix64(h); }
};

__device__ __forceinline__ uint64_t hash_words(const uint32_t *w, uint32_t n) {
  WordHash s(n);
  for (uint32_t i = 0; i < n; ++i) s.add(w[i]);
  return s.finish();
}

// The words of an item as node_find_or_insert sees them: a plain array ...
struct ArrayWords {
  const uint32_t *w;
  uint32_t n;
  __device__ __forceinline__ uint32_t size() const { return n; }
  __device__ __forceinline__ uint64_t hash() const { return hash_words(w, n); }
  __device__ __forceinline__ bool equals(const uint32_t *item) const {
    bool eq = true;
    for (uint32_t i = 0; i < n && eq; ++i) eq = item[i] == w[i];
    return eq;
  }
  __device__ __forceinline__ void write(uint32_t *dst) const {
    for (uint32_t i = 0; i < n; ++i) dst[i] = w[i];
  }
};

// ... or a node's header and its 8 child refs, of which those in the child
// mask follow the header.  Kept in registers: every loop over the children
// unrolls, so no word array goes to local memory.
struct ChildWords {
  uint32_t header; // child_mask | fill_mask << 8
  const uint32_t (&child)[8];
  __device__ __forceinline__ uint32_t size() const { return 1u + __popc(header & 0xffu); }
  __device__ __forceinline__ uint64_t hash() const {
    WordHash s(size());
    s.add(header);
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c)
      if (header & (1u << c)) s.add(child[c]);
    return s.finish();
  }
  __device__ __forceinline__ bool equals(const uint32_t *item) const {
    if (item[0] != header) return false; // equal headers: equal lengths
    bool eq = true;
    uint32_t k = 1;
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c)
      if (header & (1u << c)) eq &= item[k++] == child[c];
    return eq;
  }
  __device__ __forceinline__ void write(uint32_t *dst) const {
    dst[0] = header;
    uint32_t k = 1;
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c)
      if (header & (1u << c)) dst[k++] = child[c];
  }
};

// ------------------------------------------------------------- reading --

__device__ __forceinline__ uint64_t read_leaf(const Tables &t, uint32_t ref) {
  if (ref == kEmptyRef) return 0ull;
  if (ref == kFullRef) return ~0ull;
  return t.leaves[ref - 2];
}

// Child c of the node `ref` at inner level l (refs 0/1 are uniform subtrees);
// the item format is read by voxel_b200_device.cuh's vx_dag_item_child.
__device__ __forceinline__ uint32_t child_ref(const Tables &t, uint32_t l,
                                              uint32_t ref, uint32_t c) {
  if (ref <= kFullRef) return ref;
  return vx_dag_item_child(t.pool[l] + (ref - 2), c);
}

// ---------------------------------------------------------- hash-consing --

__device__ uint32_t leaf_find_or_insert(const Tables &t, uint64_t mask) {
  uint64_t pos = mix64(mask) & t.leaf_mask;
  for (uint32_t probe = 0; probe < kMaxProbes; ++probe) {
    const uint64_t v = ld_relaxed_u64(t.leaves + pos);
    if (v == mask) return static_cast<uint32_t>(pos + 2);
    if (v == 0) {
      const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long *>(t.leaves + pos),
                                     0ull, static_cast<unsigned long long>(mask));
      if (old == 0) {
        warp_count_u64(reinterpret_cast<unsigned long long *>(&t.hdr->node_count[t.depth]));
        return static_cast<uint32_t>(pos + 2);
      }
      if (old == mask) return static_cast<uint32_t>(pos + 2);
    }
    pos = (pos + 1) & t.leaf_mask;
  }
  set_status(&t.hdr->status, kDevCapacity);
  return kEmptyRef;
}

// Probes use relaxed loads.  An item found through a published entry is
// read after an acquire fence only when it was inserted by this edit (its
// offset is at or above pool_mark, the pool use when the edit's inserts
// began): items from earlier launches are visible without one, and most
// matches of an edit are such pre-existing subtrees.  Inserts publish with a
// release store.
// WarpCounters: bump the level's pool and node counters with one atomic per
// warp (warp_atomic_add_small), for kernels whose lanes insert side by side;
// a kernel with a few inserting lanes per warp does better with plain ones.
template <class Words, bool WarpCounters = true>
__device__ uint32_t node_find_or_insert(const Tables &t, uint32_t l, const Words &w,
                                        bool *inserted = nullptr) {
  const uint32_t n = w.size();
  const uint64_t h = w.hash();
  const uint32_t tag = static_cast<uint32_t>(h >> 32) | 1u;
  uint64_t *idx = t.index[l];
  uint32_t *pool = t.pool[l];
  const uint32_t mark = t.hdr->pool_mark[l];
  uint64_t pos = h & t.index_mask[l];
  for (uint32_t probe = 0; probe < kMaxProbes; ++probe) {
    uint64_t v = ld_relaxed_u64(idx + pos);
    if (v == 0) {
      const uint64_t claim = (static_cast<uint64_t>(tag) << 32) | kBusy;
      const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long *>(idx + pos),
                                     0ull, static_cast<unsigned long long>(claim));
      if (old == 0) {
        const uint32_t off = WarpCounters ? warp_atomic_add_small(&t.hdr->pool_used[l], n)
                                          : atomicAdd(&t.hdr->pool_used[l], n);
        if (static_cast<uint64_t>(off) + n > t.pool_cap[l]) {
          set_status(&t.hdr->status, kDevCapacity);
          // Leave a dead entry (ref 1 never matches an item) so waiters move on.
          st_release_u64(idx + pos, (static_cast<uint64_t>(tag) << 32) | kFullRef);
          return kEmptyRef;
        }
        w.write(pool + off);
        st_release_u64(idx + pos, (static_cast<uint64_t>(tag) << 32) | (off + 2u));
        if (WarpCounters)
          warp_count_u64(reinterpret_cast<unsigned long long *>(&t.hdr->node_count[l]));
        else
          atomicAdd(reinterpret_cast<unsigned long long *>(&t.hdr->node_count[l]), 1ull);
        if (inserted) *inserted = true;
        return off + 2u;
      }
      v = old;
    }
    if (static_cast<uint32_t>(v >> 32) == tag) {
      uint32_t r = static_cast<uint32_t>(v);
      if (r == kBusy) {
        const uint64_t t0 = global_ns();
        while (r == kBusy) {
          if (global_ns() - t0 > kWaitLimitNs) {
            set_status(&t.hdr->status, kDevTimeout);
            return kEmptyRef;
          }
          __nanosleep(64);
          r = static_cast<uint32_t>(ld_relaxed_u64(idx + pos));
        }
      }
      if (r >= 2u) {
        if (r - 2u >= mark) fence_acq_rel_gpu(); // inserted by this edit
        if (w.equals(pool + (r - 2u))) return r;
      }
    }
    pos = (pos + 1) & t.index_mask[l];
  }
  set_status(&t.hdr->status, kDevCapacity);
  return kEmptyRef;
}

// Canonical ref of a node given its 8 child refs: uniform nodes collapse to
// the sentinels, everything else is hash-consed into level l's table.
template <bool WarpCounters = true>
__device__ uint32_t canon_node(const Tables &t, uint32_t l,
                               const uint32_t (&child)[8]) {
  uint32_t cm = 0, fm = 0;
#pragma unroll
  for (uint32_t c = 0; c < 8; ++c) {
    const uint32_t r = child[c];
    if (r == kFullRef) fm |= 1u << c;
    else if (r >= 2u) cm |= 1u << c;
  }
  if (cm == 0) {
    if (fm == 0) return kEmptyRef;
    if (fm == 0xffu) return kFullRef;
  }
  return node_find_or_insert<ChildWords, WarpCounters>(t, l, ChildWords{cm | (fm << 8), child});
}

__device__ __forceinline__ uint32_t canon_leaf(const Tables &t, uint64_t mask) {
  if (mask == 0) return kEmptyRef;
  if (mask == ~0ull) return kFullRef;
  return leaf_find_or_insert(t, mask);
}

// ------------------------------------------------------------ pipeline --

struct Ctx {
  Tables t;
  Arena a;
  const vx_primitive *prims;
  const uint32_t *d_prim_count; // device count (NULL: use host_prim_count)
  uint32_t host_prim_count;
};

struct DagTree {
  Tables t;
  static constexpr bool kItemsForConst = false;
  __device__ uint32_t child(uint32_t l, uint32_t ref, uint32_t c) const {
    return child_ref(t, l, ref, c);
  }
  // Superseded subtrees stay in the tables until vx_dag_compact.
  __device__ void replaced(uint32_t, uint32_t, uint32_t) const {}
  template <bool Terrain>
  __device__ uint32_t classify(const vx_primitive &p, uint32_t world_exp,
                               int64_t ox, int64_t oy, int64_t oz, int64_t n) const {
    return vx::edit::classify<Terrain>(p, world_exp, ox, oy, oz, n);
  }
  __device__ uint32_t const_value(const vx_primitive &p, int64_t, int64_t) const {
    return vx_prim_op(&p) == VX_OP_ADD ? kFullRef : kEmptyRef;
  }
};

// pool_mark = pool_used of every level, before the edit inserts anything.
__global__ void mark_pools_kernel(Tables t) {
  if (threadIdx.x < kMaxDepth) t.hdr->pool_mark[threadIdx.x] = t.hdr->pool_used[threadIdx.x];
}

// Level depth - 1: evaluate the 8 leaves of every item and hash-cons the
// item.  Lanes (the tuning knob "edit.leafparent_lanes") threads share an
// item, each evaluating children q + Lanes * j of it (q its rank in the
// group): 8 lanes take one leaf each, 4 lanes two, which halves the
// per-item work that every lane repeats and doubles the items in flight.
// MinBlocks (the knob "edit.leafparent_blocks") trades registers for
// resident blocks: the kernel is bound by chains of dependent loads, so more
// items in flight can outweigh a few spilled values.
__device__ void finish_upwards(const Ctx &x, uint32_t parent, uint32_t l);

// Climb: after storing an item's result, finish its ancestors (the single
// cooperative kernel's bottom-up build, without level barriers).
// Prefetch (the knob "edit.leafparent_prefetch"): beside each item's record,
// load the old ref of the group's next item, and once the current item's old
// leaves are requested, prefetch that next old node into L2, so the next
// iteration's first dependent read (node header and child refs) is an L2 hit
// instead of a DRAM round trip.
template <bool Terrain, uint32_t Lanes, bool Climb = false, bool Prefetch = false>
__device__ __forceinline__ void leafparent_body(Ctx x, Blocks blk) {
  static_assert(Lanes == 2 || Lanes == 4 || Lanes == 8, "2, 4 or 8 lanes per item");
  constexpr uint32_t kPer = 8 / Lanes; // leaves per lane
  constexpr uint32_t kGroupBits = (1u << Lanes) - 1u;
  Header *h = x.t.hdr;
  const uint32_t l = x.t.depth - 1;
  const uint32_t W = h->item_count[l]; // loaded beside the status
  const uint32_t base = h->item_off[l];
  if (edit_failed(h)) return;
  const uint32_t *pairs = x.a.pairs[l & 1u];
  const uint32_t world_exp = x.t.depth + 2;
  const uint32_t lane = lane_id();
  const uint64_t total = static_cast<uint64_t>(W) * Lanes;
  const uint64_t stride = static_cast<uint64_t>(blk.count) * blockDim.x;
  // The item's primitives, Lanes at a time: lane q of the group loads the
  // q-th (one parallel load instead of every lane walking the list).
  __shared__ vx_primitive s_pr[kBlock / Lanes][Lanes];
  const uint32_t grp = threadIdx.x / Lanes;
  const uint32_t gbase = lane & ~(Lanes - 1u);
  const uint32_t gmask = kGroupBits << gbase;
  for (uint64_t g0 = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x - lane;
       g0 < total; g0 += stride) {
    const uint64_t g = g0 + lane;
    const bool have = g < total; // the same for the lanes of a group
    const uint32_t wi = static_cast<uint32_t>(g / Lanes), q = lane & (Lanes - 1u);
    uint32_t result[kPer], old_child[kPer];
#pragma unroll
    for (uint32_t j = 0; j < kPer; ++j) result[j] = old_child[j] = kEmptyRef;
    Item it{};
    uint32_t next_old = kEmptyRef; // Prefetch: the old ref of the group's next item
    if (have) {
      it = x.a.items[base + wi];
      if (Prefetch && q == 0 && g + stride < total)
        next_old = x.a.items[base + static_cast<uint32_t>((g + stride) / Lanes)].old;
      const Cell cell = unpack_cell(it.cell);
      // Independent loads side by side: the first chunk's pair index and the
      // old node, then its primitive and the old leaves (read speculatively:
      // the kernel is bound by dependent round trips, not by bandwidth).
      int64_t ox[kPer], oy[kPer], oz[kPer];
#pragma unroll
      for (uint32_t j = 0; j < kPer; ++j) {
        const uint32_t c = q + Lanes * j;
        ox[j] = int64_t(2 * cell.x + (c & 1u)) * 4;
        oy[j] = int64_t(2 * cell.y + ((c >> 1) & 1u)) * 4;
        oz[j] = int64_t(2 * cell.z + ((c >> 2) & 1u)) * 4;
      }
      const uint32_t n0 = it.pcount < Lanes ? it.pcount : Lanes;
      const uint32_t pidx = q < n0 ? pairs[it.pstart + q] : 0u;
#pragma unroll
      for (uint32_t j = 0; j < kPer; ++j) old_child[j] = child_ref(x.t, l, it.old, q + Lanes * j);
      vx_primitive first{};
      if (q < n0) first = x.prims[pidx];
      uint64_t old_mask[kPer], mask[kPer];
      bool loaded[kPer], touched[kPer];
#pragma unroll
      for (uint32_t j = 0; j < kPer; ++j) {
        old_mask[j] = read_leaf(x.t, old_child[j]);
        mask[j] = 0;
        loaded[j] = touched[j] = false;
      }
      if (Prefetch && next_old > kFullRef) prefetch_l2(x.t.pool[l] + (next_old - 2u));
      __syncwarp(gmask); // the group's previous item no longer reads s_pr
      s_pr[grp][q] = first;
      __syncwarp(gmask);
      for (uint32_t k = 0; k < it.pcount; ++k) {
        if (k % Lanes == 0 && k != 0) {
          __syncwarp(gmask); // the previous chunk is no longer read
          if (k + q < it.pcount) s_pr[grp][q] = x.prims[pairs[it.pstart + k + q]];
          __syncwarp(gmask);
        }
        const vx_primitive &pr = s_pr[grp][k % Lanes]; // read in place: fewer registers
        const bool add = vx_prim_op(&pr) == VX_OP_ADD;
#pragma unroll
        for (uint32_t j = 0; j < kPer; ++j) {
          const uint32_t cls = classify<Terrain>(pr, world_exp, ox[j], oy[j], oz[j], 4);
          if (cls == VX_CELL_EMPTY) continue;
          touched[j] = true;
          if (cls == VX_CELL_FULL) {
            mask[j] = add ? ~0ull : 0ull;
            loaded[j] = true;
            continue;
          }
          if (!loaded[j]) {
            mask[j] = old_mask[j];
            loaded[j] = true;
          }
          const uint64_t m = leaf_mask<Terrain>(pr, world_exp, ox[j], oy[j], oz[j]);
          mask[j] = add ? (mask[j] | m) : (mask[j] & ~m);
        }
      }
      // An unchanged mask keeps its canonical ref: no probe of the leaf set.
#pragma unroll
      for (uint32_t j = 0; j < kPer; ++j)
        result[j] = (touched[j] && mask[j] != old_mask[j]) ? canon_leaf(x.t, mask[j])
                                                           : old_child[j];
    }
    // A node whose 8 children all kept their refs is the old node itself
    // (refs are canonical), so its hash-consing is skipped.
    bool mine_changed = false;
#pragma unroll
    for (uint32_t j = 0; j < kPer; ++j) mine_changed |= result[j] != old_child[j];
    const uint32_t changed = __ballot_sync(kFullMask, mine_changed);
    const bool same = ((changed >> gbase) & kGroupBits) == 0u;
    uint32_t child[8];
#pragma unroll
    for (uint32_t j = 0; j < kPer; ++j)
#pragma unroll
      for (uint32_t k = 0; k < Lanes; ++k)
        child[k + Lanes * j] = __shfl_sync(kFullMask, result[j], gbase + k);
    // At most 32 / Lanes lanes of a warp insert a node here: plain counters.
    if (have && q == 0) {
      x.a.items[base + wi].result = same ? it.old : canon_node<false>(x.t, l, child);
      if (Climb) finish_upwards(x, it.result, l); // it.result: the parent's index
    }
  }
}

template <bool Terrain, int MinBlocks, uint32_t Lanes, bool Prefetch = false>
__global__ void __launch_bounds__(kBlock, MinBlocks) leafparent_kernel(Ctx x) {
  leafparent_body<Terrain, Lanes, false, Prefetch>(x, launch_blocks());
}

// The rebuilt ref of one item at inner level l from its children's results.
// WarpCounters: the pool and node counters are bumped once per warp, which
// needs every active lane of the warp at the same level (true for the
// level-by-level build, not for climbs, where lanes may be at any level).
// Climb: the children's results come from L2 (other SMs wrote them in this
// launch); the level-by-level build reads them in a later launch.
template <bool WarpCounters = true, bool Climb = false>
__device__ __forceinline__ uint32_t build_item(const Ctx &x, uint32_t l, const Item &it) {
  const uint32_t cm = it.masks & 0xffu, km = (it.masks >> 8) & 0xffu,
                 kf = (it.masks >> 16) & 0xffu;
  uint32_t child[8];
  uint32_t k = 0;
#pragma unroll
  for (uint32_t c = 0; c < 8; ++c) {
    const uint32_t bit = 1u << c;
    if (cm & bit) {
      const uint32_t *r = &x.a.items[it.child_base + k++].result;
      child[c] = Climb ? __ldcg(r) : *r;
    } else if (km & bit) {
      child[c] = (kf & bit) ? kFullRef : kEmptyRef;
    }
    else child[c] = child_ref(x.t, l, it.old, c);
  }
  // Every child kept its ref: the node is the old one (refs are canonical).
  bool same = true;
#pragma unroll
  for (uint32_t c = 0; c < 8; ++c)
    if ((cm | km) & (1u << c)) same = same && child[c] == child_ref(x.t, l, it.old, c);
  return same ? it.old : canon_node<WarpCounters>(x.t, l, child);
}

__device__ __forceinline__ void build_body(Ctx x, uint32_t l, Blocks blk) {
  Header *h = x.t.hdr;
  const uint32_t W = h->item_count[l]; // loaded beside the status
  const uint32_t base = h->item_off[l];
  if (edit_failed(h)) return;
  for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < W; i += static_cast<uint64_t>(blk.count) * blockDim.x)
    x.a.items[base + i].result = build_item(x, l, x.a.items[base + i]);
}

// Bottom-up without level barriers: an item at level l has just stored its
// result; count it off its parent's pending children with one
// acquire-release decrement (its result store is published, and the last
// child sees every sibling's), and when it was the last one rebuild the parent
// and go on up.
__device__ void finish_upwards(const Ctx &x, uint32_t parent, uint32_t l) {
  while (parent != kNoParent) {
    // The parent's own fields were written by its expansion, stages ago:
    // read them while the decrement is in flight (only the children's
    // results need its acquire).
    const Item it = load_item_l2(&x.a.items[parent]);
    if (atomic_sub_acq_rel(&x.a.items[parent].pstart, 1u) != 1u) return;
    --l;
    x.a.items[parent].result = build_item<false, true>(x, l, it);
    parent = it.result; // the grandparent, stored there until now
  }
}

// Items below the leaf-parent level with no child items (every child
// unchanged or uniform) have nothing to wait for: they rebuild at once and
// start their own climb.
__device__ __forceinline__ void rebuild_childless_body(Ctx x, Blocks blk) {
  Header *h = x.t.hdr;
  // every level's counts in one round trip
  __shared__ uint32_t s_w[kMaxDepth], s_base[kMaxDepth];
  if (threadIdx.x < kMaxDepth) {
    s_w[threadIdx.x] = h->item_count[threadIdx.x];
    s_base[threadIdx.x] = h->item_off[threadIdx.x];
  }
  if (edit_failed(h)) return; // (its barrier also publishes s_w, s_base)
  for (uint32_t l = 0; l + 1 < x.t.depth; ++l) {
    const uint32_t W = s_w[l];
    const uint32_t base = s_base[l];
    for (uint64_t i = blk.id * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
         i < W; i += static_cast<uint64_t>(blk.count) * blockDim.x) {
      const Item it = x.a.items[base + i];
      if (it.masks & 0xffu) continue;
      x.a.items[base + i].result = build_item<false, true>(x, l, it);
      finish_upwards(x, it.result, l);
    }
  }
}

__global__ void __launch_bounds__(kBlock) build_kernel(Ctx x, uint32_t l) {
  build_body(x, l, launch_blocks());
}

__global__ void publish_kernel(Ctx x) {
  Header *h = x.t.hdr;
  if (h->status == kDevOk && h->item_count[0] == 1) h->root = x.a.items[0].result;
}

// A whole edit in one cooperative launch, the stages separated by grid-wide
// barriers instead of kernel boundaries: for small batches, where the ~37
// launches of the level-synchronous pipeline (and their mostly idle grids)
// cost more than the work.  The stages are the kernels' own bodies; long
// primitive lists are expanded block by block with a 256-thread block and a
// 4 KiB classification cache (lists beyond it are classified again).
// Requires every block of the grid to be resident (cudaLaunchCooperativeKernel
// checks it).
constexpr uint32_t kSmallBigCache = 4096;

// With Plain, the edit's input is a voxel list (one op): the first stages
// turn it into leaf-mask primitives (PlainPrep) in place of the sort-based
// preparation of the multi-launch path.
// One block per SM runs it, so it may take up to 255 registers (the
// default cap for 256-thread blocks, 128, made it spill).
template <uint32_t Lanes, bool Plain>
__global__ void __maxnreg__(255) small_edit_kernel(Ctx x, EditCtx e, PlainPrep prep,
                                                            uint32_t *status_out) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const Blocks blk = launch_blocks();
  const DagTree tree{x.t};
  if (Plain) {
    plain_prep_clear(prep, blk);
    grid.sync();
    plain_prep_aggregate(prep, x.t.depth, blk);
    grid.sync();
    plain_prep_fill(prep, blk); // beside init: both need only the final count
  }
  init_body(e, kUseHeaderRoot, blk);
  // pool_mark: nothing is inserted before the leaf-parent level
  if (blk.id == 0 && threadIdx.x < kMaxDepth)
    x.t.hdr->pool_mark[threadIdx.x] = x.t.hdr->pool_used[threadIdx.x];
  grid.sync();
  for (uint32_t l = 0; l + 1 < x.t.depth; ++l) {
    // Short and long lists of level l side by side, one barrier per level:
    // the long ones were listed when level l was emitted (their count is
    // final at the barrier before, the same in every block) and go to the
    // blocks from the last one down, the short ones from block 0 up.
    expand_body<DagTree, false>(e, tree, l, blk);
    if (x.t.hdr->big_count[l] != 0)
      expand_big_body<DagTree, false, kBlock, kSmallBigCache>(e, tree, l,
                                                          Blocks{blk.count - 1u - blk.id, blk.count});
    grid.sync();
  }
  // The bottom-up build without level barriers: the leaf-parent items and
  // the childless items of the levels above finish their ancestors, each
  // item rebuilt by the last of its children to finish.
  leafparent_body<false, Lanes, true>(x, blk);
  rebuild_childless_body(x, blk);
  grid.sync();
  if (blk.id == 0 && threadIdx.x == 0) {
    Header *h = x.t.hdr;
    if (h->status == kDevOk && h->item_count[0] == 1) h->root = x.a.items[0].result;
    if (status_out) *status_out = h->status; // the caller's mapped host word
  }
}

__global__ void query_kernel(vx_dag_view v, const vx_voxel *pts, uint32_t n,
                             uint8_t *out) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const vx_voxel p = pts[i];
  out[i] = vx_dag_get_voxel(v, p.x, p.y, p.z);
}

__global__ void raycast_kernel(vx_dag_view v, const vx_ray *rays, uint32_t n,
                               vx_ray_hit *hits) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  hits[i] = vx_dag_raycast(v, rays[i]);
}

__global__ void read_leaves_kernel(vx_dag_view v, uint32_t lx0, uint32_t ly0, uint32_t lz0,
                                   uint32_t nx, uint32_t ny, uint32_t n, uint64_t *out) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = static_cast<uint32_t>(i % nx), y = static_cast<uint32_t>((i / nx) % ny),
                 z = static_cast<uint32_t>(i / (uint64_t(nx) * ny));
  out[i] = vx_dag_get_leaf(v, lx0 + x, ly0 + y, lz0 + z);
}

// ------------------------------------------------------- plain path prep --

// Voxel -> (leaf key, bit).  The key is the leaf's Morton path, 3 bits per
// inner level with the root's child in the top bits (the reference's
// make_leaf_key, hash_dag_gpu/detail/node.cuh:67-85, widened to 64 bits);
// voxels outside the world get key 1 << (3 * depth) and are dropped.
__global__ void pack_voxels_kernel(const vx_voxel *v, uint32_t n, uint32_t depth,
                                   uint64_t *keys, uint32_t *bits) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const vx_voxel p = v[i];
  const uint32_t side_exp = depth + 2;
  if ((p.x >> side_exp) | (p.y >> side_exp) | (p.z >> side_exp)) {
    keys[i] = 1ull << (3 * depth);
    bits[i] = 0;
    return;
  }
  uint64_t key = 0;
  for (uint32_t l = 0; l < depth; ++l) {
    const uint32_t s = side_exp - 1 - l;
    key = (key << 3) | (((p.x >> s) & 1u) | (((p.y >> s) & 1u) << 1) | (((p.z >> s) & 1u) << 2));
  }
  keys[i] = key;
  bits[i] = (p.x & 3u) + 4u * (p.y & 3u) + 16u * (p.z & 3u);
}

__global__ void run_flags_kernel(const uint64_t *keys, uint32_t n, uint32_t depth,
                                 uint32_t *flags) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const bool valid = keys[i] < (1ull << (3 * depth));
  flags[i] = (valid && (i == 0 || keys[i - 1] != keys[i])) ? 1u : 0u;
}

// Leaf edit command -> (leaf key, command index); leaves outside the world
// get key 1 << (3 * depth) and are dropped.
__global__ void pack_leaf_commands_kernel(const vx_leaf_command *c, uint32_t n, uint32_t depth,
                                          uint64_t *keys, uint32_t *index) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const vx_leaf_command cmd = c[i];
  index[i] = static_cast<uint32_t>(i);
  if ((cmd.leaf_x >> depth) | (cmd.leaf_y >> depth) | (cmd.leaf_z >> depth)) {
    keys[i] = 1ull << (3 * depth);
    return;
  }
  uint64_t key = 0;
  for (uint32_t l = 0; l < depth; ++l) {
    const uint32_t s = depth - 1 - l;
    key = (key << 3) | (((cmd.leaf_x >> s) & 1u) | (((cmd.leaf_y >> s) & 1u) << 1) |
                        (((cmd.leaf_z >> s) & 1u) << 2));
  }
  keys[i] = key;
}

// Each run start ORs its run's voxel bits (a voxel list) or its commands'
// masks (leaf edit commands, selected by index) into one leaf-mask primitive.
template <bool Commands>
__global__ void reduce_runs_kernel(const uint64_t *keys, const uint32_t *bits,
                                   const vx_leaf_command *cmds,
                                   const uint32_t *offsets, uint32_t n,
                                   uint32_t depth, uint32_t op, uint32_t material,
                                   vx_primitive *out, uint32_t *out_count) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const uint64_t key = keys[i];
  const bool valid = key < (1ull << (3 * depth));
  const bool start = valid && (i == 0 || keys[i - 1] != key);
  if (start) {
    uint64_t mask = 0;
    for (uint64_t j = i; j < n && keys[j] == key; ++j) {
      if constexpr (Commands) {
        const vx_leaf_command &c = cmds[bits[j]];
        mask |= static_cast<uint64_t>(c.voxel_data_low) |
                (static_cast<uint64_t>(c.voxel_data_high) << 32);
      } else {
        mask |= 1ull << bits[j];
      }
    }
    uint32_t lx = 0, ly = 0, lz = 0;
    for (uint32_t l = 0; l < depth; ++l) {
      const uint32_t c = static_cast<uint32_t>(key >> (3 * (depth - 1 - l))) & 7u;
      lx = (lx << 1) | (c & 1u);
      ly = (ly << 1) | ((c >> 1) & 1u);
      lz = (lz << 1) | ((c >> 2) & 1u);
    }
    vx_primitive p{};
    p.c[0] = static_cast<int32_t>(lx * 4);
    p.c[1] = static_cast<int32_t>(ly * 4);
    p.c[2] = static_cast<int32_t>(lz * 4);
    p.r[0] = static_cast<uint32_t>(mask);
    p.r[1] = static_cast<uint32_t>(mask >> 32);
    p.flags = vx_make_flags(kShapeLeafMask, op, material);
    out[offsets[i]] = p;
  }
  if (i == n - 1) *out_count = offsets[i] + (start ? 1u : 0u);
}

} // namespace vx::dag

// ================================================================ handle ==

struct vx_dag {
  vx::dag::Tables t{};
  vx::edit::Arena a{};
  uint64_t index_slots[vx::dag::kMaxDepth] = {};
  uint64_t leaf_slots = 0;
  void *arena_mem = nullptr;
  size_t bytes = 0;
  vx_primitive *tmp_prim = nullptr; // one terrain primitive
  uint32_t *host_status = nullptr;  // pinned word for status reads (allocated on first use)
  uint32_t *status_alias = nullptr; // its device address, when mapped at creation
};

namespace vx::dag {

inline uint64_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// The single cooperative launch of small_edit_kernel, on as many blocks as
// are resident at once (at most the edit.small_blocks_per_sm knob per SM).
// Resident blocks per SM of small_edit_kernel<2 / 4 / 8 lanes, plain or
// not>, queried once (at DAG creation, so never first inside a stream
// capture).
void *small_kernel(int64_t lanes, bool plain) {
  if (plain)
    return lanes == 2   ? reinterpret_cast<void *>(&small_edit_kernel<2, true>)
           : lanes == 4 ? reinterpret_cast<void *>(&small_edit_kernel<4, true>)
                        : reinterpret_cast<void *>(&small_edit_kernel<8, true>);
  return lanes == 2   ? reinterpret_cast<void *>(&small_edit_kernel<2, false>)
         : lanes == 4 ? reinterpret_cast<void *>(&small_edit_kernel<4, false>)
                      : reinterpret_cast<void *>(&small_edit_kernel<8, false>);
}
int g_small_resident[6] = {-1, -1, -1, -1, -1, -1};
inline int small_slot(int64_t lanes, bool plain) {
  return (lanes == 2 ? 0 : (lanes == 4 ? 1 : 2)) + (plain ? 3 : 0);
}
vx_status query_small_residency() {
  const int64_t lanes[3] = {2, 4, 8};
  for (int plain = 0; plain < 2; ++plain)
    for (int i = 0; i < 3; ++i) {
      int &slot = g_small_resident[small_slot(lanes[i], plain != 0)];
      if (slot >= 0) continue;
      int n = 0;
      VX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &n, small_kernel(lanes[i], plain != 0), kBlock, 0));
      slot = n;
    }
  return VX_OK;
}

// status_out: a mapped host word the kernel's last act writes the status to.
vx_status run_small(vx_dag *d, Ctx &x, const EditCtx &e, cudaStream_t s,
                    const PlainPrep *prep = nullptr, uint32_t *status_out = nullptr) {
  const int64_t lanes = tune::get(tune::kEditLeafparentLanes);
  void *fn = small_kernel(lanes, prep != nullptr);
  VX_TRY(query_small_residency());
  const int per_sm = g_small_resident[small_slot(lanes, prep != nullptr)];
  const int want = static_cast<int>(tune::get(tune::kEditSmallBlocksPerSm));
  const uint32_t grid = static_cast<uint32_t>(sm_count()) *
                        static_cast<uint32_t>(std::max(1, std::min(per_sm, want)));
  if (per_sm < 1) return VX_ERR_INVALID_VALUE;
  EditCtx ec = e;
  PlainPrep pp = prep ? *prep : PlainPrep{};
  void *args[] = {&x, &ec, &pp, &status_out};
  prof::Scope sc("dag_small_edit", s);
  VX_TRY_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, 0, s));
  (void)d;
  return VX_OK;
}

// Small edits (by the edit.small_max_* knobs) run as one cooperative kernel:
// a batch of primitives by its count, a voxel list or leaf commands (one
// leaf-mask primitive per touched leaf) by its length.
inline bool small_batch(uint32_t n, bool voxel_list) {
  return n <= static_cast<uint32_t>(tune::get(voxel_list ? tune::kEditSmallMaxVoxels
                                                         : tune::kEditSmallMaxPrims));
}

vx_status run_pipeline(vx_dag *d, const vx_primitive *prims,
                       const uint32_t *d_count, uint32_t host_count,
                       cudaStream_t s, bool terrain = false,
                       uint32_t blocks_per_sm = 0 /* 0: the edit.blocks_per_sm knob */,
                       int small = -1 /* -1: by host_count as a primitive batch */) {
  Ctx x{d->t, d->a, prims, d_count, host_count};
  const EditCtx e{d->t.hdr, d->a, prims, d_count, host_count, d->t.depth,
                  static_cast<uint32_t>(tune::get(tune::kEditBigItem))};
  const uint32_t depth = d->t.depth;
  const uint32_t grid = static_cast<uint32_t>(sm_count()) *
                        (blocks_per_sm ? blocks_per_sm
                                       : static_cast<uint32_t>(tune::get(tune::kEditBlocksPerSm)));
  if (!terrain && (small < 0 ? small_batch(host_count, false) : small != 0))
    return run_small(d, x, e, s);
  {
    prof::Scope sc("dag_init", s);
    init_kernel<<<std::min<uint32_t>(grid, ceil_div(std::max(host_count, 1u), kBlock) + 1),
                  kBlock, 0, s>>>(e, kUseHeaderRoot);
  }
  VX_TRY_CUDA(cudaGetLastError());
  DagTree tree{d->t};
  for (uint32_t l = 0; l + 1 < depth; ++l) {
    {
      prof::Scope sc("dag_expand", s);
      if (terrain)
        expand_kernel<DagTree, true><<<grid, kBlock, 0, s>>>(e, tree, l);
      else
        expand_kernel<DagTree, false><<<grid, kBlock, 0, s>>>(e, tree, l);
    }
    VX_TRY_CUDA(cudaGetLastError());
    {
      prof::Scope sc("dag_expand_big", s);
      if (terrain)
        expand_big_kernel<DagTree, true><<<sm_count() * 2, kBlock, 0, s>>>(e, tree, l);
      else
        expand_big_kernel<DagTree, false><<<sm_count(), kBigBlock, 0, s>>>(e, tree, l);
    }
    VX_TRY_CUDA(cudaGetLastError());
  }
  {
    prof::Scope sc("dag_mark_pools", s);
    mark_pools_kernel<<<1, 32, 0, s>>>(d->t);
  }
  VX_TRY_CUDA(cudaGetLastError());
  {
    prof::Scope sc("dag_leafparent", s);
    const int64_t lb = tune::get(tune::kEditLeafparentBlocks);
    const int64_t lanes = tune::get(tune::kEditLeafparentLanes);
    const bool four = lanes == 4;
    const bool prefetch = tune::get(tune::kEditLeafparentPrefetch) != 0;
    if (terrain)
      leafparent_kernel<true, 4, 8><<<grid, kBlock, 0, s>>>(x);
    else if (four && prefetch && lb == 6)
      leafparent_kernel<false, 6, 4, true><<<grid, kBlock, 0, s>>>(x);
    else if (four && prefetch && lb == 5)
      leafparent_kernel<false, 5, 4, true><<<grid, kBlock, 0, s>>>(x);
    else if (four && prefetch)
      leafparent_kernel<false, 4, 4, true><<<grid, kBlock, 0, s>>>(x);
    else if (lanes == 2 && lb == 6)
      leafparent_kernel<false, 6, 2><<<grid, kBlock, 0, s>>>(x);
    else if (lanes == 2 && lb == 5)
      leafparent_kernel<false, 5, 2><<<grid, kBlock, 0, s>>>(x);
    else if (lanes == 2)
      leafparent_kernel<false, 4, 2><<<grid, kBlock, 0, s>>>(x);
    else if (four && lb == 6)
      leafparent_kernel<false, 6, 4><<<grid, kBlock, 0, s>>>(x);
    else if (four && lb == 5)
      leafparent_kernel<false, 5, 4><<<grid, kBlock, 0, s>>>(x);
    else if (four)
      leafparent_kernel<false, 4, 4><<<grid, kBlock, 0, s>>>(x);
    else if (lb == 6)
      leafparent_kernel<false, 6, 8><<<grid, kBlock, 0, s>>>(x);
    else if (lb == 5)
      leafparent_kernel<false, 5, 8><<<grid, kBlock, 0, s>>>(x);
    else
      leafparent_kernel<false, 4, 8><<<grid, kBlock, 0, s>>>(x);
  }
  VX_TRY_CUDA(cudaGetLastError());
  for (uint32_t r = depth - 1; r > 0; --r) {
    prof::Scope sc("dag_build", s);
    build_kernel<<<grid, kBlock, 0, s>>>(x, r - 1);
    VX_TRY_CUDA(cudaGetLastError());
  }
  {
    prof::Scope sc("dag_publish", s);
    publish_kernel<<<1, 1, 0, s>>>(x);
  }
  return from_cuda(cudaGetLastError());
}

// The device status, read through a pinned word (a copy into pageable
// memory goes through a staging buffer); a failed status is cleared.
vx_status read_status(vx_dag *d, cudaStream_t s, bool clear) {
  if (d->host_status == nullptr &&
      cudaHostAlloc(reinterpret_cast<void **>(&d->host_status), sizeof(uint32_t),
                    cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError(); // not fatal: read through a stack word instead
    d->host_status = nullptr;
  }
  uint32_t stack_code = 0;
  uint32_t *code = d->host_status ? d->host_status : &stack_code;
  VX_TRY_CUDA(cudaMemcpyAsync(code, &d->t.hdr->status, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  const uint32_t c = *code;
  if (clear && c != kDevOk) {
    VX_TRY_CUDA(cudaMemsetAsync(&d->t.hdr->status, 0, sizeof(uint32_t), s));
    VX_TRY_CUDA(cudaStreamSynchronize(s));
  }
  return status_from_device(c);
}

// The status a small kernel wrote into the mapped host word (set to
// kStatusUnset before the launch): after the kernel there is no copy to
// wait for.  A word the kernel did not write falls back to read_status.
constexpr uint32_t kStatusUnset = 0xffffffffu;
vx_status read_written_status(vx_dag *d, cudaStream_t s) {
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  const uint32_t c = *reinterpret_cast<volatile uint32_t *>(d->host_status);
  if (c == kStatusUnset) return read_status(d, s, true);
  if (c != kDevOk) {
    VX_TRY_CUDA(cudaMemsetAsync(&d->t.hdr->status, 0, sizeof(uint32_t), s));
    VX_TRY_CUDA(cudaStreamSynchronize(s));
  }
  return status_from_device(c);
}

struct PlainLayout {
  uint64_t *keys;
  uint32_t *bits;
  uint32_t *offsets;
  vx_primitive *prims;
  uint32_t *count;
  void *sort_ws;
  size_t sort_ws_bytes;
  void *scan_ws;
  size_t scan_ws_bytes;
};

template <class C> PlainLayout plain_layout(C &c, uint32_t n) {
  PlainLayout p{};
  p.keys = c.template take<uint64_t>(n);
  p.bits = c.template take<uint32_t>(n);
  p.offsets = c.template take<uint32_t>(n);
  p.prims = c.template take<vx_primitive>(n);
  p.count = c.template take<uint32_t>(1);
  p.sort_ws_bytes = vx_sort_workspace_size(n, 8);
  p.sort_ws = c.template take<char>(p.sort_ws_bytes);
  p.scan_ws_bytes = vx_scan_workspace_size(n);
  p.scan_ws = c.template take<char>(p.scan_ws_bytes);
  return p;
}

struct NullCarver {
  size_t offset = 0;
  template <class T> T *take(size_t count) {
    offset = align_up(offset, 256);
    offset += count * sizeof(T);
    return nullptr;
  }
};

} // namespace vx::dag

namespace vx::plain {

size_t workspace_size(uint32_t count) {
  if (count == 0) return 0;
  vx::dag::NullCarver c;
  vx::dag::plain_layout(c, count);
  return c.offset;
}

// Voxel list -> one leaf-mask primitive per touched leaf (op, material),
// written into the workspace; *out_prims / *out_count point into it.
vx_status prepare(const vx_voxel *edits, uint32_t count, uint32_t depth,
                  uint32_t op, uint32_t material, void *workspace,
                  const vx_primitive **out_prims, const uint32_t **out_count,
                  cudaStream_t s) {
  using namespace vx::dag;
  vx::Carver c(workspace);
  const PlainLayout p = plain_layout(c, count);
  const uint32_t blocks = vx::ceil_div(count, kBlock);
  {
    vx::prof::Scope sc("plain_pack_voxels", s);
    pack_voxels_kernel<<<blocks, kBlock, 0, s>>>(edits, count, depth, p.keys, p.bits);
  }
  VX_TRY_CUDA(cudaGetLastError());
  VX_TRY(vx_sort_pairs_u64(p.keys, p.bits, count, 3 * depth + 1, p.sort_ws,
                           p.sort_ws_bytes, s));
  {
    vx::prof::Scope sc("plain_run_flags", s);
    run_flags_kernel<<<blocks, kBlock, 0, s>>>(p.keys, count, depth, p.offsets);
  }
  VX_TRY_CUDA(cudaGetLastError());
  VX_TRY(vx_scan_exclusive_sum_u32(p.offsets, count, p.scan_ws, p.scan_ws_bytes, s));
  {
    vx::prof::Scope sc("plain_reduce_runs", s);
    reduce_runs_kernel<false><<<blocks, kBlock, 0, s>>>(p.keys, p.bits, nullptr, p.offsets,
                                                        count, depth, op, material, p.prims,
                                                        p.count);
  }
  VX_TRY_CUDA(cudaGetLastError());
  *out_prims = p.prims;
  *out_count = p.count;
  return VX_OK;
}

// Leaf edit commands -> one leaf-mask primitive per named leaf, the masks of
// commands naming the same leaf OR-merged (the engine's merge_commands).
vx_status prepare_leaf_commands(const vx_leaf_command *cmds, uint32_t count, uint32_t depth,
                                uint32_t op, uint32_t material, void *workspace,
                                const vx_primitive **out_prims, const uint32_t **out_count,
                                cudaStream_t s) {
  using namespace vx::dag;
  vx::Carver c(workspace);
  const PlainLayout p = plain_layout(c, count);
  const uint32_t blocks = vx::ceil_div(count, kBlock);
  {
    vx::prof::Scope sc("plain_pack_leaf_commands", s);
    pack_leaf_commands_kernel<<<blocks, kBlock, 0, s>>>(cmds, count, depth, p.keys, p.bits);
  }
  VX_TRY_CUDA(cudaGetLastError());
  VX_TRY(vx_sort_pairs_u64(p.keys, p.bits, count, 3 * depth + 1, p.sort_ws,
                           p.sort_ws_bytes, s));
  {
    vx::prof::Scope sc("plain_run_flags", s);
    run_flags_kernel<<<blocks, kBlock, 0, s>>>(p.keys, count, depth, p.offsets);
  }
  VX_TRY_CUDA(cudaGetLastError());
  VX_TRY(vx_scan_exclusive_sum_u32(p.offsets, count, p.scan_ws, p.scan_ws_bytes, s));
  {
    vx::prof::Scope sc("plain_reduce_runs", s);
    reduce_runs_kernel<true><<<blocks, kBlock, 0, s>>>(p.keys, p.bits, cmds, p.offsets, count,
                                                       depth, op, material, p.prims, p.count);
  }
  VX_TRY_CUDA(cudaGetLastError());
  *out_prims = p.prims;
  *out_count = p.count;
  return VX_OK;
}

} // namespace vx::plain

using namespace vx::dag;

extern "C" {

vx_status vx_dag_create(const vx_dag_config *cfg, vx_dag **out) {
  if (cfg == nullptr || out == nullptr || cfg->depth < 1 || cfg->depth > kMaxDepth ||
      cfg->max_nodes < 16)
    return VX_ERR_INVALID_VALUE;
  int devs = 0;
  if (cudaGetDeviceCount(&devs) != cudaSuccess || devs == 0) return VX_ERR_NO_DEVICE;
  auto *d = new (std::nothrow) vx_dag;
  if (d == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  d->t.depth = cfg->depth;
  auto fail = [&](cudaError_t e) {
    vx_dag_destroy(d);
    return vx::from_cuda(e);
  };
  cudaError_t e;
  for (uint32_t l = 0; l < cfg->depth; ++l) {
    // Level l holds at most 8^l live nodes, plus superseded ones from earlier
    // edits: every edit copies the path above what it changes, so the small
    // levels fill with garbage first. They keep room for max(2^20,
    // max_nodes / 16) items, which sets how often a long-running editor
    // (the serving loop) has to compact.
    const double live = l < 21 ? std::pow(8.0, static_cast<double>(l)) : 1e30;
    const uint64_t floor_cap = std::max<uint64_t>(1u << 20, cfg->max_nodes / 16);
    const uint64_t cap = std::min<uint64_t>(
        cfg->max_nodes, std::max<uint64_t>(floor_cap, static_cast<uint64_t>(std::min(live * 4, 1e18))));
    d->index_slots[l] = next_pow2(cap * 2);
    d->t.index_mask[l] = d->index_slots[l] - 1;
    d->t.pool_cap[l] = std::min<uint64_t>(cap * 6, 0xfffffff0ull);
    if ((e = cudaMalloc(&d->t.index[l], d->index_slots[l] * 8)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&d->t.pool[l], d->t.pool_cap[l] * 4)) != cudaSuccess) return fail(e);
    d->bytes += d->index_slots[l] * 8 + d->t.pool_cap[l] * 4;
  }
  d->leaf_slots = next_pow2(cfg->max_nodes * 2);
  d->t.leaf_mask = d->leaf_slots - 1;
  if ((e = cudaMalloc(&d->t.leaves, d->leaf_slots * 8)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&d->t.hdr, sizeof(vx::edit::Header))) != cudaSuccess) return fail(e);
  // the status word, mapped so that a small kernel can write it directly
  if (cudaHostAlloc(reinterpret_cast<void **>(&d->host_status), sizeof(uint32_t),
                    cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void **>(&d->status_alias), d->host_status,
                               0) != cudaSuccess) {
    cudaGetLastError(); // not fatal: statuses are then copied
    d->status_alias = nullptr;
  }
  if ((e = cudaMalloc(&d->tmp_prim, sizeof(vx_primitive))) != cudaSuccess) return fail(e);
  d->bytes += d->leaf_slots * 8;
  if (vx_status qs = vx::dag::query_small_residency(); qs != VX_OK) {
    vx_dag_destroy(d);
    return qs;
  }
  const uint64_t arena = cfg->arena_bytes ? cfg->arena_bytes : (512ull << 20);
  if ((e = cudaMalloc(&d->arena_mem, arena)) != cudaSuccess) return fail(e);
  d->bytes += arena;
  // Items take 60 % of the arena, the two pair buffers the rest; every
  // sub-buffer starts on a 256-byte boundary.
  const uint64_t big_bytes = std::min<uint64_t>(arena / 64, 4ull << 20) / 256 * 256;
  const uint64_t item_bytes = (arena - big_bytes) / 10 * 6 / 256 * 256;
  d->a.items = static_cast<vx::edit::Item *>(d->arena_mem);
  d->a.item_cap = static_cast<uint32_t>(std::min<uint64_t>(item_bytes / sizeof(vx::edit::Item), 0xffffffffull));
  const uint64_t pair_bytes = (arena - big_bytes - item_bytes) / 2 / 256 * 256;
  d->a.big = reinterpret_cast<uint32_t *>(static_cast<char *>(d->arena_mem) + item_bytes + 2 * pair_bytes);
  d->a.big_cap = static_cast<uint32_t>(big_bytes / 4);
  d->a.pairs[0] = reinterpret_cast<uint32_t *>(static_cast<char *>(d->arena_mem) + item_bytes);
  d->a.pairs[1] = reinterpret_cast<uint32_t *>(static_cast<char *>(d->arena_mem) + item_bytes + pair_bytes);
  d->a.pair_cap = static_cast<uint32_t>(std::min<uint64_t>(pair_bytes / 4, 0xffffffffull));
  const vx_status st = vx_dag_reset(d, nullptr);
  if (st != VX_OK) {
    vx_dag_destroy(d);
    return st;
  }
  if ((e = cudaStreamSynchronize(nullptr)) != cudaSuccess) return fail(e);
  *out = d;
  return VX_OK;
}

vx_status vx_dag_destroy(vx_dag *d) {
  if (d == nullptr) return VX_ERR_INVALID_VALUE;
  for (uint32_t l = 0; l < kMaxDepth; ++l) {
    cudaFree(d->t.index[l]);
    cudaFree(d->t.pool[l]);
  }
  cudaFree(d->t.leaves);
  cudaFree(d->t.hdr);
  cudaFree(d->arena_mem);
  cudaFree(d->tmp_prim);
  if (d->host_status) cudaFreeHost(d->host_status);
  delete d;
  return VX_OK;
}

vx_status vx_dag_reset(vx_dag *d, vx_stream stream) {
  if (d == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (uint32_t l = 0; l < d->t.depth; ++l)
    VX_TRY_CUDA(cudaMemsetAsync(d->t.index[l], 0, d->index_slots[l] * 8, s));
  VX_TRY_CUDA(cudaMemsetAsync(d->t.leaves, 0, d->leaf_slots * 8, s));
  VX_TRY_CUDA(cudaMemsetAsync(d->t.hdr, 0, sizeof(vx::edit::Header), s));
  return VX_OK;
}

uint32_t vx_dag_depth(const vx_dag *d) { return d ? d->t.depth : 0; }

size_t vx_dag_voxel_workspace_size(uint32_t count) {
  return vx::plain::workspace_size(count);
}

vx_status vx_dag_apply_voxels(vx_dag *d, const vx_voxel *edits, uint32_t count,
                              uint32_t op, void *workspace,
                              size_t workspace_bytes, vx_stream stream) {
  if (d == nullptr || (edits == nullptr && count != 0) || op > 1)
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  if (workspace == nullptr || workspace_bytes < vx_dag_voxel_workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PlainPrep prep;
  if (small_batch(count, true) &&
      plain_prep_layout(workspace, workspace_bytes, edits, count, op, 0, &prep)) {
    // one cooperative launch: voxels -> leaf masks -> the edit
    Ctx x{d->t, d->a, prep.prims, prep.nprims, count};
    const EditCtx e{d->t.hdr, d->a, prep.prims, prep.nprims, count, d->t.depth,
                    static_cast<uint32_t>(vx::tune::get(vx::tune::kEditBigItem))};
    if (d->status_alias == nullptr) {
      VX_TRY(run_small(d, x, e, s, &prep));
      return read_status(d, s, true);
    }
    *reinterpret_cast<volatile uint32_t *>(d->host_status) = kStatusUnset;
    VX_TRY(run_small(d, x, e, s, &prep, d->status_alias));
    return read_written_status(d, s);
  }
  const vx_primitive *prims = nullptr;
  const uint32_t *n = nullptr;
  VX_TRY(vx::plain::prepare(edits, count, d->t.depth, op, 0, workspace, &prims, &n, s));
  VX_TRY(run_pipeline(d, prims, n, count, s, false, 0, small_batch(count, true)));
  return read_status(d, s, true);
}

size_t vx_leaf_command_workspace_size(uint32_t count) { return vx::plain::workspace_size(count); }

vx_status vx_dag_apply_leaf_commands(vx_dag *d, const vx_leaf_command *cmds, uint32_t count,
                                     uint32_t op, void *workspace, size_t workspace_bytes,
                                     vx_stream stream) {
  if (d == nullptr || (cmds == nullptr && count != 0) || op > 1) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  if (workspace == nullptr || workspace_bytes < vx_leaf_command_workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const vx_primitive *prims = nullptr;
  const uint32_t *n = nullptr;
  VX_TRY(vx::plain::prepare_leaf_commands(cmds, count, d->t.depth, op, 0, workspace, &prims, &n,
                                          s));
  VX_TRY(run_pipeline(d, prims, n, count, s, false, 0, small_batch(count, true)));
  return read_status(d, s, true);
}

vx_status vx_dag_apply_primitives(vx_dag *d, const vx_primitive *prims,
                                  uint32_t count, vx_stream stream) {
  if (d == nullptr || (prims == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  return run_pipeline(d, prims, nullptr, count, static_cast<cudaStream_t>(stream));
}

vx_status vx_dag_graph_primitives(vx_dag *d, const vx_primitive *prims,
                                  const uint32_t *device_count, uint32_t capacity,
                                  vx_graph **out) {
  if (d == nullptr || out == nullptr || prims == nullptr || capacity == 0)
    return VX_ERR_INVALID_VALUE;
  return vx::graph::capture(
      [&](cudaStream_t s) { return run_pipeline(d, prims, device_count, capacity, s); }, out);
}

} // extern "C"

namespace vx::dag {
vx_status graph_primitives_grid(vx_dag *d, const vx_primitive *prims, const uint32_t *d_count,
                                uint32_t capacity, uint32_t blocks_per_sm, vx_graph **out) {
  if (d == nullptr || out == nullptr || prims == nullptr || capacity == 0)
    return VX_ERR_INVALID_VALUE;
  return vx::graph::capture(
      [&](cudaStream_t s) {
        return run_pipeline(d, prims, d_count, capacity, s, false, blocks_per_sm);
      },
      out);
}
} // namespace vx::dag

extern "C" {

vx_status vx_dag_graph_voxels(vx_dag *d, const vx_voxel *edits, uint32_t count, uint32_t op,
                              void *workspace, size_t workspace_bytes, vx_graph **out) {
  if (d == nullptr || out == nullptr || edits == nullptr || count == 0 || op > 1)
    return VX_ERR_INVALID_VALUE;
  if (workspace == nullptr || workspace_bytes < vx_dag_voxel_workspace_size(count))
    return VX_ERR_INVALID_VALUE;
  return vx::graph::capture(
      [&](cudaStream_t s) {
        const vx_primitive *prims = nullptr;
        const uint32_t *n = nullptr;
        VX_TRY(vx::plain::prepare(edits, count, d->t.depth, op, 0, workspace, &prims, &n, s));
        return run_pipeline(d, prims, n, count, s, false, 0, small_batch(count, true));
      },
      out);
}

vx_status vx_dag_status(vx_dag *d, vx_stream stream) {
  if (d == nullptr) return VX_ERR_INVALID_VALUE;
  return read_status(d, static_cast<cudaStream_t>(stream), true);
}

vx_status vx_dag_build_terrain(vx_dag *d, const vx_terrain *terrain,
                               vx_stream stream) {
  if (d == nullptr || terrain == nullptr || terrain->scale == 0) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx_primitive p{};
  p.c[0] = static_cast<int32_t>(terrain->seed);
  p.c[1] = static_cast<int32_t>(terrain->scale);
  p.c[2] = static_cast<int32_t>(terrain->caves);
  p.flags = vx_make_flags(vx::edit::kShapeTerrain, VX_OP_ADD, 0);
  VX_TRY(vx_dag_reset(d, stream));
  VX_TRY_CUDA(cudaMemcpyAsync(d->tmp_prim, &p, sizeof(p), cudaMemcpyHostToDevice, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  return run_pipeline(d, d->tmp_prim, nullptr, 1, s, true);
}

vx_status vx_dag_query(const vx_dag *d, const vx_voxel *pts, uint32_t count,
                       uint8_t *out, vx_stream stream) {
  if (d == nullptr || ((pts == nullptr || out == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("dag_query", s);
  vx_dag_view view;
  VX_TRY(vx_dag_device_view(d, &view));
  query_kernel<<<vx::ceil_div(count, kBlock), kBlock, 0, s>>>(view, pts, count, out);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_dag_raycast(const vx_dag *d, const vx_ray *rays, uint32_t count,
                         vx_ray_hit *hits, vx_stream stream) {
  if (d == nullptr || ((rays == nullptr || hits == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("dag_raycast", s);
  vx_dag_view view;
  VX_TRY(vx_dag_device_view(d, &view));
  raycast_kernel<<<vx::ceil_div(count, kBlock), kBlock, 0, s>>>(view, rays, count, hits);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_dag_read_leaves(const vx_dag *d, uint32_t lx0, uint32_t ly0, uint32_t lz0,
                             uint32_t nx, uint32_t ny, uint32_t nz, uint64_t *out,
                             vx_stream stream) {
  const uint64_t n = uint64_t(nx) * ny * nz;
  if (d == nullptr || (out == nullptr && n != 0) || n >= (1ull << 32)) return VX_ERR_INVALID_VALUE;
  if (n == 0) return VX_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::prof::Scope sc("dag_read_leaves", s);
  vx_dag_view view;
  VX_TRY(vx_dag_device_view(d, &view));
  read_leaves_kernel<<<vx::ceil_div(static_cast<uint32_t>(n), kBlock), kBlock, 0, s>>>(
      view, lx0, ly0, lz0, nx, ny, static_cast<uint32_t>(n), out);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_dag_device_view(const vx_dag *d, vx_dag_view *out) {
  if (d == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  *out = vx_dag_view{};
  out->depth = d->t.depth;
  out->root = &d->t.hdr->root;
  for (uint32_t l = 0; l < d->t.depth; ++l) out->pool[l] = d->t.pool[l];
  out->leaves = d->t.leaves;
  return VX_OK;
}

vx_status vx_dag_get_stats(const vx_dag *d, vx_dag_stats *st, vx_stream stream) {
  if (d == nullptr || st == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::edit::Header h;
  VX_TRY_CUDA(cudaMemcpyAsync(&h, d->t.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  *st = vx_dag_stats{};
  for (uint32_t l = 0; l <= d->t.depth && l < 16; ++l) {
    st->nodes_per_level[l] = h.node_count[l];
    st->words_per_level[l] = l < d->t.depth ? h.pool_used[l] : 2 * h.node_count[l];
  }
  for (uint32_t l = 0; l < 16; ++l) {
    st->items_per_level[l] = h.item_count[l];
    st->pairs_per_level[l] = h.pair_count[l];
  }
  st->bytes_reserved = d->bytes;
  st->root = h.root;
  st->status = h.status;
  return VX_OK;
}

vx_status vx_dag_export_canonical(const vx_dag *d, uint32_t *host_root,
                                  uint64_t *host_counts, uint32_t *host_nodes,
                                  uint64_t nodes_capacity_words,
                                  uint64_t *host_leaves,
                                  uint64_t leaves_capacity, vx_stream stream) {
  return vx_dag_export_canonical_at(d, 0xffffffffu, host_root, host_counts, host_nodes,
                                    nodes_capacity_words, host_leaves, leaves_capacity,
                                    stream);
}

vx_status vx_dag_export_canonical_at(const vx_dag *d, uint32_t root, uint32_t *host_root,
                                     uint64_t *host_counts, uint32_t *host_nodes,
                                     uint64_t nodes_capacity_words,
                                     uint64_t *host_leaves, uint64_t leaves_capacity,
                                     vx_stream stream) {
  if (d == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t D = d->t.depth;
  vx::edit::Header h;
  VX_TRY_CUDA(cudaMemcpyAsync(&h, d->t.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  if (root != 0xffffffffu) h.root = root;
  std::vector<std::vector<uint32_t>> pools(D);
  for (uint32_t l = 0; l < D; ++l) {
    const uint64_t used = std::min<uint64_t>(h.pool_used[l], d->t.pool_cap[l]);
    pools[l].resize(used);
    if (used)
      VX_TRY_CUDA(cudaMemcpyAsync(pools[l].data(), d->t.pool[l], used * 4,
                                  cudaMemcpyDeviceToHost, s));
  }
  std::vector<uint64_t> leaves(d->leaf_slots);
  VX_TRY_CUDA(cudaMemcpyAsync(leaves.data(), d->t.leaves, d->leaf_slots * 8,
                              cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  // DFS first-visit numbering per level (children 0..7).
  std::vector<std::vector<uint32_t>> out_nodes(D);
  std::vector<uint64_t> out_leaves;
  std::vector<std::vector<int64_t>> ids(D + 1);
  for (uint32_t l = 0; l < D; ++l) ids[l].assign(pools[l].size() + 2, -1);
  std::vector<int64_t> leaf_ids(d->leaf_slots + 2, -1);
  // iterative DFS with an explicit stack of (level, ref, next child)
  struct Frame {
    uint32_t l, ref, c, id;
    uint32_t rec[10];
  };
  auto visit_leaf = [&](uint32_t ref) -> uint32_t {
    if (leaf_ids[ref] < 0) {
      leaf_ids[ref] = static_cast<int64_t>(out_leaves.size());
      out_leaves.push_back(leaves[ref - 2]);
    }
    return static_cast<uint32_t>(leaf_ids[ref]) + 2;
  };
  uint32_t root_id = h.root;
  if (h.root >= 2) {
    if (D == 0) return VX_ERR_INVALID_VALUE;
    std::vector<Frame> st;
    auto open = [&](uint32_t l, uint32_t ref) {
      Frame f{};
      f.l = l;
      f.ref = ref;
      f.c = 0;
      f.id = static_cast<uint32_t>(out_nodes[l].size() / 10);
      ids[l][ref] = f.id;
      out_nodes[l].resize(out_nodes[l].size() + 10, 0);
      st.push_back(f);
    };
    open(0, h.root);
    root_id = 2;
    while (!st.empty()) {
      Frame &f = st.back();
      if (f.c == 8) {
        for (uint32_t w = 0; w < 10; ++w) out_nodes[f.l][f.id * 10 + w] = f.rec[w];
        const uint32_t id = f.id, l = f.l;
        st.pop_back();
        if (!st.empty()) {
          Frame &p = st.back();
          p.rec[2 + p.c] = id + 2;
          p.rec[0] |= 1u << p.c;
          ++p.c;
        }
        (void)l;
        continue;
      }
      const uint32_t *item = pools[f.l].data() + (f.ref - 2);
      const uint32_t cm = item[0] & 0xffu, fm = (item[0] >> 8) & 0xffu;
      const uint32_t bit = 1u << f.c;
      if (cm & bit) {
        const uint32_t child = item[1 + __builtin_popcount(cm & (bit - 1u))];
        if (f.l + 1 == D) {
          f.rec[2 + f.c] = visit_leaf(child);
          f.rec[0] |= bit;
          ++f.c;
        } else if (ids[f.l + 1][child] >= 0) {
          f.rec[2 + f.c] = static_cast<uint32_t>(ids[f.l + 1][child]) + 2;
          f.rec[0] |= bit;
          ++f.c;
        } else {
          open(f.l + 1, child); // completes when popped
        }
      } else {
        if (fm & bit) {
          f.rec[2 + f.c] = 1;
          f.rec[1] |= bit;
        }
        ++f.c;
      }
    }
  }
  if (host_root) *host_root = root_id;
  uint64_t words = 0;
  for (uint32_t l = 0; l < D; ++l) {
    if (host_counts) host_counts[l] = out_nodes[l].size() / 10;
    words += out_nodes[l].size();
  }
  if (host_counts) host_counts[D] = out_leaves.size();
  if (host_nodes) {
    if (words > nodes_capacity_words) return VX_ERR_INVALID_VALUE;
    uint64_t o = 0;
    for (uint32_t l = 0; l < D; ++l)
      for (uint32_t w : out_nodes[l]) host_nodes[o++] = w;
  }
  if (host_leaves) {
    if (out_leaves.size() > leaves_capacity) return VX_ERR_INVALID_VALUE;
    std::copy(out_leaves.begin(), out_leaves.end(), host_leaves);
  }
  return VX_OK;
}

} // extern "C"

// ============================================================ snapshots ==

extern "C" {

// Copy the whole table state (roots, counters, indexes, pools, leaves) of src
// into dst; both must have been created with the same configuration.
vx_status vx_dag_copy(vx_dag *dst, const vx_dag *src, vx_stream stream) {
  if (dst == nullptr || src == nullptr || dst->t.depth != src->t.depth ||
      dst->leaf_slots != src->leaf_slots)
    return VX_ERR_INVALID_VALUE;
  for (uint32_t l = 0; l < src->t.depth; ++l)
    if (dst->index_slots[l] != src->index_slots[l] ||
        dst->t.pool_cap[l] != src->t.pool_cap[l])
      return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx::edit::Header h;
  VX_TRY_CUDA(cudaMemcpyAsync(&h, src->t.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  for (uint32_t l = 0; l < src->t.depth; ++l) {
    VX_TRY_CUDA(cudaMemcpyAsync(dst->t.index[l], src->t.index[l],
                                src->index_slots[l] * 8, cudaMemcpyDeviceToDevice, s));
    const uint64_t used = std::min<uint64_t>(h.pool_used[l], src->t.pool_cap[l]);
    if (used)
      VX_TRY_CUDA(cudaMemcpyAsync(dst->t.pool[l], src->t.pool[l], used * 4,
                                  cudaMemcpyDeviceToDevice, s));
  }
  VX_TRY_CUDA(cudaMemcpyAsync(dst->t.leaves, src->t.leaves, src->leaf_slots * 8,
                              cudaMemcpyDeviceToDevice, s));
  VX_TRY_CUDA(cudaMemcpyAsync(dst->t.hdr, src->t.hdr, sizeof(vx::edit::Header),
                              cudaMemcpyDeviceToDevice, s));
  return VX_OK;
}

} // extern "C"

// ============================================================ compaction ==
//
// Edits are copy-on-write: every changed node gets a new item and the items
// it replaced stay in the tables until compaction (the reference CPU DAG's
// collect_garbage, svt/hash_dag.hpp:133-191).  Compaction marks the nodes
// reachable from the root level by level, stages their items, clears every
// table and hash-conses the live items back bottom-up, remapping child refs
// through sorted (old ref -> new ref) arrays of the level below.  It is a
// maintenance call: it synchronises, and its temporaries live in the DAG's
// edit arena (VX_ERR_CAPACITY if the arena cannot hold them).

namespace vx::dag {

// Compaction.  Every level l gets a mark bitmap over its old ref space (ref
// - 2 = pool word offset, or leaf slot) and, after an exclusive scan of the
// bitmap words' popcounts, a rank for every live ref: the live refs of a
// level, listed in ascending order, are ranks 0..live-1, and the new ref of
// an old one is new_refs[rank(old)].  Nothing is sized on the host except by
// upper bounds, so the whole pass is stream-ordered.
struct LevelMarks {
  uint32_t *bits;   // mark bitmap word w at bits[2w]; bits[2w + 1] holds prefix[w]
                    // once ranked, so that a rank costs one 8-byte load
  uint32_t *prefix; // exclusive prefix of popcount(bits[2w]) (the scan's array)
  uint32_t *refs;   // live old refs in ascending order (rank order)
  uint32_t *new_refs;
  uint32_t *live;   // device count of live refs
  uint64_t words;   // bitmap words
  uint32_t cap;     // capacity of refs / new_refs
};

__device__ __forceinline__ uint32_t rank_of(const LevelMarks &m, uint32_t ref) {
  const uint32_t b = ref - 2u;
  const uint2 w = reinterpret_cast<const uint2 *>(m.bits)[b >> 5]; // {bits, prefix}
  return w.y + __popc(w.x & ((1u << (b & 31u)) - 1u));
}

// Marks the children of level l's live items in level l+1's bitmap.
__global__ void mark_children_kernel(Tables t, uint32_t l, LevelMarks m, LevelMarks next) {
  const uint32_t n = *m.live;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t *item = t.pool[l] + (m.refs[i] - 2);
    const uint32_t cm = item[0] & 0xffu;
    for (uint32_t k = 0; k < static_cast<uint32_t>(__popc(cm)); ++k) {
      const uint32_t b = item[1 + k] - 2u;
      const uint32_t bit = 1u << (b & 31u);
      uint32_t *word = next.bits + 2u * (b >> 5);
      if (!(ld_relaxed_u32(word) & bit)) atomicOr(word, bit);
    }
  }
}

__global__ void popcount_kernel(LevelMarks m) {
  for (uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; w < m.words;
       w += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    m.prefix[w] = __popc(m.bits[2 * w]);
}

// After the scan: the live count and the rank-ordered list of live refs.
__global__ void list_kernel(Tables t, LevelMarks m) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t first = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (first == 0) {
    const uint64_t last = m.words - 1;
    const uint32_t total = m.prefix[last] + __popc(m.bits[2 * last]);
    if (total > m.cap) set_status(&t.hdr->status, kDevCapacity);
    *m.live = min(total, m.cap);
  }
  for (uint64_t w = first; w < m.words; w += stride) {
    uint32_t bits = m.bits[2 * w];
    uint32_t at = m.prefix[w];
    m.bits[2 * w + 1] = at; // beside the bitmap word, for rank_of
    while (bits) {
      const uint32_t b = __ffs(bits) - 1u;
      bits &= bits - 1u;
      if (at < m.cap) m.refs[at] = static_cast<uint32_t>(w * 32u + b + 2u);
      ++at;
    }
  }
}

__global__ void stage_kernel(Tables t, uint32_t l, LevelMarks m,
                             uint32_t *staged /* 9 words per item */, uint64_t *leaf_masks) {
  const uint32_t n = *m.live;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (l == t.depth) {
      leaf_masks[i] = t.leaves[m.refs[i] - 2];
      continue;
    }
    const uint32_t *item = t.pool[l] + (m.refs[i] - 2);
    const uint32_t w = 1 + __popc(item[0] & 0xffu);
    for (uint32_t k = 0; k < 9; ++k) staged[i * 9 + k] = k < w ? item[k] : 0u;
  }
}

// Re-insertion.  The live items of a level are distinct by content (the
// tables hash-cons them) and stay distinct after their children are renamed
// (renaming is injective), so an item needs no lookup: its pool offset is the
// exclusive scan of the items' word counts and its index entry takes the
// first empty slot of its probe sequence.  No shared counter is touched per
// item; the level's counts are written once at the end.
// Unique inserts (the item is known not to be in the table): the leaf takes
// the first empty slot of its probe sequence; the node is written at its
// pool offset and its index entry takes the first empty slot.
__device__ uint32_t unique_insert_leaf(const Tables &t, uint64_t mask) {
  uint64_t pos = mix64(mask) & t.leaf_mask;
  for (uint32_t probe = 0; probe < kMaxProbes; ++probe) {
    if (ld_relaxed_u64(t.leaves + pos) == 0 &&
        atomicCAS(reinterpret_cast<unsigned long long *>(t.leaves + pos), 0ull,
                  static_cast<unsigned long long>(mask)) == 0ull)
      return static_cast<uint32_t>(pos + 2);
    pos = (pos + 1) & t.leaf_mask;
  }
  set_status(&t.hdr->status, kDevCapacity);
  return kEmptyRef;
}

__device__ uint32_t unique_insert_node(const Tables &t, uint32_t l, const uint32_t *w,
                                       uint32_t n, uint32_t off) {
  if (static_cast<uint64_t>(off) + n > t.pool_cap[l]) {
    set_status(&t.hdr->status, kDevCapacity);
    return kEmptyRef;
  }
  uint32_t *dst = t.pool[l] + off;
  for (uint32_t j = 0; j < n; ++j) dst[j] = w[j];
  const uint64_t h = hash_words(w, n);
  const uint64_t entry =
      (static_cast<uint64_t>(static_cast<uint32_t>(h >> 32) | 1u) << 32) | (off + 2u);
  uint64_t *idx = t.index[l];
  uint64_t pos = h & t.index_mask[l];
  for (uint32_t probe = 0; probe < kMaxProbes; ++probe) {
    if (ld_relaxed_u64(idx + pos) == 0 &&
        atomicCAS(reinterpret_cast<unsigned long long *>(idx + pos), 0ull,
                  static_cast<unsigned long long>(entry)) == 0ull)
      return off + 2u;
    pos = (pos + 1) & t.index_mask[l];
  }
  set_status(&t.hdr->status, kDevCapacity);
  return off + 2u;
}

__global__ void reinsert_leaves_kernel(Tables t, LevelMarks m, const uint64_t *masks) {
  const uint32_t n = *m.live;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    m.new_refs[i] = unique_insert_leaf(t, masks[i]);
}

__global__ void item_words_kernel(LevelMarks m, const uint32_t *staged, uint32_t *words) {
  const uint32_t n = *m.live;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    words[i] = 1u + __popc(staged[i * 9] & 0xffu);
}

__global__ void reinsert_nodes_kernel(Tables t, uint32_t l, LevelMarks m, LevelMarks child,
                                      const uint32_t *staged, const uint32_t *offsets) {
  const uint32_t n = *m.live;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t w[9];
    w[0] = staged[i * 9];
    const uint32_t k = __popc(w[0] & 0xffu);
    for (uint32_t j = 0; j < k; ++j) w[1 + j] = child.new_refs[rank_of(child, staged[i * 9 + 1 + j])];
    m.new_refs[i] = unique_insert_node(t, l, w, 1 + k, offsets[i]);
  }
}

// ---- import of a canonical dump (records of 10 words per inner node:
// [child_mask, fill_mask, child ids x 8], id k + 2 = node k of the next
// level; leaves as u64 masks).  Canonical nodes are distinct per level, so
// the unique inserts above apply; child ids are checked against the next
// level's count (a malformed dump raises kDevInvalid, never an out-of-range
// read).

__global__ void import_leaves_kernel(Tables t, const uint64_t *masks, uint32_t n,
                                     uint32_t *new_refs) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t m = masks[i];
    if (m == 0 || m == ~0ull) {
      set_status(&t.hdr->status, kDevInvalid);
      new_refs[i] = kEmptyRef;
      continue;
    }
    new_refs[i] = unique_insert_leaf(t, m);
  }
}

__global__ void import_words_kernel(const uint32_t *rec, uint32_t n, uint32_t *words) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    words[i] = 1u + __popc(rec[i * 10] & 0xffu);
}

__global__ void import_nodes_kernel(Tables t, uint32_t l, const uint32_t *rec, uint32_t n,
                                    const uint32_t *child_refs, uint32_t child_count,
                                    const uint32_t *offsets, uint32_t *new_refs) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t *r = rec + i * 10;
    const uint32_t cm = r[0] & 0xffu, fm = r[1] & 0xffu;
    uint32_t w[9];
    w[0] = cm | (fm << 8);
    uint32_t k = 0;
    bool ok = (cm & fm) == 0 && (cm != 0 || (fm != 0 && fm != 0xffu));
    for (uint32_t c = 0; c < 8; ++c) {
      if (!(cm & (1u << c))) continue;
      const uint32_t id = r[2 + c];
      ok = ok && id >= 2u && id - 2u < child_count;
      w[1 + k++] = ok ? child_refs[id - 2u] : kEmptyRef;
    }
    if (!ok) {
      set_status(&t.hdr->status, kDevInvalid);
      new_refs[i] = kEmptyRef;
      continue;
    }
    new_refs[i] = unique_insert_node(t, l, w, 1 + k, offsets[i]);
  }
}

__global__ void import_finish_kernel(Tables t, uint32_t l, uint32_t n, const uint32_t *rec,
                                     const uint32_t *offsets) {
  t.hdr->node_count[l] = n;
  if (l < t.depth)
    t.hdr->pool_used[l] = n ? offsets[n - 1] + 1u + __popc(rec[(n - 1) * 10ull] & 0xffu) : 0u;
}

__global__ void import_root_kernel(Tables t, const uint32_t *level0_refs, uint32_t root_id) {
  if (t.hdr->status != kDevOk) return;
  t.hdr->root = root_id >= 2u ? level0_refs[root_id - 2u] : root_id;
}

// The level's node count and pool use, once its items are in.
__global__ void finish_level_kernel(Tables t, uint32_t l, LevelMarks m, const uint32_t *staged,
                                    const uint32_t *offsets) {
  const uint32_t n = *m.live;
  t.hdr->node_count[l] = n;
  if (l < t.depth)
    t.hdr->pool_used[l] = n ? offsets[n - 1] + 1u + __popc(staged[(n - 1) * 9ull] & 0xffu) : 0u;
}

__global__ void seed_root_kernel(LevelMarks m, uint32_t root) {
  m.refs[0] = root;
  *m.live = 1;
}

__global__ void set_root_kernel(Tables t, uint32_t root) { t.hdr->root = root; }

__global__ void publish_compacted_root_kernel(Tables t, LevelMarks m0) {
  if (t.hdr->status == kDevOk) t.hdr->root = m0.new_refs[0];
}

// Carver stand-in that only adds up sizes (pointers come back null).
struct SizingCarver {
  Sizer z;
  template <class T> T *take(size_t n) {
    z.take<T>(n);
    return nullptr;
  }
};

// ------------------------------------------------------------ item set --
// A standalone content-addressed store of fixed-width items (the reference's
// AccelerationHashSet32, cuda/hash_table/acceleration_hash/set/*): one table
// of the same kind as a DAG level.  Pointers are item index + 1 (0 = null).

__device__ __forceinline__ uint32_t item_ptr(uint32_t ref, uint32_t width) {
  return ref >= 2u ? (ref - 2u) / width + 1u : 0u;
}

// Probe only: the ref of an equal item, or 0.
__device__ uint32_t node_find(const Tables &t, uint32_t l, const uint32_t *w, uint32_t n) {
  const uint64_t h = hash_words(w, n);
  const uint32_t tag = static_cast<uint32_t>(h >> 32) | 1u;
  const uint64_t *idx = t.index[l];
  const uint32_t *pool = t.pool[l];
  uint64_t pos = h & t.index_mask[l];
  for (uint32_t probe = 0; probe < kMaxProbes; ++probe) {
    const uint64_t v = ld_relaxed_u64(idx + pos);
    if (v == 0) return 0u;
    const uint32_t r = static_cast<uint32_t>(v);
    if (static_cast<uint32_t>(v >> 32) == tag && r >= 2u && r != kBusy) {
      fence_acq_rel_gpu();
      bool eq = true;
      for (uint32_t i = 0; i < n && eq; ++i) eq = pool[r - 2u + i] == w[i];
      if (eq) return r;
    }
    pos = (pos + 1) & t.index_mask[l];
  }
  return 0u;
}

enum class ItemOp { Find, FindOrInsert, InsertUnique };

template <ItemOp Op>
__global__ void itemset_kernel(Tables t, uint32_t width, const uint32_t *items, uint32_t n,
                               uint32_t *ptrs, uint32_t *statuses) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t w[9];
    for (uint32_t j = 0; j < width; ++j) w[j] = items[i * width + j];
    uint32_t ref = 0, status = VX_HASH_NOT_FOUND;
    if (Op == ItemOp::Find) {
      ref = node_find(t, 0, w, width);
      status = ref ? VX_HASH_FOUND : VX_HASH_NOT_FOUND;
    } else if (Op == ItemOp::FindOrInsert) {
      bool inserted = false;
      ref = node_find_or_insert(t, 0, ArrayWords{w, width}, &inserted);
      status = ref >= 2u ? (inserted ? VX_HASH_INSERTED : VX_HASH_FOUND) : VX_HASH_OVERFLOW;
      if (ref < 2u) ref = 0;
    } else {
      const uint32_t off = atomicAdd(&t.hdr->pool_used[0], width);
      if (static_cast<uint64_t>(off) + width > t.pool_cap[0]) {
        status = VX_HASH_OVERFLOW;
      } else {
        ref = unique_insert_node(t, 0, w, width, off);
        status = VX_HASH_INSERTED;
        atomicAdd(reinterpret_cast<unsigned long long *>(&t.hdr->node_count[0]), 1ull);
      }
    }
    ptrs[i] = item_ptr(ref, width);
    if (statuses) statuses[i] = status;
  }
}

__global__ void itemset_read_kernel(Tables t, uint32_t width, const uint32_t *ptrs, uint32_t n,
                                    uint32_t *out, uint32_t *statuses) {
  const uint32_t stored = t.hdr->pool_used[0] / width;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t p = ptrs[i];
    const bool ok = p >= 1u && p <= stored;
    for (uint32_t j = 0; j < width; ++j)
      out[i * width + j] = ok ? t.pool[0][(p - 1u) * static_cast<uint64_t>(width) + j] : 0u;
    if (statuses) statuses[i] = ok ? VX_HASH_FOUND : VX_HASH_NOT_FOUND;
  }
}

} // namespace vx::dag

struct vx_itemset {
  vx::dag::Tables t{};
  uint32_t width = 0;
  uint64_t index_slots = 0;
};

namespace {
template <vx::dag::ItemOp Op>
vx_status itemset_launch(const vx_itemset *s, const uint32_t *items, uint32_t count,
                         uint32_t *ptrs, uint32_t *statuses, vx_stream stream) {
  if (s == nullptr || ((items == nullptr || ptrs == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t grid = std::min<uint32_t>(vx::ceil_div(count, vx::dag::kBlock),
                                           static_cast<uint32_t>(vx::sm_count()) * 16u);
  vx::prof::Scope sc("itemset", st);
  vx::dag::itemset_kernel<Op><<<grid, vx::dag::kBlock, 0, st>>>(s->t, s->width, items, count,
                                                                 ptrs, statuses);
  return vx::from_cuda(cudaGetLastError());
}
} // namespace

extern "C" {

vx_status vx_itemset_clear(vx_itemset *s, vx_stream stream) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  VX_TRY_CUDA(cudaMemsetAsync(s->t.index[0], 0, s->index_slots * 8, st));
  VX_TRY_CUDA(cudaMemsetAsync(s->t.hdr, 0, sizeof(vx::edit::Header), st));
  return VX_OK;
}

vx_status vx_itemset_destroy(vx_itemset *s) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  cudaFree(s->t.index[0]);
  cudaFree(s->t.pool[0]);
  cudaFree(s->t.hdr);
  delete s;
  return VX_OK;
}

vx_status vx_itemset_create(uint32_t width, uint32_t max_items, vx_itemset **out) {
  if (out == nullptr || width < 1 || width > 9 || max_items == 0) return VX_ERR_INVALID_VALUE;
  auto *s = new (std::nothrow) vx_itemset;
  if (s == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  s->width = width;
  s->t.depth = 1;
  s->index_slots = vx::dag::next_pow2(2ull * max_items);
  s->t.index_mask[0] = s->index_slots - 1;
  s->t.pool_cap[0] = std::min<uint64_t>(static_cast<uint64_t>(max_items) * width, 0xfffffff0ull);
  cudaError_t e = cudaMalloc(&s->t.index[0], s->index_slots * 8);
  if (e == cudaSuccess) e = cudaMalloc(&s->t.pool[0], s->t.pool_cap[0] * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->t.hdr, sizeof(vx::edit::Header));
  if (e != cudaSuccess) {
    vx_itemset_destroy(s);
    return vx::from_cuda(e);
  }
  const vx_status st = vx_itemset_clear(s, nullptr);
  if (st != VX_OK) {
    vx_itemset_destroy(s);
    return st;
  }
  VX_TRY_CUDA(cudaStreamSynchronize(nullptr));
  *out = s;
  return VX_OK;
}


vx_status vx_itemset_find(const vx_itemset *s, const uint32_t *items, uint32_t count,
                          uint32_t *ptrs, uint32_t *statuses, vx_stream stream) {
  return itemset_launch<vx::dag::ItemOp::Find>(s, items, count, ptrs, statuses, stream);
}

vx_status vx_itemset_find_or_insert(vx_itemset *s, const uint32_t *items, uint32_t count,
                                    uint32_t *ptrs, uint32_t *statuses, vx_stream stream) {
  return itemset_launch<vx::dag::ItemOp::FindOrInsert>(s, items, count, ptrs, statuses, stream);
}

vx_status vx_itemset_insert_unique_unchecked(vx_itemset *s, const uint32_t *items,
                                             uint32_t count, uint32_t *ptrs,
                                             uint32_t *statuses, vx_stream stream) {
  return itemset_launch<vx::dag::ItemOp::InsertUnique>(s, items, count, ptrs, statuses, stream);
}

vx_status vx_itemset_read(const vx_itemset *s, const uint32_t *ptrs, uint32_t count,
                          uint32_t *items, uint32_t *statuses, vx_stream stream) {
  if (s == nullptr || ((items == nullptr || ptrs == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t grid = std::min<uint32_t>(vx::ceil_div(count, vx::dag::kBlock),
                                           static_cast<uint32_t>(vx::sm_count()) * 16u);
  vx::prof::Scope sc("itemset_read", st);
  vx::dag::itemset_read_kernel<<<grid, vx::dag::kBlock, 0, st>>>(s->t, s->width, ptrs, count,
                                                                 items, statuses);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_itemset_count(const vx_itemset *s, uint64_t *host_count, vx_stream stream) {
  if (s == nullptr || host_count == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  VX_TRY_CUDA(cudaMemcpyAsync(host_count, &s->t.hdr->node_count[0], 8, cudaMemcpyDeviceToHost, st));
  VX_TRY_CUDA(cudaStreamSynchronize(st));
  return VX_OK;
}

vx_status vx_dag_import_canonical(vx_dag *d, uint32_t root, const uint64_t *host_counts,
                                  const uint32_t *host_nodes, const uint64_t *host_leaves,
                                  vx_stream stream) {
  if (d == nullptr || host_counts == nullptr || root > 2u) return VX_ERR_INVALID_VALUE;
  const uint32_t D = d->t.depth;
  uint64_t total_nodes = 0, max_n = 1;
  for (uint32_t l = 0; l <= D; ++l) {
    if (host_counts[l] > 0xffffffffull) return VX_ERR_CAPACITY;
    if (l < D) total_nodes += host_counts[l];
    max_n = std::max<uint64_t>(max_n, host_counts[l]);
  }
  if ((total_nodes && host_nodes == nullptr) || (host_counts[D] && host_leaves == nullptr))
    return VX_ERR_INVALID_VALUE;
  if (root == 2u && host_counts[0] != 1) return VX_ERR_INVALID_VALUE;
  if (root < 2u && total_nodes + host_counts[D] != 0) return VX_ERR_INVALID_VALUE;
  uint64_t rec0 = 0;
  for (uint32_t l = 0; l < D; ++l) {
    uint64_t words = 0; // exact pool words of the level
    for (uint64_t i = 0; i < host_counts[l]; ++i)
      words += 1 + __builtin_popcount(host_nodes[(rec0 + i) * 10] & 0xffu);
    rec0 += host_counts[l];
    if (host_counts[l] > d->index_slots[l] / 2 || words > d->t.pool_cap[l])
      return VX_ERR_CAPACITY;
  }
  if (host_counts[D] > d->leaf_slots / 2) return VX_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t grid = static_cast<uint32_t>(vx::sm_count()) * 8u;
  // One temporary block: records of the largest level, its offsets, new
  // refs of two adjacent levels, the leaf masks and the scan workspace.
  const size_t scan_bytes = vx_scan_workspace_size(static_cast<uint32_t>(max_n));
  vx::Sizer z;
  z.take<uint32_t>(max_n * 10);
  z.take<uint32_t>(max_n);
  z.take<uint32_t>(max_n);
  z.take<uint32_t>(max_n);
  z.take<uint64_t>(std::max<uint64_t>(host_counts[D], 1));
  z.take<unsigned char>(scan_bytes);
  struct TempBlock {
    void *p = nullptr;
    ~TempBlock() { if (p) cudaFree(p); }
  } temp;
  VX_TRY_CUDA(cudaMalloc(&temp.p, z.offset));
  vx::Carver c(temp.p);
  uint32_t *rec = c.take<uint32_t>(max_n * 10);
  uint32_t *offsets = c.take<uint32_t>(max_n);
  uint32_t *refs[2] = {c.take<uint32_t>(max_n), c.take<uint32_t>(max_n)};
  uint64_t *masks = c.take<uint64_t>(std::max<uint64_t>(host_counts[D], 1));
  void *scan_ws = c.take<unsigned char>(scan_bytes);
  VX_TRY(vx_dag_reset(d, stream));
  const uint32_t nl = static_cast<uint32_t>(host_counts[D]);
  if (nl) {
    VX_TRY_CUDA(cudaMemcpyAsync(masks, host_leaves, nl * 8ull, cudaMemcpyHostToDevice, s));
    vx::prof::Scope sc("dag_import", s);
    import_leaves_kernel<<<grid, kBlock, 0, s>>>(d->t, masks, nl, refs[D & 1u]);
    VX_TRY_CUDA(cudaGetLastError());
  }
  import_finish_kernel<<<1, 1, 0, s>>>(d->t, D, nl, nullptr, nullptr);
  VX_TRY_CUDA(cudaGetLastError());
  std::vector<uint64_t> first(D + 1, 0); // first record of each level
  for (uint32_t l = 1; l < D; ++l) first[l] = first[l - 1] + host_counts[l - 1] * 10;
  for (uint32_t r = D; r > 0; --r) {
    const uint32_t l = r - 1;
    const uint32_t n = static_cast<uint32_t>(host_counts[l]);
    if (n) {
      VX_TRY_CUDA(cudaMemcpyAsync(rec, host_nodes + first[l], n * 40ull, cudaMemcpyHostToDevice,
                                  s));
      {
        vx::prof::Scope sc("dag_import", s);
        import_words_kernel<<<grid, kBlock, 0, s>>>(rec, n, offsets);
        VX_TRY_CUDA(cudaGetLastError());
      }
      VX_TRY(vx_scan_exclusive_sum_u32(offsets, n, scan_ws, scan_bytes, s));
      vx::prof::Scope sc("dag_import", s);
      import_nodes_kernel<<<grid, kBlock, 0, s>>>(d->t, l, rec, n, refs[(l + 1) & 1u],
                                                  static_cast<uint32_t>(host_counts[l + 1]),
                                                  offsets, refs[l & 1u]);
      VX_TRY_CUDA(cudaGetLastError());
    }
    import_finish_kernel<<<1, 1, 0, s>>>(d->t, l, n, rec, offsets);
    VX_TRY_CUDA(cudaGetLastError());
  }
  import_root_kernel<<<1, 1, 0, s>>>(d->t, refs[0], root);
  VX_TRY_CUDA(cudaGetLastError());
  return read_status(d, s, true);
}

namespace {
constexpr char kDagFileMagic[8] = {'V', 'X', 'D', 'A', 'G', 'C', 'N', '1'};
} // namespace

vx_status vx_dag_save(const vx_dag *d, const char *path, vx_stream stream) {
  if (d == nullptr || path == nullptr) return VX_ERR_INVALID_VALUE;
  const uint32_t D = d->t.depth;
  uint32_t root = 0;
  std::vector<uint64_t> counts(D + 1, 0);
  VX_TRY(vx_dag_export_canonical(d, &root, counts.data(), nullptr, 0, nullptr, 0, stream));
  uint64_t words = 0;
  for (uint32_t l = 0; l < D; ++l) words += counts[l] * 10;
  std::vector<uint32_t> nodes(words);
  std::vector<uint64_t> leaves(counts[D]);
  VX_TRY(vx_dag_export_canonical(d, &root, counts.data(), nodes.data(), words, leaves.data(),
                                 leaves.size(), stream));
  FILE *f = std::fopen(path, "wb");
  if (f == nullptr) return VX_ERR_IO;
  const uint32_t head[4] = {1u /* version */, D, root, 0u};
  bool ok = std::fwrite(kDagFileMagic, 1, 8, f) == 8 && std::fwrite(head, 4, 4, f) == 4 &&
            std::fwrite(counts.data(), 8, counts.size(), f) == counts.size() &&
            std::fwrite(nodes.data(), 4, nodes.size(), f) == nodes.size() &&
            std::fwrite(leaves.data(), 8, leaves.size(), f) == leaves.size();
  ok = std::fclose(f) == 0 && ok;
  return ok ? VX_OK : VX_ERR_IO;
}

vx_status vx_dag_load(vx_dag *d, const char *path, vx_stream stream) {
  if (d == nullptr || path == nullptr) return VX_ERR_INVALID_VALUE;
  FILE *f = std::fopen(path, "rb");
  if (f == nullptr) return VX_ERR_IO;
  struct Closer {
    FILE *f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  char magic[8];
  uint32_t head[4];
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kDagFileMagic, 8) != 0 ||
      std::fread(head, 4, 4, f) != 4 || head[0] != 1u)
    return VX_ERR_INVALID_VALUE;
  const uint32_t D = head[1], root = head[2];
  if (D != d->t.depth || root > 2u) return VX_ERR_INVALID_VALUE;
  std::vector<uint64_t> counts(D + 1);
  if (std::fread(counts.data(), 8, counts.size(), f) != counts.size()) return VX_ERR_IO;
  uint64_t words = 0;
  for (uint32_t l = 0; l < D; ++l) {
    if (counts[l] > (1ull << 32)) return VX_ERR_INVALID_VALUE;
    words += counts[l] * 10;
  }
  if (counts[D] > (1ull << 32)) return VX_ERR_INVALID_VALUE;
  std::vector<uint32_t> nodes(words);
  std::vector<uint64_t> leaves(counts[D]);
  if (std::fread(nodes.data(), 4, nodes.size(), f) != nodes.size() ||
      std::fread(leaves.data(), 8, leaves.size(), f) != leaves.size())
    return VX_ERR_IO;
  return vx_dag_import_canonical(d, root, counts.data(), nodes.data(), leaves.data(), stream);
}

vx_status vx_dag_compact(vx_dag *d, vx_stream stream) {
  if (d == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t D = d->t.depth;
  vx::edit::Header h;
  VX_TRY_CUDA(cudaMemcpyAsync(&h, d->t.hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  if (h.status != vx::kDevOk) return vx::status_from_device(h.status);
  if (h.root < 2) { // empty or full world: nothing is live
    VX_TRY(vx_dag_reset(d, stream));
    vx::prof::Scope sc("dag_set_root", s);
    set_root_kernel<<<1, 1, 0, s>>>(d->t, h.root);
    return vx::from_cuda(cudaGetLastError());
  }
  const uint32_t grid = static_cast<uint32_t>(vx::sm_count()) * 8u;
  // Temporaries: per level a bitmap and prefix over its old ref space and
  // live-ref / new-ref lists sized by the level's node count, the scan
  // workspace, then (once the live counts are known) the staged items.  They
  // live in the idle edit arena when it is large enough, else in temporary
  // allocations.
  std::vector<LevelMarks> m(D + 1);
  uint64_t max_words = 1;
  for (uint32_t l = 0; l <= D; ++l) {
    const uint64_t space = l == D ? d->leaf_slots
                                  : std::min<uint64_t>(h.pool_used[l], d->t.pool_cap[l]);
    m[l].words = std::max<uint64_t>((space + 31) / 32, 1);
    m[l].cap = static_cast<uint32_t>(std::max<uint64_t>(h.node_count[l], 1));
    max_words = std::max(max_words, m[l].words);
  }
  if (max_words > 0xffffffffull) return VX_ERR_CAPACITY;
  uint64_t max_scan = max_words;
  for (uint32_t l = 0; l <= D; ++l) max_scan = std::max<uint64_t>(max_scan, m[l].cap);
  const size_t scan_bytes = vx_scan_workspace_size(static_cast<uint32_t>(max_scan));
  uint32_t *counts = nullptr;
  void *scan_ws = nullptr;
  auto carve_marks = [&](auto &c) {
    counts = c.template take<uint32_t>(D + 1);
    scan_ws = c.template take<unsigned char>(scan_bytes);
    for (uint32_t l = 0; l <= D; ++l) {
      m[l].live = counts + l;
      m[l].bits = c.template take<uint32_t>(2 * m[l].words);
      m[l].prefix = c.template take<uint32_t>(m[l].words);
      m[l].refs = c.template take<uint32_t>(m[l].cap);
      m[l].new_refs = c.template take<uint32_t>(m[l].cap);
    }
  };
  const size_t arena_bytes = static_cast<size_t>(d->a.item_cap) * sizeof(vx::edit::Item) +
                             2ull * d->a.pair_cap * 4;
  struct TempBlock {
    void *p = nullptr;
    ~TempBlock() { if (p) cudaFree(p); }
  } temp_marks, temp_staged;
  SizingCarver marks_size;
  carve_marks(marks_size);
  void *marks_base = d->arena_mem;
  if (marks_size.z.offset > arena_bytes) {
    VX_TRY_CUDA(cudaMalloc(&temp_marks.p, marks_size.z.offset));
    marks_base = temp_marks.p;
  }
  vx::Carver carver(marks_base);
  carve_marks(carver);
  for (uint32_t l = 1; l <= D; ++l)
    VX_TRY_CUDA(cudaMemsetAsync(m[l].bits, 0, m[l].words * 8, s));
  {
    vx::prof::Scope sc("dag_compact_mark", s);
    seed_root_kernel<<<1, 1, 0, s>>>(m[0], h.root);
  }
  VX_TRY_CUDA(cudaGetLastError());
  // Mark top-down: children of level l's live items, then rank level l+1.
  for (uint32_t l = 0; l < D; ++l) {
    {
      vx::prof::Scope sc("dag_compact_mark", s);
      mark_children_kernel<<<grid, kBlock, 0, s>>>(d->t, l, m[l], m[l + 1]);
      VX_TRY_CUDA(cudaGetLastError());
    }
    {
      vx::prof::Scope sc("dag_compact_rank", s);
      popcount_kernel<<<grid, kBlock, 0, s>>>(m[l + 1]);
      VX_TRY_CUDA(cudaGetLastError());
    }
    VX_TRY(vx_scan_exclusive_sum_u32(m[l + 1].prefix, static_cast<uint32_t>(m[l + 1].words),
                                     scan_ws, scan_bytes, s));
    {
      vx::prof::Scope sc("dag_compact_rank", s);
      list_kernel<<<grid, kBlock, 0, s>>>(d->t, m[l + 1]);
      VX_TRY_CUDA(cudaGetLastError());
    }
  }
  // Live counts (and a capacity error raised while listing, which must not
  // be lost to the reset below).
  std::vector<uint32_t> live(D + 1, 0);
  uint32_t mark_status = 0;
  VX_TRY_CUDA(cudaMemcpyAsync(live.data(), counts, 4 * (D + 1), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaMemcpyAsync(&mark_status, &d->t.hdr->status, 4, cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  if (mark_status != vx::kDevOk) return vx::status_from_device(mark_status);
  // Staging, sized by the live counts: 9 words per inner item, leaf masks.
  std::vector<uint32_t *> staged(D + 1, nullptr), offsets(D + 1, nullptr);
  uint64_t *leaf_masks = nullptr;
  auto carve_staged = [&](auto &c) {
    leaf_masks = c.template take<uint64_t>(std::max<uint32_t>(live[D], 1));
    for (uint32_t l = 0; l < D; ++l) {
      staged[l] = c.template take<uint32_t>(std::max<uint32_t>(live[l], 1) * 9ull);
      offsets[l] = c.template take<uint32_t>(std::max<uint32_t>(live[l], 1));
    }
  };
  SizingCarver staged_size;
  staged_size.z.offset = marks_base == d->arena_mem ? carver.offset : 0;
  carve_staged(staged_size);
  if (marks_base == d->arena_mem && staged_size.z.offset <= arena_bytes) {
    carve_staged(carver);
  } else {
    SizingCarver alone;
    carve_staged(alone);
    VX_TRY_CUDA(cudaMalloc(&temp_staged.p, alone.z.offset));
    vx::Carver c2(temp_staged.p);
    carve_staged(c2);
  }
  // Stage every live item, then clear the tables.
  for (uint32_t l = 0; l <= D; ++l) {
    vx::prof::Scope sc("dag_compact_stage", s);
    stage_kernel<<<grid, kBlock, 0, s>>>(d->t, l, m[l], staged[l], leaf_masks);
    VX_TRY_CUDA(cudaGetLastError());
  }
  VX_TRY(vx_dag_reset(d, stream));
  // Re-insert bottom-up; a child's new ref is new_refs[rank(old ref)].
  for (uint32_t r = D + 1; r > 0; --r) {
    const uint32_t l = r - 1;
    if (l < D && live[l]) {
      {
        vx::prof::Scope sc("dag_compact_reinsert", s);
        item_words_kernel<<<grid, kBlock, 0, s>>>(m[l], staged[l], offsets[l]);
        VX_TRY_CUDA(cudaGetLastError());
      }
      VX_TRY(vx_scan_exclusive_sum_u32(offsets[l], live[l], scan_ws, scan_bytes, s));
    }
    vx::prof::Scope sc("dag_compact_reinsert", s);
    if (l == D)
      reinsert_leaves_kernel<<<grid, kBlock, 0, s>>>(d->t, m[D], leaf_masks);
    else
      reinsert_nodes_kernel<<<grid, kBlock, 0, s>>>(d->t, l, m[l], m[l + 1], staged[l],
                                                    offsets[l]);
    VX_TRY_CUDA(cudaGetLastError());
    finish_level_kernel<<<1, 1, 0, s>>>(d->t, l, m[l], staged[l], offsets[l]);
    VX_TRY_CUDA(cudaGetLastError());
  }
  {
    vx::prof::Scope sc("dag_set_root", s);
    publish_compacted_root_kernel<<<1, 1, 0, s>>>(d->t, m[0]);
  }
  VX_TRY_CUDA(cudaGetLastError());
  return read_status(d, s, true);
}

} // extern "C"

// ======================================================= serving hooks ==

#include "dag_internal.cuh"

namespace vx::dag {

const void *device_header(const vx_dag *d) { return d->t.hdr; }
size_t header_bytes() { return sizeof(vx::edit::Header); }
uint32_t header_root(const void *hh) { return static_cast<const vx::edit::Header *>(hh)->root; }
uint32_t header_status(const void *hh) { return static_cast<const vx::edit::Header *>(hh)->status; }

TableRoom table_room(const vx_dag *d, const void *hh) {
  const auto *h = static_cast<const vx::edit::Header *>(hh);
  TableRoom r{};
  r.depth = d->t.depth;
  for (uint32_t l = 0; l < d->t.depth; ++l) {
    r.node_cap[l] = d->index_slots[l] / 2;
    r.word_cap[l] = d->t.pool_cap[l];
    r.nodes[l] = h->node_count[l];
    r.words[l] = h->pool_used[l];
  }
  r.node_cap[d->t.depth] = d->leaf_slots / 2;
  r.nodes[d->t.depth] = h->node_count[d->t.depth];
  return r;
}

vx_status read_header(const vx_dag *d, void *host, cudaStream_t s) {
  VX_TRY_CUDA(cudaMemcpyAsync(host, d->t.hdr, sizeof(vx::edit::Header), cudaMemcpyDeviceToHost, s));
  VX_TRY_CUDA(cudaStreamSynchronize(s));
  return VX_OK;
}

double fill_fraction(const vx_dag *d, const void *hh) {
  const auto *h = static_cast<const vx::edit::Header *>(hh);
  double f = 0.0;
  for (uint32_t l = 0; l < d->t.depth; ++l) {
    f = std::max(f, static_cast<double>(h->node_count[l]) / (d->index_slots[l] / 2.0));
    f = std::max(f, static_cast<double>(h->pool_used[l]) / static_cast<double>(d->t.pool_cap[l]));
  }
  f = std::max(f, static_cast<double>(h->node_count[d->t.depth]) / (d->leaf_slots / 2.0));
  return f;
}

} // namespace vx::dag
