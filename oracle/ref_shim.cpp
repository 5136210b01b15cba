// ORACLE - test infrastructure only.  A thin C shim over the reference's own
// CPU implementations, compiled from the reference headers where they lie
// (algorithm/lib/include/algo/svt/hash_dag.hpp and svo.hpp); see build.py.
// It exists to pin this project's oracle and to time the reference's CPU path
// as a baseline.  Nothing here is part of the product.
//
// The canonical dumps below read the reference objects' internal node stores,
// so the shim opens their private members to this translation unit only.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#define private public
#include <algo/svt/hash_dag.hpp>
#include <algo/svt/svo.hpp>
#undef private

using u32 = std::uint32_t;
using u64 = std::uint64_t;
using algo::svt::HashDAG;
using algo::svt::SVO;

namespace {

// DFS first-visit canonical form of a HashDAG (children 0..7): per inner level
// 10 words per node [child_mask, fill_mask, id x 8] where id 0 = empty,
// 1 = full, k + 2 = node k of the next level; leaves as u64 masks.  Full
// subtrees (HashDAG::full_node_ptrs_, full_leaf_ptr_, hash_dag.hpp:329-341)
// become id 1.
struct DagDump {
  const HashDAG &dag;
  std::vector<std::unordered_map<u32, u32>> ids;
  std::vector<std::vector<u32>> nodes;
  std::vector<u64> leaves;

  explicit DagDump(const HashDAG &d)
      : dag(d), ids(d.depth_ + 1), nodes(d.depth_) {}

  bool is_full(u32 level, u32 ptr) const {
    if (level == dag.depth_) return ptr == dag.full_leaf_ptr_;
    return ptr == dag.full_node_ptrs_[level];
  }

  u32 visit(u32 level, u32 ptr) {
    if (ptr == 0) return 0;
    if (is_full(level, ptr)) return 1;
    auto it = ids[level].find(ptr);
    if (it != ids[level].end()) return it->second + 2;
    if (level == dag.depth_) {
      const u32 id = static_cast<u32>(leaves.size());
      ids[level][ptr] = id;
      leaves.push_back(dag.read_leaf(ptr));
      return id + 2;
    }
    const u32 id = static_cast<u32>(nodes[level].size() / 10);
    ids[level][ptr] = id;
    nodes[level].resize(nodes[level].size() + 10, 0);
    const auto node = dag.read_node(ptr);
    u32 rec[10] = {0};
    for (u32 c = 0; c < 8; ++c) {
      u32 child = 0;
      if (node.child_mask & (1u << c)) child = visit(level + 1, node.child_ptrs[c]);
      rec[2 + c] = child;
      if (child == 1) rec[1] |= 1u << c;
      if (child >= 2) rec[0] |= 1u << c;
    }
    for (u32 w = 0; w < 10; ++w) nodes[level][id * 10 + w] = rec[w];
    return id + 2;
  }
};

// DFS pre-order canonical form of an SVO: node ids in first-visit order (root
// = 0), leaf ids in first-visit order; an absent child keeps its word (bit 31
// = filled), a present child is bit 30 | canonical index (svo.hpp:19-91,
// CHILD_* constants at svo.hpp:11-16).
struct SvoDump {
  const SVO &svo;
  std::vector<u32> nodes;
  std::vector<u64> leaves;

  explicit SvoDump(const SVO &s) : svo(s) {}

  u32 visit(u32 index, u32 depth) {
    const u32 id = static_cast<u32>(nodes.size() / 8);
    nodes.resize(nodes.size() + 8, 0);
    const auto &node = svo.nodes_[index];
    u32 rec[8];
    for (u32 c = 0; c < 8; ++c) {
      const u32 info = node.child_info[c].info;
      if (info & algo::svt::CHILD_MASK_BIT) {
        const u32 child = info & algo::svt::CHILD_INDEX_MASK;
        u32 cid;
        if (depth + 1 < svo.max_depth_) {
          cid = visit(child, depth + 1);
        } else {
          cid = static_cast<u32>(leaves.size());
          leaves.push_back(svo.leaves_[child].voxel_data);
        }
        // Bit 31 of a child-present word is a don't-care (the reference
        // reads it only when bit 30 is clear); canonical form drops it.
        rec[c] = algo::svt::CHILD_MASK_BIT | cid;
      } else {
        rec[c] = info;
      }
    }
    for (u32 c = 0; c < 8; ++c) nodes[id * 8 + c] = rec[c];
    return id;
  }
};

} // namespace

extern "C" {

void *ref_dag_new(u32 depth) {
  try {
    return new HashDAG(depth);
  } catch (...) {
    return nullptr;
  }
}
void ref_dag_free(void *h) { delete static_cast<HashDAG *>(h); }

// Boxes are half-open [min, max) like HashDAG::Box (hash_dag.hpp:22-29).
int ref_dag_edit_box(void *h, u32 x0, u32 y0, u32 z0, u32 x1, u32 y1, u32 z1,
                     int fill) {
  try {
    HashDAG::Box b{x0, y0, z0, x1, y1, z1};
    auto *d = static_cast<HashDAG *>(h);
    if (fill) d->fill_box(b);
    else d->clear_box(b);
    return 0;
  } catch (...) {
    return 1;
  }
}

// Apply one sphere (|p - c|^2 <= r^2) or box as x-runs of fill_box / clear_box
// calls, clipped to the box [lo, hi) (the world when lo / hi are null);
// returns the number of voxels covered (the CPU baseline's unit of work), or
// -1 on error.
long long ref_dag_apply_prim_clipped(void *h, int shape, long long cx, long long cy,
                                     long long cz, long long r0, long long r1, long long r2,
                                     int fill, const long long *lo, const long long *hi) {
  auto *d = static_cast<HashDAG *>(h);
  const long long world = d->world_voxel_count();
  const long long b0[3] = {lo ? std::max(0ll, lo[0]) : 0, lo ? std::max(0ll, lo[1]) : 0,
                           lo ? std::max(0ll, lo[2]) : 0};
  const long long b1[3] = {hi ? std::min(world, hi[0]) : world, hi ? std::min(world, hi[1]) : world,
                           hi ? std::min(world, hi[2]) : world};
  long long voxels = 0;
  try {
    if (shape == 1) {
      const long long x0 = std::max(b0[0], cx - r0), x1 = std::min(b1[0], cx + r0 + 1);
      const long long y0 = std::max(b0[1], cy - r1), y1 = std::min(b1[1], cy + r1 + 1);
      const long long z0 = std::max(b0[2], cz - r2), z1 = std::min(b1[2], cz + r2 + 1);
      if (x1 <= x0 || y1 <= y0 || z1 <= z0) return 0;
      HashDAG::Box b{u32(x0), u32(y0), u32(z0), u32(x1), u32(y1), u32(z1)};
      fill ? d->fill_box(b) : d->clear_box(b);
      return (x1 - x0) * (y1 - y0) * (z1 - z0);
    }
    const long long r = r0;
    for (long long z = std::max(b0[2], cz - r); z < std::min(b1[2], cz + r + 1); ++z)
      for (long long y = std::max(b0[1], cy - r); y < std::min(b1[1], cy + r + 1); ++y) {
        const long long rem = r * r - (z - cz) * (z - cz) - (y - cy) * (y - cy);
        if (rem < 0) continue;
        long long dx = static_cast<long long>(std::sqrt(static_cast<double>(rem)));
        while (dx * dx > rem) --dx;
        while ((dx + 1) * (dx + 1) <= rem) ++dx;
        const long long x0 = std::max(b0[0], cx - dx), x1 = std::min(b1[0], cx + dx + 1);
        if (x1 <= x0) continue;
        HashDAG::Box b{u32(x0), u32(y), u32(z), u32(x1), u32(y + 1), u32(z + 1)};
        fill ? d->fill_box(b) : d->clear_box(b);
        voxels += x1 - x0;
      }
  } catch (...) {
    return -1;
  }
  return voxels;
}

long long ref_dag_apply_prim(void *h, int shape, long long cx, long long cy, long long cz,
                             long long r0, long long r1, long long r2, int fill) {
  return ref_dag_apply_prim_clipped(h, shape, cx, cy, cz, r0, r1, r2, fill, nullptr, nullptr);
}

int ref_dag_set_voxel(void *h, u32 x, u32 y, u32 z, int value) {
  try {
    static_cast<HashDAG *>(h)->set_voxel(x, y, z, value != 0);
    return 0;
  } catch (...) {
    return 1;
  }
}

int ref_dag_get_voxel(void *h, u32 x, u32 y, u32 z) {
  try {
    return static_cast<HashDAG *>(h)->get_voxel(x, y, z) ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

u64 ref_dag_node_count(void *h) { return static_cast<HashDAG *>(h)->node_count(); }

// Canonical dump; arrays may be NULL to query sizes.  counts has depth + 1
// entries (nodes per inner level, then leaves).
int ref_dag_export(void *h, u32 *root, u64 *counts, u32 *nodes, u64 cap_words,
                   u64 *leaves, u64 cap_leaves) {
  const HashDAG &d = *static_cast<HashDAG *>(h);
  DagDump dump(d);
  const u32 r = dump.visit(0, d.root_);
  if (root) *root = r;
  u64 words = 0;
  for (u32 l = 0; l < d.depth_; ++l) {
    if (counts) counts[l] = dump.nodes[l].size() / 10;
    words += dump.nodes[l].size();
  }
  if (counts) counts[d.depth_] = dump.leaves.size();
  if (nodes) {
    if (words > cap_words) return 2;
    u64 o = 0;
    for (u32 l = 0; l < d.depth_; ++l)
      for (u32 w : dump.nodes[l]) nodes[o++] = w;
  }
  if (leaves) {
    if (dump.leaves.size() > cap_leaves) return 2;
    for (u64 i = 0; i < dump.leaves.size(); ++i) leaves[i] = dump.leaves[i];
  }
  return 0;
}

// Load the canonical dump (format of ref_dag_export, relative levels
// 0..depth-base) of the cell at level `base` that contains voxel (cx, cy, cz)
// into an empty HashDAG: leaves and nodes are inserted bottom-up with the
// reference's own find_or_append_leaf / find_or_append_node (hash_dag.hpp:
// 535-560), full subtrees become its full_node_ptrs_ / full_leaf_ptr_, and the
// rest of the world stays empty.  Returns 0, or 1 when a bucket overflows.
int ref_dag_import_region(void *h, u32 base, u32 cx, u32 cy, u32 cz, u32 root_id,
                          const u64 *counts, const u32 *nodes, const u64 *leaves) {
  HashDAG &d = *static_cast<HashDAG *>(h);
  const u32 D = d.depth_;
  if (base > D) return 1;
  const u32 L = D - base;
  try {
    std::vector<u32> leaf_ptr(counts[L]);
    for (u64 i = 0; i < counts[L]; ++i) leaf_ptr[i] = d.find_or_append_leaf(leaves[i]);
    std::vector<u64> off(L + 1, 0);
    for (u32 l = 0; l < L; ++l) off[l + 1] = off[l] + counts[l] * 10;
    std::vector<std::vector<u32>> ptr(L);
    auto child_ptr = [&](u32 rl, u32 id) -> u32 {
      if (id == 0) return 0;
      if (id == 1) return rl == L ? d.full_leaf_ptr_ : d.full_node_ptrs_[base + rl];
      return rl == L ? leaf_ptr[id - 2] : ptr[rl][id - 2];
    };
    for (u32 rl = L; rl-- > 0;) {
      ptr[rl].resize(counts[rl]);
      for (u64 i = 0; i < counts[rl]; ++i) {
        const u32 *rec = nodes + off[rl] + 10 * i;
        std::array<u32, 8> children{};
        u32 mask = 0;
        for (u32 c = 0; c < 8; ++c) {
          children[c] = child_ptr(rl + 1, rec[2 + c]);
          if (children[c] != 0) mask |= 1u << c;
        }
        ptr[rl][i] = d.find_or_append_node(base + rl, static_cast<uint8_t>(mask), children);
      }
    }
    u32 sub = child_ptr(0, root_id);
    for (u32 level = base; level > 0; --level) {
      const u32 sh = D + 2 - level; // the parent's split bit
      const u32 c = ((cx >> sh) & 1u) | (((cy >> sh) & 1u) << 1) | (((cz >> sh) & 1u) << 2);
      std::array<u32, 8> children{};
      children[c] = sub;
      sub = sub ? d.find_or_append_node(level - 1, static_cast<uint8_t>(1u << c), children) : 0;
    }
    d.root_ = sub;
  } catch (...) {
    return 1;
  }
  return 0;
}

void *ref_svo_new(u32 depth) {
  try {
    return new SVO(depth);
  } catch (...) {
    return nullptr;
  }
}
void ref_svo_free(void *h) { delete static_cast<SVO *>(h); }

int ref_svo_set_voxel(void *h, u32 x, u32 y, u32 z, int value) {
  try {
    static_cast<SVO *>(h)->set_voxel(x, y, z, value != 0);
    return 0;
  } catch (...) {
    return 1;
  }
}

int ref_svo_get_voxel(void *h, u32 x, u32 y, u32 z) {
  try {
    return static_cast<SVO *>(h)->get_voxel(x, y, z) ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

u64 ref_svo_node_count(void *h) { return static_cast<SVO *>(h)->node_count(); }
u64 ref_svo_leaf_count(void *h) { return static_cast<SVO *>(h)->leaf_count(); }

int ref_svo_export(void *h, u32 *node_count, u32 *leaf_count, u32 *nodes,
                   u32 cap_nodes, u64 *leaves, u32 cap_leaves) {
  SvoDump dump(*static_cast<SVO *>(h));
  dump.visit(0, 0);
  const u32 nn = static_cast<u32>(dump.nodes.size() / 8);
  const u32 nl = static_cast<u32>(dump.leaves.size());
  if (node_count) *node_count = nn;
  if (leaf_count) *leaf_count = nl;
  if (nodes) {
    if (nn > cap_nodes) return 2;
    for (u64 i = 0; i < dump.nodes.size(); ++i) nodes[i] = dump.nodes[i];
  }
  if (leaves) {
    if (nl > cap_leaves) return 2;
    for (u32 i = 0; i < nl; ++i) leaves[i] = dump.leaves[i];
  }
  return 0;
}

} // extern "C"
