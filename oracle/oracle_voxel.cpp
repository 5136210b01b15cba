// ORACLE - test infrastructure only.  CPU restatement of the reference's
// voxel-editing semantics, used by tests/ as the checker:
//
//   * sequential application: each edit sets or clears every voxel it covers,
//     in order (HashDAG::fill_box / clear_box / set_voxel,
//     algorithm/lib/include/algo/svt/hash_dag.hpp:37-49, 343-533; SVO::
//     set_voxel, svo.hpp:26-91), evaluated voxel by voxel on a dense grid with
//     the reference bench's inside-sphere test (bench_cuda_svt.cu:37-44);
//   * the canonical Hash DAG of an occupancy grid: leaves are 4^3 masks with
//     bit = x + 4y + 16z (hash_dag.hpp:782-801), uniform subtrees collapse to
//     empty / full, equal subtrees are shared (hash_dag.hpp:535-670); dumped
//     in DFS first-visit order (children 0..7) with the GPU item convention
//     [child_mask, fill_mask, child ids] (hash_dag_gpu/detail/node.cuh:266-289);
//   * the canonical SVO of an occupancy / material grid: a node exists iff its
//     region is not uniform (the root always exists), leaves are the
//     non-uniform 4^3 bricks, child words keep bit 30 (child present) and
//     bit 31 (filled when absent) (svo.hpp:11-16, 26-91, 341-376).
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "vx_workload.h"

using u8 = std::uint8_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;

namespace {

// Dense grid of 4^3 leaves at depth D (world side 4 << D).
struct Grid {
  u32 depth;
  u32 side;  // leaves per axis
  std::vector<u64> occ;
  std::vector<u8> mat; // optional, 64 bytes per leaf
  bool materials;

  Grid(u32 d, bool m) : depth(d), side(1u << d), materials(m) {
    occ.assign(static_cast<size_t>(side) * side * side, 0);
    if (m) mat.assign(occ.size() * 64, 0);
  }
  size_t leaf(u32 lx, u32 ly, u32 lz) const {
    return (static_cast<size_t>(lz) * side + ly) * side + lx;
  }
  void set(u32 x, u32 y, u32 z, bool on, u8 m) {
    const size_t l = leaf(x >> 2, y >> 2, z >> 2);
    const u32 bit = (x & 3u) + 4u * (y & 3u) + 16u * (z & 3u);
    if (on) occ[l] |= 1ull << bit;
    else occ[l] &= ~(1ull << bit);
    if (materials) mat[l * 64 + bit] = on ? m : 0;
  }
};

void fill_terrain(Grid &g, const vx_terrain &t, u32 lx0, u32 ly0, u32 lz0,
                  u32 nleaves) {
  // nleaves = cell side in leaves; classification is exact (conservative
  // bounds answer full / empty only when true), leaves are evaluated exactly.
  const u32 c = vx_terrain_classify(&t, lx0 * 4, ly0 * 4, lz0 * 4, nleaves * 4);
  if (c == VX_CELL_EMPTY) return;
  if (c == VX_CELL_FULL && !g.materials) {
    for (u32 z = 0; z < nleaves; ++z)
      for (u32 y = 0; y < nleaves; ++y)
        for (u32 x = 0; x < nleaves; ++x)
          g.occ[g.leaf(lx0 + x, ly0 + y, lz0 + z)] = ~0ull;
    return;
  }
  if (nleaves > 1) {
    const u32 h = nleaves / 2;
    for (u32 k = 0; k < 8; ++k)
      fill_terrain(g, t, lx0 + (k & 1) * h, ly0 + ((k >> 1) & 1) * h,
                   lz0 + ((k >> 2) & 1) * h, h);
    return;
  }
  const size_t l = g.leaf(lx0, ly0, lz0);
  // Voxel by voxel (the definition), not the leaf-mask helper.
  for (u32 z = 0; z < 4; ++z)
    for (u32 y = 0; y < 4; ++y)
      for (u32 x = 0; x < 4; ++x) {
        const u32 vx = lx0 * 4 + x, vy = ly0 * 4 + y, vz = lz0 * 4 + z;
        if (vx_terrain_solid(&t, vx, vy, vz))
          g.set(vx, vy, vz, true, static_cast<u8>(vx_terrain_material(&t, vz)));
      }
  (void)l;
}

void apply_prim(Grid &g, const vx_primitive &p) {
  const int64_t world = int64_t(4) << g.depth;
  int64_t lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    int64_t b0, b1;
    if (vx_prim_shape(&p) == VX_SHAPE_SPHERE) {
      b0 = int64_t(p.c[a]) - p.r[0];
      b1 = int64_t(p.c[a]) + p.r[0];
    } else {
      vx_prim_axis_range(&p, a, &b0, &b1);
    }
    lo[a] = std::max<int64_t>(0, b0);
    hi[a] = std::min<int64_t>(world - 1, b1);
  }
  const bool add = vx_prim_op(&p) == VX_OP_ADD;
  const u8 m = static_cast<u8>(vx_prim_material(&p));
  for (int64_t z = lo[2]; z <= hi[2]; ++z)
    for (int64_t y = lo[1]; y <= hi[1]; ++y)
      for (int64_t x = lo[0]; x <= hi[0]; ++x)
        if (vx_prim_contains_voxel(&p, x, y, z))
          g.set(static_cast<u32>(x), static_cast<u32>(y), static_cast<u32>(z), add, m);
}

// ------------------------------------------------------- canonical DAG --

struct ArrHash {
  size_t operator()(const std::array<u32, 8> &a) const {
    u64 h = 1469598103934665603ull;
    for (u32 v : a) h = (h ^ v) * 1099511628211ull;
    return static_cast<size_t>(h);
  }
};

struct DagBuild {
  u32 depth;
  // per level: node children (8 refs each, 0 empty, 1 full, k+2 = node k)
  std::vector<std::vector<std::array<u32, 8>>> nodes;
  std::vector<u64> leaves;
  u32 root = 0;
};

DagBuild build_dag(const Grid &g) {
  const u32 D = g.depth;
  DagBuild b;
  b.depth = D;
  b.nodes.resize(D);
  // leaf level refs per leaf cell
  std::unordered_map<u64, u32> leaf_ids;
  std::vector<u32> cur(g.occ.size());
  for (size_t i = 0; i < g.occ.size(); ++i) {
    const u64 m = g.occ[i];
    if (m == 0) cur[i] = 0;
    else if (m == ~0ull) cur[i] = 1;
    else {
      auto it = leaf_ids.find(m);
      if (it == leaf_ids.end()) {
        it = leaf_ids.emplace(m, static_cast<u32>(b.leaves.size())).first;
        b.leaves.push_back(m);
      }
      cur[i] = it->second + 2;
    }
  }
  u32 side = g.side;
  for (u32 r = D; r > 0; --r) {
    const u32 l = r - 1;
    const u32 ps = side / 2;
    std::vector<u32> up(static_cast<size_t>(ps) * ps * ps);
    std::unordered_map<std::array<u32, 8>, u32, ArrHash> ids;
    for (u32 z = 0; z < ps; ++z)
      for (u32 y = 0; y < ps; ++y)
        for (u32 x = 0; x < ps; ++x) {
          std::array<u32, 8> ch;
          bool all_e = true, all_f = true;
          for (u32 c = 0; c < 8; ++c) {
            const u32 cx = 2 * x + (c & 1), cy = 2 * y + ((c >> 1) & 1),
                      cz = 2 * z + ((c >> 2) & 1);
            ch[c] = cur[(static_cast<size_t>(cz) * side + cy) * side + cx];
            all_e &= ch[c] == 0;
            all_f &= ch[c] == 1;
          }
          u32 ref;
          if (all_e) ref = 0;
          else if (all_f) ref = 1;
          else {
            auto it = ids.find(ch);
            if (it == ids.end()) {
              it = ids.emplace(ch, static_cast<u32>(b.nodes[l].size())).first;
              b.nodes[l].push_back(ch);
            }
            ref = it->second + 2;
          }
          up[(static_cast<size_t>(z) * ps + y) * ps + x] = ref;
        }
    cur.swap(up);
    side = ps;
  }
  b.root = cur[0];
  return b;
}

struct DagDump {
  const DagBuild &b;
  std::vector<std::vector<int64_t>> ids;
  std::vector<int64_t> leaf_ids;
  std::vector<std::vector<u32>> out;
  std::vector<u64> leaves;
  explicit DagDump(const DagBuild &bb) : b(bb), ids(bb.depth), leaf_ids(bb.leaves.size(), -1), out(bb.depth) {
    for (u32 l = 0; l < bb.depth; ++l) ids[l].assign(bb.nodes[l].size(), -1);
  }
  u32 visit(u32 l, u32 ref) {
    if (ref < 2) return ref;
    if (l == b.depth) {
      int64_t &id = leaf_ids[ref - 2];
      if (id < 0) {
        id = static_cast<int64_t>(leaves.size());
        leaves.push_back(b.leaves[ref - 2]);
      }
      return static_cast<u32>(id) + 2;
    }
    int64_t &id = ids[l][ref - 2];
    if (id >= 0) return static_cast<u32>(id) + 2;
    id = static_cast<int64_t>(out[l].size() / 10);
    const u32 my = static_cast<u32>(id);
    out[l].resize(out[l].size() + 10, 0);
    u32 rec[10] = {0};
    for (u32 c = 0; c < 8; ++c) {
      const u32 cid = visit(l + 1, b.nodes[l][ref - 2][c]);
      rec[2 + c] = cid;
      if (cid == 1) rec[1] |= 1u << c;
      if (cid >= 2) rec[0] |= 1u << c;
    }
    std::memcpy(&out[l][my * 10], rec, sizeof(rec));
    return my + 2;
  }
};

int export_dag(const Grid &g, u32 *root, u64 *counts, u32 *nodes, u64 cap_words,
               u64 *leaves, u64 cap_leaves) {
  const DagBuild b = build_dag(g);
  DagDump d(b);
  const u32 r = d.visit(0, b.root);
  if (root) *root = r;
  u64 words = 0;
  for (u32 l = 0; l < g.depth; ++l) {
    if (counts) counts[l] = d.out[l].size() / 10;
    words += d.out[l].size();
  }
  if (counts) counts[g.depth] = d.leaves.size();
  if (nodes) {
    if (words > cap_words) return 2;
    u64 o = 0;
    for (u32 l = 0; l < g.depth; ++l)
      for (u32 w : d.out[l]) nodes[o++] = w;
  }
  if (leaves) {
    if (d.leaves.size() > cap_leaves) return 2;
    std::copy(d.leaves.begin(), d.leaves.end(), leaves);
  }
  return 0;
}

// ------------------------------------------------------- canonical SVO --

struct SvoDump {
  const Grid &g;
  std::vector<u32> nodes;
  std::vector<u64> leaves;
  std::vector<u8> mats;
  explicit SvoDump(const Grid &gg) : g(gg) {}

  // Uniform value of a cell of nl leaves per side: returns true and the value
  // (0 empty, else material or 1) if every voxel has the same value.
  bool uniform(u32 lx, u32 ly, u32 lz, u32 nl, u32 &value) const {
    bool first = true;
    u32 v0 = 0;
    for (u32 z = 0; z < nl; ++z)
      for (u32 y = 0; y < nl; ++y)
        for (u32 x = 0; x < nl; ++x) {
          const size_t l = g.leaf(lx + x, ly + y, lz + z);
          const u64 m = g.occ[l];
          if (m != 0 && m != ~0ull) return false;
          u32 v;
          if (g.materials) {
            v = g.mat[l * 64];
            for (u32 b = 1; b < 64; ++b)
              if (g.mat[l * 64 + b] != v) return false;
          } else {
            v = m ? 1u : 0u;
          }
          if (first) {
            v0 = v;
            first = false;
          } else if (v != v0) {
            return false;
          }
        }
    value = v0;
    return true;
  }

  u32 visit(u32 lx, u32 ly, u32 lz, u32 nl) {
    const u32 id = static_cast<u32>(nodes.size() / 8);
    nodes.resize(nodes.size() + 8, 0);
    u32 rec[8];
    const u32 h = nl / 2;
    for (u32 c = 0; c < 8; ++c) {
      const u32 cx = lx + (c & 1) * h, cy = ly + ((c >> 1) & 1) * h,
                cz = lz + ((c >> 2) & 1) * h;
      u32 v;
      if (uniform(cx, cy, cz, h, v)) {
        rec[c] = (v ? (1u << 31) : 0u) | (g.materials ? v : 0u);
      } else if (h == 1) {
        const size_t l = g.leaf(cx, cy, cz);
        rec[c] = (1u << 30) | static_cast<u32>(leaves.size());
        leaves.push_back(g.occ[l]);
        if (g.materials) mats.insert(mats.end(), &g.mat[l * 64], &g.mat[l * 64] + 64);
      } else {
        rec[c] = (1u << 30) | visit(cx, cy, cz, h);
      }
    }
    std::memcpy(&nodes[id * 8], rec, sizeof(rec));
    return id;
  }
};

} // namespace

extern "C" {

void *orc_grid_new(u32 depth, int materials) { return new Grid(depth, materials != 0); }
void orc_grid_free(void *g) { delete static_cast<Grid *>(g); }

void orc_grid_terrain(void *gp, const vx_terrain *t) {
  Grid &g = *static_cast<Grid *>(gp);
  vx_terrain tt = *t;
  tt.world_exp = g.depth + 2;
  if (!g.materials) {
    fill_terrain(g, tt, 0, 0, 0, g.side);
    return;
  }
  // with materials every solid voxel needs its band material
  for (u32 lz = 0; lz < g.side; ++lz)
    for (u32 ly = 0; ly < g.side; ++ly)
      for (u32 lx = 0; lx < g.side; ++lx) fill_terrain(g, tt, lx, ly, lz, 1);
}

void orc_grid_apply_prims(void *gp, const vx_primitive *p, u64 n) {
  Grid &g = *static_cast<Grid *>(gp);
  for (u64 i = 0; i < n; ++i) apply_prim(g, p[i]);
}

// Terminal edits (svt/cuda/terminal/detail/count_requests.cuh:13-158,
// emit_requests.cuh:1-484, common.cuh): the cell at (depth, prefix) or the
// brick at the full-depth leaf_prefix, moved by a voxel offset, clipped to
// the world; every covered voxel is set (op 1) or cleared (op 0).  Inputs
// with depth > the grid's depth or prefix bits above 3 * depth are ignored
// (common.cuh terminal_prefix_to_leaf_coord).  Restated per voxel.
struct OrcTerminalNode {
  u32 depth, prefix;
  int32_t offset[3];
};
struct OrcTerminalLeaf {
  u32 leaf_prefix, pad0;
  u64 mask64;
  int32_t offset[3];
  u32 pad1;
};

static bool orc_prefix_origin(u32 depth, u32 prefix, u32 depth_max, int64_t o[3]) {
  if (depth > depth_max) return false;
  if (depth < 11 && (u64(prefix) >> (3 * depth)) != 0) return false;
  u32 c[3] = {0, 0, 0};
  for (u32 i = 0; i < depth; ++i) {
    const u32 child = (prefix >> (3 * (depth - 1 - i))) & 7u;
    for (int a = 0; a < 3; ++a) c[a] = (c[a] << 1) | ((child >> a) & 1u);
  }
  for (int a = 0; a < 3; ++a) o[a] = int64_t(c[a] << (depth_max - depth)) * 4;
  return true;
}

void orc_grid_apply_terminal(void *gp, const OrcTerminalNode *nodes, u64 n_nodes,
                             const OrcTerminalLeaf *leaves, u64 n_leaves, int op,
                             u32 material) {
  Grid &g = *static_cast<Grid *>(gp);
  const int64_t world = int64_t(4) << g.depth;
  const bool add = op != 0;
  const u8 m = add ? static_cast<u8>(material ? material : 1) : 0;
  auto set = [&](int64_t x, int64_t y, int64_t z) {
    if (x < 0 || y < 0 || z < 0 || x >= world || y >= world || z >= world) return;
    g.set(u32(x), u32(y), u32(z), add, m);
  };
  for (u64 i = 0; i < n_nodes; ++i) {
    int64_t o[3];
    if (!orc_prefix_origin(nodes[i].depth, nodes[i].prefix, g.depth, o)) continue;
    const int64_t side = int64_t(4) << (g.depth - nodes[i].depth);
    for (int a = 0; a < 3; ++a) o[a] += nodes[i].offset[a];
    for (int64_t z = std::max<int64_t>(o[2], 0); z < std::min(o[2] + side, world); ++z)
      for (int64_t y = std::max<int64_t>(o[1], 0); y < std::min(o[1] + side, world); ++y)
        for (int64_t x = std::max<int64_t>(o[0], 0); x < std::min(o[0] + side, world); ++x)
          set(x, y, z);
  }
  for (u64 i = 0; i < n_leaves; ++i) {
    int64_t o[3];
    if (!orc_prefix_origin(g.depth, leaves[i].leaf_prefix, g.depth, o)) continue;
    for (u32 b = 0; b < 64; ++b)
      if ((leaves[i].mask64 >> b) & 1ull)
        set(o[0] + (b & 3u) + leaves[i].offset[0], o[1] + ((b >> 2) & 3u) + leaves[i].offset[1],
            o[2] + ((b >> 4) & 3u) + leaves[i].offset[2]);
  }
}

// Plain-path semantics: one op (1 place, 0 destroy) for a voxel list;
// out-of-world voxels are ignored (hash_dag_gpu/edit.cuh:28-29).
void orc_grid_apply_voxels(void *gp, const u32 *xyz, u64 n, int op, u32 material) {
  Grid &g = *static_cast<Grid *>(gp);
  const u32 world = 4u << g.depth;
  for (u64 i = 0; i < n; ++i) {
    const u32 x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (x >= world || y >= world || z >= world) continue;
    g.set(x, y, z, op != 0, static_cast<u8>(material));
  }
}

u64 orc_grid_count(void *gp) {
  const Grid &g = *static_cast<Grid *>(gp);
  u64 c = 0;
  for (u64 m : g.occ) c += static_cast<u64>(__builtin_popcountll(m));
  return c;
}

int orc_grid_get(void *gp, u32 x, u32 y, u32 z) {
  const Grid &g = *static_cast<Grid *>(gp);
  const size_t l = g.leaf(x >> 2, y >> 2, z >> 2);
  const u32 bit = (x & 3u) + 4u * (y & 3u) + 16u * (z & 3u);
  if (g.materials) return g.mat[l * 64 + bit];
  return static_cast<int>((g.occ[l] >> bit) & 1ull);
}

int orc_grid_export_dag(void *gp, u32 *root, u64 *counts, u32 *nodes,
                        u64 cap_words, u64 *leaves, u64 cap_leaves) {
  return export_dag(*static_cast<Grid *>(gp), root, counts, nodes, cap_words,
                    leaves, cap_leaves);
}

int orc_grid_export_svo(void *gp, u32 *node_count, u32 *leaf_count, u32 *nodes,
                        u32 cap_nodes, u64 *leaves, u8 *mats, u32 cap_leaves) {
  const Grid &g = *static_cast<Grid *>(gp);
  SvoDump d(g);
  d.visit(0, 0, 0, g.side);
  const u32 nn = static_cast<u32>(d.nodes.size() / 8);
  const u32 nl = static_cast<u32>(d.leaves.size());
  if (node_count) *node_count = nn;
  if (leaf_count) *leaf_count = nl;
  if (nodes) {
    if (nn > cap_nodes) return 2;
    std::copy(d.nodes.begin(), d.nodes.end(), nodes);
  }
  if (leaves) {
    if (nl > cap_leaves) return 2;
    std::copy(d.leaves.begin(), d.leaves.end(), leaves);
  }
  if (mats && g.materials) std::copy(d.mats.begin(), d.mats.end(), mats);
  return 0;
}

// Final state of single voxels after the terrain (optional) and primitives
// applied in order: the last primitive covering a voxel decides it.
void orc_eval_voxels(const vx_terrain *t, u32 world_exp, const vx_primitive *p,
                     u64 n, const u32 *xyz, u64 count, u8 *out, int materials) {
  vx_terrain tt{};
  if (t) {
    tt = *t;
    tt.world_exp = world_exp;
  }
  for (u64 i = 0; i < count; ++i) {
    const u32 x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    int v = -1;
    for (u64 k = n; k-- > 0;) {
      if (vx_prim_contains_voxel(&p[k], x, y, z)) {
        const bool add = vx_prim_op(&p[k]) == VX_OP_ADD;
        v = add ? (materials ? static_cast<int>(vx_prim_material(&p[k])) : 1) : 0;
        break;
      }
    }
    if (v < 0) {
      if (t && vx_terrain_solid(&tt, x, y, z))
        v = materials ? static_cast<int>(vx_terrain_material(&tt, z)) : 1;
      else
        v = 0;
    }
    out[i] = static_cast<u8>(v);
  }
}

} // extern "C"
