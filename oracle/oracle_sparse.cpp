// ORACLE - test infrastructure only.  A sparse, hash-consed CPU restatement
// of sequential voxel editing, for checking the GPU path at full size (the
// dense Grid of oracle_voxel.cpp stops at 1024^3):
//
//   * the terrain is built top-down: a cell the terrain classification calls
//     full or empty becomes a uniform ref, other cells split, and a 4^3 leaf is
//     evaluated voxel by voxel (its lattice values read once per leaf);
//   * then every primitive is applied in order, recursively, the way the
//     reference's HashDAG::edit_node does it (algorithm/lib/include/algo/svt/
//     hash_dag.hpp:369-443): a cell the primitive misses keeps its subtree, a
//     cell it covers becomes uniform (add: full / its material, remove:
//     empty), any other cell recurses, and at the leaf level the primitive's
//     4^3 mask is OR-ed in or cleared (edit_leaf_parent, :445-533);
//   * nodes and leaves are hash-consed (find_or_append_node / _leaf,
//     :535-670); uniform subtrees collapse to uniform refs, which is the
//     canonical form of the reference's full_node_ptrs_ / kEmptyNode.
//
// The world splits into shards (the cells of one level), each built and
// edited by one thread in its own store: a primitive only changes the shards
// it intersects, so each shard sees the primitives that touch it in order.
// Canonical dumps then walk the shards in DFS order with one content table
// per level across all shards (the same canonical forms as oracle_voxel.cpp:
// DAG = per-level first-visit ids, 10-word records; SVO = pre-order tree).
//
// Values: occupancy (0 empty, 1 full) or, with materials, a byte per voxel
// (0 empty, 1..255 the material of a filled voxel).  The plain voxel path is
// expressed as 1^3 half-open boxes.
#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <thread>
#include <type_traits>
#include <vector>

#include "vx_workload.h"

using u8 = std::uint8_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;

namespace {

inline u64 mix64(u64 x) {
  x ^= x >> 31;
  x *= 0x7fb5d329728ea185ull;
  x ^= x >> 27;
  x *= 0x81dadef4bc2dd44dull;
  x ^= x >> 33;
  return x;
}

using Node = std::array<u32, 8>;
struct MatLeaf {
  u8 v[64];
  bool operator==(const MatLeaf &o) const { return std::memcmp(v, o.v, 64) == 0; }
};

inline u64 hash_of(const Node &n) {
  u64 h = 0x243f6a8885a308d3ull;
  for (u32 w : n) h = mix64(h ^ w);
  return h;
}
inline u64 hash_of(u64 m) { return mix64(m ^ 0x13198a2e03707344ull); }
inline u64 hash_of(const MatLeaf &l) {
  u64 h = 0xa4093822299f31d0ull, w;
  for (int i = 0; i < 8; ++i) {
    std::memcpy(&w, l.v + 8 * i, 8);
    h = mix64(h ^ w);
  }
  return h;
}

// Content-addressed store of items: intern() returns the index of the item
// equal to its argument, appending it on first sight.  Open addressing with
// linear probing at load <= 1/2; a slot holds the item index + 1 in its low
// half and 32 bits of the item's hash in its high half, so a probe reads the
// item itself only when the hashes agree.
template <class Item> struct Interner {
  std::vector<Item> items;
  std::vector<u64> slots; // (hash >> 32) << 32 | (index + 1); 0 = empty
  u64 mask = 0;

  void rehash(size_t n) {
    slots.assign(n, 0);
    mask = n - 1;
    for (size_t i = 0; i < items.size(); ++i) {
      const u64 h = hash_of(items[i]);
      u64 j = h & mask;
      while (slots[j] != 0) j = (j + 1) & mask;
      slots[j] = (h & 0xffffffff00000000ull) | (i + 1);
    }
  }
  // Room for at least n items without growing.
  void reserve(size_t n) {
    items.reserve(n);
    size_t cap = 1024;
    while (cap < 2 * n + 2) cap *= 2;
    if (cap > slots.size()) rehash(cap);
  }
  u32 intern(const Item &it) {
    if ((items.size() + 1) * 2 > slots.size()) rehash(std::max<size_t>(1024, slots.size() * 2));
    const u64 h = hash_of(it);
    const u64 tag = h & 0xffffffff00000000ull;
    for (u64 j = h & mask;; j = (j + 1) & mask) {
      const u64 e = slots[j];
      if (e == 0) {
        items.push_back(it);
        slots[j] = tag | items.size();
        return static_cast<u32>(items.size() - 1);
      }
      if ((e & 0xffffffff00000000ull) == tag && items[(e & 0xffffffffu) - 1] == it)
        return static_cast<u32>((e & 0xffffffffu) - 1);
    }
  }
};

// ------------------------------------------------------------ geometry --

enum Cover { kOut = 0, kIn = 1, kPart = 2 };

// Inclusive voxel range of a box / half-open AABB primitive on axis a.
inline void axis_range(const vx_primitive &p, int a, i64 &lo, i64 &hi) {
  if ((p.flags & 0xffu) == VX_SHAPE_AABB) {
    lo = p.c[a];
    hi = i64(p.c[a]) + i64(p.r[a]) - 1;
  } else {
    lo = i64(p.c[a]) - i64(p.r[a]);
    hi = i64(p.c[a]) + i64(p.r[a]);
  }
}

// How primitive p covers the voxel cube [o, o + n)^3: the nearest and the
// farthest voxel of the cube decide for a sphere (|v - c|^2 <= r^2), the
// per-axis ranges for a box.
inline Cover cover(const vx_primitive &p, const i64 o[3], i64 n) {
  if ((p.flags & 0xffu) == VX_SHAPE_SPHERE) {
    const i64 r2 = i64(p.r[0]) * i64(p.r[0]);
    i64 near2 = 0, far2 = 0;
    for (int a = 0; a < 3; ++a) {
      const i64 lo = o[a], hi = o[a] + n - 1, c = p.c[a];
      const i64 dn = c < lo ? lo - c : (c > hi ? c - hi : 0);
      const i64 df = std::max(c - lo, hi - c);
      near2 += dn * dn;
      far2 += df * df;
    }
    if (near2 > r2) return kOut;
    return far2 <= r2 ? kIn : kPart;
  }
  bool in = true;
  for (int a = 0; a < 3; ++a) {
    i64 lo, hi;
    axis_range(p, a, lo, hi);
    if (hi < lo || hi < o[a] || lo > o[a] + n - 1) return kOut;
    in = in && lo <= o[a] && hi >= o[a] + n - 1;
  }
  return in ? kIn : kPart;
}

// Voxels of the 4^3 leaf at o that p covers (bit = x + 4y + 16z).
inline u64 leaf_cover(const vx_primitive &p, const i64 o[3]) {
  u64 m = 0;
  if ((p.flags & 0xffu) == VX_SHAPE_SPHERE) {
    const i64 r2 = i64(p.r[0]) * i64(p.r[0]);
    for (int z = 0; z < 4; ++z)
      for (int y = 0; y < 4; ++y) {
        const i64 dy = o[1] + y - p.c[1], dz = o[2] + z - p.c[2];
        const i64 rem = r2 - dy * dy - dz * dz;
        if (rem < 0) continue;
        for (int x = 0; x < 4; ++x) {
          const i64 dx = o[0] + x - p.c[0];
          if (dx * dx <= rem) m |= 1ull << (x + 4 * y + 16 * z);
        }
      }
    return m;
  }
  i64 lo[3], hi[3];
  for (int a = 0; a < 3; ++a) axis_range(p, a, lo[a], hi[a]);
  for (int z = 0; z < 4; ++z)
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) {
        const i64 v[3] = {o[0] + x, o[1] + y, o[2] + z};
        bool in = true;
        for (int a = 0; a < 3; ++a) in = in && v[a] >= lo[a] && v[a] <= hi[a];
        if (in) m |= 1ull << (x + 4 * y + 16 * z);
      }
  return m;
}

// Lattice values of the lattice cells that contain a cube: the 4 corner
// values of each height octave's cell and the 8 of the cave noise's cell.
// Valid for every cube inside those cells (side <= the finest spacing,
// aligned), so a subtree's classifications and leaf evaluations read the
// lattice once instead of hashing it per query.
struct Lattice {
  i64 li[3], lj[3];  // octave cell indices
  i64 h[3][4];       // v00, v10, v01, v11 per octave
  i64 ci, cj, ck;    // cave cell
  i64 cave[8];       // corner k = (i + (k & 1), j + (k >> 1 & 1), k + (k >> 2))
};

struct TerrainEval {
  const vx_terrain &t;
  i64 s, den, c, thr;
  explicit TerrainEval(const vx_terrain &tt)
      : t(tt), s(tt.scale), den(vx_terrain_hden(&tt)), c(8 * i64(tt.scale)),
        thr(55 * c * c * c * VX_NOISE_ONE) {}

  // Cubes of this side or less (aligned) lie in one cell of every lattice.
  i64 cached_side() const { return t.caves ? c : 16 * s; }

  void fetch(i64 x0, i64 y0, i64 z0, Lattice &L) const {
    for (u32 o = 0; o < 3; ++o) {
      const i64 sp = (64 * s) >> o;
      L.li[o] = x0 / sp;
      L.lj[o] = y0 / sp;
      L.h[o][0] = vx_lattice_value(t.seed, 1u + o, L.li[o], L.lj[o], 0);
      L.h[o][1] = vx_lattice_value(t.seed, 1u + o, L.li[o] + 1, L.lj[o], 0);
      L.h[o][2] = vx_lattice_value(t.seed, 1u + o, L.li[o], L.lj[o] + 1, 0);
      L.h[o][3] = vx_lattice_value(t.seed, 1u + o, L.li[o] + 1, L.lj[o] + 1, 0);
    }
    if (t.caves) {
      L.ci = x0 / c;
      L.cj = y0 / c;
      L.ck = z0 / c;
      for (int k = 0; k < 8; ++k)
        L.cave[k] = vx_lattice_value(t.seed, 4u, L.ci + (k & 1), L.cj + ((k >> 1) & 1),
                                     L.ck + (k >> 2));
    }
  }
  // Inside the cells of L the fractional coordinates of x are
  // x % sp = (x0 % sp) + (x - x0), so each query needs one modulo per axis.
  // Height numerator of column (fx[o], fy[o]) given per-octave fractions
  // (vx_terrain_hnum).
  i64 hnum_f(const Lattice &L, const i64 fx[3], const i64 fy[3]) const {
    i64 acc = 0;
    for (u32 o = 0; o < 3; ++o) {
      const i64 sp = (64 * s) >> o;
      const i64 gx = sp - fx[o], gy = sp - fy[o];
      acc += (i64(1) << o) * (gx * gy * L.h[o][0] + fx[o] * gy * L.h[o][1] +
                              gx * fy[o] * L.h[o][2] + fx[o] * fy[o] * L.h[o][3]);
    }
    return acc;
  }
  // Cave numerator (vx_noise3_num, stream 4) factored along x, then y, then
  // z: sum_k wx wy wz v_k = sum_c wz_c sum_b wy_b sum_a wx_a v_abc, exact in
  // 64-bit integers; w0 / w1 are the z = 0 / 1 planes at fractions (fx, fy).
  void cave_xy(const Lattice &L, i64 fx, i64 fy, i64 &w0, i64 &w1) const {
    const i64 gx = c - fx, gy = c - fy;
    const i64 u00 = gx * L.cave[0] + fx * L.cave[1]; // (y 0, z 0)
    const i64 u10 = gx * L.cave[2] + fx * L.cave[3]; // (y 1, z 0)
    const i64 u01 = gx * L.cave[4] + fx * L.cave[5]; // (y 0, z 1)
    const i64 u11 = gx * L.cave[6] + fx * L.cave[7]; // (y 1, z 1)
    w0 = gy * u00 + fy * u10;
    w1 = gy * u01 + fy * u11;
  }
  i64 cave_z(i64 w0, i64 w1, i64 fz) const { return (c - fz) * w0 + fz * w1; }
  bool carved(i64 cn) const { return 100 * cn > thr; }

  // vx_terrain_classify for a cube inside the cells of L: the multilinear
  // interpolants take their extrema over the cube at its corners.
  u32 classify(const Lattice &L, i64 x0, i64 y0, i64 z0, i64 n) const {
    i64 hlo = 0, hhi = 0;
    for (u32 o = 0; o < 3; ++o) {
      const i64 sp = (64 * s) >> o;
      const i64 fx0 = x0 % sp, fy0 = y0 % sp;
      i64 mn = 0, mx = 0;
      for (int k = 0; k < 4; ++k) {
        const i64 fx = fx0 + ((k & 1) ? n - 1 : 0), fy = fy0 + ((k & 2) ? n - 1 : 0);
        const i64 gx = sp - fx, gy = sp - fy;
        const i64 v = gx * gy * L.h[o][0] + fx * gy * L.h[o][1] + gx * fy * L.h[o][2] +
                      fx * fy * L.h[o][3];
        mn = (k == 0 || v < mn) ? v : mn;
        mx = (k == 0 || v > mx) ? v : mx;
      }
      hlo += (i64(1) << o) * mn;
      hhi += (i64(1) << o) * mx;
    }
    const i64 z1 = z0 + n - 1;
    const bool all_below = z1 * den < 128 * s * den + 40 * s * hlo;
    const bool none_below = z0 * den >= 128 * s * den + 40 * s * hhi;
    if (none_below) return VX_CELL_EMPTY;
    if (!t.caves) return all_below ? VX_CELL_FULL : VX_CELL_MIXED;
    const i64 fx0 = x0 % c, fy0 = y0 % c, fz0 = z0 % c;
    i64 clo = 0, chi = 0;
    for (int k = 0; k < 4; ++k) {
      i64 w0, w1;
      cave_xy(L, fx0 + ((k & 1) ? n - 1 : 0), fy0 + ((k & 2) ? n - 1 : 0), w0, w1);
      for (int zz = 0; zz < 2; ++zz) {
        const i64 v = cave_z(w0, w1, fz0 + (zz ? n - 1 : 0));
        clo = (k == 0 && zz == 0) || v < clo ? v : clo;
        chi = (k == 0 && zz == 0) || v > chi ? v : chi;
      }
    }
    if (100 * clo > thr) return VX_CELL_EMPTY;
    return (all_below && 100 * chi <= thr) ? VX_CELL_FULL : VX_CELL_MIXED;
  }

  // Values of the 4^3 leaf at (x0, y0, z0) inside the cells of L: 0 empty,
  // else 1 or (materials) the band material; bit / byte = x + 4y + 16z.
  void leaf(const Lattice &L, i64 x0, i64 y0, i64 z0, bool mats, u8 out[64]) const {
    i64 fx0[3], fy0[3];
    for (u32 o = 0; o < 3; ++o) {
      const i64 sp = (64 * s) >> o;
      fx0[o] = x0 % sp;
      fy0[o] = y0 % sp;
    }
    const i64 cx0 = x0 % c, cy0 = y0 % c, cz0 = z0 % c;
    u8 band[4];
    for (int z = 0; z < 4; ++z)
      band[z] = static_cast<u8>(mats ? vx_terrain_material(&t, u32(z0 + z)) : 1u);
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) {
        i64 fx[3], fy[3];
        for (u32 o = 0; o < 3; ++o) {
          fx[o] = fx0[o] + x;
          fy[o] = fy0[o] + y;
        }
        const i64 rhs = 128 * s * den + 40 * s * hnum_f(L, fx, fy);
        i64 w0 = 0, w1 = 0;
        if (t.caves) cave_xy(L, cx0 + x, cy0 + y, w0, w1);
        for (int z = 0; z < 4; ++z) {
          bool solid = (z0 + z) * den < rhs;
          if (solid && t.caves) solid = !carved(cave_z(w0, w1, cz0 + z));
          out[x + 4 * y + 16 * z] = solid ? band[z] : 0u;
        }
      }
  }
};

// ------------------------------------------------------------- a store --

// One shard's hash-consed nodes and leaves.  Refs below kU are uniform
// values; ref kU + k is item k of its level's table.
template <bool Mat> struct Store {
  static constexpr u32 kU = Mat ? 256u : 2u;
  using Leaf = std::conditional_t<Mat, MatLeaf, u64>;
  u32 depth; // leaf level
  std::vector<Interner<Node>> nodes;
  Interner<Leaf> leaves;

  explicit Store(u32 d) : depth(d), nodes(d) {}

  u32 node(u32 level, const Node &ch) {
    bool uniform = ch[0] < kU;
    for (int k = 1; k < 8 && uniform; ++k) uniform = ch[k] == ch[0];
    if (uniform) return ch[0];
    return nodes[level].intern(ch) + kU;
  }
  Node children(u32 level, u32 ref) const {
    Node n;
    if (ref < kU) n.fill(ref);
    else n = nodes[level].items[ref - kU];
    return n;
  }
  // leaf values as 64 bytes (occupancy: 0 / 1)
  void leaf_values(u32 ref, u8 out[64]) const {
    if (ref < kU) {
      std::memset(out, static_cast<int>(ref), 64);
      return;
    }
    if constexpr (Mat) {
      std::memcpy(out, leaves.items[ref - kU].v, 64);
    } else {
      const u64 m = leaves.items[ref - kU];
      for (int b = 0; b < 64; ++b) out[b] = static_cast<u8>((m >> b) & 1u);
    }
  }
  u32 leaf(const u8 v[64]) {
    bool uniform = true;
    for (int b = 1; b < 64 && uniform; ++b) uniform = v[b] == v[0];
    if (uniform) return v[0];
    if constexpr (Mat) {
      MatLeaf l;
      std::memcpy(l.v, v, 64);
      return leaves.intern(l) + kU;
    } else {
      u64 m = 0;
      for (int b = 0; b < 64; ++b) m |= u64(v[b] != 0) << b;
      return leaves.intern(m) + kU;
    }
  }
  u64 leaf_mask(u32 ref) const {
    if (ref < kU) return ref ? ~0ull : 0ull;
    if constexpr (Mat) {
      u64 m = 0;
      for (int b = 0; b < 64; ++b) m |= u64(leaves.items[ref - kU].v[b] != 0) << b;
      return m;
    } else {
      return leaves.items[ref - kU];
    }
  }
};

template <bool Mat> struct Builder {
  Store<Mat> &s;
  const vx_terrain *t; // null: empty world
  TerrainEval te;
  static const vx_terrain kNone;

  Builder(Store<Mat> &st, const vx_terrain *tt) : s(st), t(tt), te(tt ? *tt : kNone) {}

  i64 side(u32 level) const { return i64(4) << (s.depth - level); }

  // Terrain subtree of the cell at `level`; L holds the lattice cells of the
  // cell once it is small enough to lie inside them.
  u32 terrain(u32 level, const i64 o[3], const Lattice *L = nullptr) {
    if (t == nullptr) return 0;
    const i64 n = side(level);
    Lattice mine;
    if (L == nullptr && n <= te.cached_side()) {
      te.fetch(o[0], o[1], o[2], mine);
      L = &mine;
    }
    const u32 c = L ? te.classify(*L, o[0], o[1], o[2], n)
                    : vx_terrain_classify(t, u32(o[0]), u32(o[1]), u32(o[2]), u32(n));
    if (c == VX_CELL_EMPTY) return 0;
    if (c == VX_CELL_FULL) {
      if (!Mat) return 1;
      const i64 band = 8 * i64(t->scale);
      if (o[2] / band == (o[2] + n - 1) / band) return vx_terrain_material(t, u32(o[2]));
    }
    if (level == s.depth) {
      u8 v[64];
      te.leaf(*L, o[0], o[1], o[2], Mat, v);
      return s.leaf(v);
    }
    Node ch;
    const i64 h = n / 2;
    for (u32 k = 0; k < 8; ++k) {
      const i64 co[3] = {o[0] + (k & 1) * h, o[1] + ((k >> 1) & 1) * h, o[2] + ((k >> 2) & 1) * h};
      ch[k] = terrain(level + 1, co, L);
    }
    return s.node(level, ch);
  }

  // Sequential application of one primitive (value: what it writes).
  u32 edit(u32 level, u32 ref, const i64 o[3], const vx_primitive &p, u32 value) {
    const i64 n = side(level);
    const Cover c = cover(p, o, n);
    if (c == kOut) return ref;
    if (c == kIn) return value;
    if (level == s.depth) {
      u8 v[64];
      s.leaf_values(ref, v);
      const u64 m = leaf_cover(p, o);
      for (int b = 0; b < 64; ++b)
        if ((m >> b) & 1u) v[b] = static_cast<u8>(value);
      return s.leaf(v);
    }
    const Node old = s.children(level, ref);
    Node nw;
    bool changed = false;
    const i64 h = n / 2;
    for (u32 k = 0; k < 8; ++k) {
      const i64 co[3] = {o[0] + (k & 1) * h, o[1] + ((k >> 1) & 1) * h, o[2] + ((k >> 2) & 1) * h};
      nw[k] = edit(level + 1, old[k], co, p, value);
      changed = changed || nw[k] != old[k];
    }
    return changed ? s.node(level, nw) : ref;
  }
};
template <bool Mat> const vx_terrain Builder<Mat>::kNone = {0, 1, 0, 2};

// What an add primitive writes (the material, 1 when it names none) and a
// remove writes (0); occupancy stores write 1 / 0.
inline u32 prim_value(const vx_primitive &p, bool mats) {
  if (((p.flags >> 8) & 0xffu) != VX_OP_ADD) return 0;
  if (!mats) return 1;
  const u32 m = (p.flags >> 16) & 0xffu;
  return m ? m : 1u;
}

// ---------------------------------------------------------- the world --

// A global ref: a uniform value, a node of the top levels (above the shard
// level, no dedup), or a ref inside one shard's store.
struct GRef {
  int32_t shard; // -1: top node or uniform
  u32 ref;
};

template <bool Mat> struct World {
  static constexpr u32 kU = Store<Mat>::kU;
  u32 depth;        // leaf level of the whole world
  u32 base;         // level of the region cell (0 = whole world)
  i64 origin[3];    // region origin (voxels)
  u32 shard_level;  // absolute level of the shards (>= base)
  std::vector<std::unique_ptr<Store<Mat>>> stores;
  std::vector<u32> roots;
  std::vector<std::vector<std::array<GRef, 8>>> top; // per level base..shard_level-1
  GRef root{-1, 0};

  i64 side(u32 level) const { return i64(4) << (depth - level); }

  // Cell origin of shard k (k's base-8 digits, most significant first, are
  // the child indices from the region cell down).
  void shard_origin(u64 k, i64 o[3]) const {
    for (int a = 0; a < 3; ++a) o[a] = origin[a];
    const u32 levels = shard_level - base;
    for (u32 i = 0; i < levels; ++i) {
      const u32 child = u32(k >> (3 * (levels - 1 - i))) & 7u;
      const i64 h = side(base + i) / 2;
      for (int a = 0; a < 3; ++a) o[a] += ((child >> a) & 1u) * h;
    }
  }

  void run(const vx_terrain *t, const vx_primitive *p, u64 n, int threads) {
    const u64 shards = u64(1) << (3 * (shard_level - base));
    stores.resize(shards);
    roots.assign(shards, 0);
    std::atomic<u64> next{0};
    auto work = [&] {
      for (;;) {
        const u64 k = next.fetch_add(1);
        if (k >= shards) return;
        stores[k] = std::make_unique<Store<Mat>>(depth);
        Builder<Mat> b(*stores[k], t);
        i64 o[3];
        shard_origin(k, o);
        u32 r = b.terrain(shard_level, o);
        const i64 sn = side(shard_level);
        for (u64 i = 0; i < n; ++i) {
          if (cover(p[i], o, sn) == kOut) continue;
          r = b.edit(shard_level, r, o, p[i], prim_value(p[i], Mat));
        }
        roots[k] = r;
      }
    };
    const int nt = std::max(1, std::min<int>(threads, int(shards)));
    std::vector<std::thread> pool;
    for (int i = 1; i < nt; ++i) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    // top levels, bottom-up (uniform cells collapse)
    top.assign(shard_level - base, {});
    std::vector<GRef> cur(shards);
    for (u64 k = 0; k < shards; ++k)
      cur[k] = roots[k] < kU ? GRef{-1, roots[k]} : GRef{int32_t(k), roots[k]};
    for (u32 l = shard_level; l > base; --l) {
      std::vector<GRef> up(cur.size() / 8);
      auto &lev = top[l - 1 - base];
      for (size_t i = 0; i < up.size(); ++i) {
        std::array<GRef, 8> ch;
        bool uniform = true;
        for (u32 c = 0; c < 8; ++c) {
          ch[c] = cur[8 * i + c];
          uniform = uniform && ch[c].shard < 0 && ch[c].ref < kU && ch[c].ref == ch[0].ref;
        }
        if (uniform) {
          up[i] = ch[0];
        } else {
          lev.push_back(ch);
          up[i] = GRef{-1, kU + u32(lev.size() - 1)};
        }
      }
      cur.swap(up);
    }
    root = cur[0];
  }

  // children of a global ref at `level`
  std::array<GRef, 8> children(u32 level, GRef g) const {
    std::array<GRef, 8> out;
    if (g.shard < 0) {
      if (g.ref < kU) {
        out.fill(g);
        return out;
      }
      return top[level - base][g.ref - kU];
    }
    const Node n = stores[g.shard]->children(level, g.ref);
    for (u32 c = 0; c < 8; ++c)
      out[c] = n[c] < kU ? GRef{-1, n[c]} : GRef{g.shard, n[c]};
    return out;
  }
};

// Canonical Hash DAG dump of the region (occupancy): per level, nodes in
// first-visit order of a DFS with children 0..7, 10-word records
// [child_mask, fill_mask, child ids] (0 empty, 1 full, k + 2 = node k of the
// next level / leaf k); equal subtrees share one id.
template <bool Mat> struct DagCanon {
  const World<Mat> &w;
  std::vector<Interner<Node>> levels;
  Interner<u64> leaves;
  std::vector<std::vector<std::vector<u32>>> memo; // [shard][level][index]
  std::vector<std::vector<u32>> leaf_memo;         // [shard][leaf index]

  explicit DagCanon(const World<Mat> &ww) : w(ww), levels(ww.depth - ww.base) {
    memo.resize(w.stores.size());
    leaf_memo.resize(w.stores.size());
    std::vector<size_t> bound(w.depth - w.base, 0);
    size_t leaf_bound = 0;
    for (size_t k = 0; k < w.stores.size(); ++k) {
      if (!w.stores[k]) continue;
      memo[k].resize(w.depth);
      for (u32 l = w.shard_level; l < w.depth; ++l) {
        memo[k][l].assign(w.stores[k]->nodes[l].items.size(), 0xffffffffu);
        bound[l - w.base] += w.stores[k]->nodes[l].items.size();
      }
      leaf_bound += w.stores[k]->leaves.items.size();
      leaf_memo[k].assign(w.stores[k]->leaves.items.size(), 0xffffffffu);
    }
    for (u32 l = w.base; l < w.shard_level; ++l) bound[l - w.base] += w.top[l - w.base].size();
    // distinct contents are at most the shards' items together
    for (size_t l = 0; l < bound.size(); ++l) levels[l].reserve(bound[l]);
    leaves.reserve(leaf_bound);
  }
  u32 uniform_id(u32 v) const { return v ? 1u : 0u; }

  u32 visit(u32 level, GRef g) {
    if (g.shard < 0 && g.ref < World<Mat>::kU) return uniform_id(g.ref);
    if (level == w.depth) {
      u32 &lid = leaf_memo[g.shard][g.ref - World<Mat>::kU];
      if (lid == 0xffffffffu) {
        const u64 m = w.stores[g.shard]->leaf_mask(g.ref);
        lid = m == 0 ? 0u : (m == ~0ull ? 1u : leaves.intern(m) + 2);
      }
      return lid;
    }
    u32 *slot = nullptr;
    if (g.shard >= 0) {
      slot = &memo[g.shard][level][g.ref - World<Mat>::kU];
      if (*slot != 0xffffffffu) return *slot;
    }
    const auto ch = w.children(level, g);
    Node ids;
    for (u32 c = 0; c < 8; ++c) ids[c] = visit(level + 1, ch[c]);
    u32 id;
    bool uniform = ids[0] < 2;
    for (int c = 1; c < 8 && uniform; ++c) uniform = ids[c] == ids[0];
    if (uniform) id = ids[0]; // a material-uniform-free occupancy region
    else id = levels[level - w.base].intern(ids) + 2;
    if (slot) *slot = id;
    return id;
  }
};

// Canonical SVO dump of the region: a node exists iff its region is not
// uniform (the region's root always exists); pre-order node ids, leaves in
// first-visit order; child words = (1 << 30) | index for a node or leaf,
// else (filled << 31) | material (materials only).
template <bool Mat> struct SvoCanon {
  const World<Mat> &w;
  std::vector<u32> nodes;
  std::vector<u64> leaves;
  std::vector<u8> mats;
  explicit SvoCanon(const World<Mat> &ww) : w(ww) {}

  u32 visit(u32 level, GRef g) {
    const u32 id = u32(nodes.size() / 8);
    nodes.resize(nodes.size() + 8, 0);
    const auto ch = w.children(level, g);
    for (u32 c = 0; c < 8; ++c) {
      u32 word;
      if (ch[c].shard < 0 && ch[c].ref < World<Mat>::kU) {
        const u32 v = ch[c].ref;
        word = (v ? (1u << 31) : 0u) | (Mat ? v : 0u);
      } else if (level + 1 == w.depth) {
        word = (1u << 30) | u32(leaves.size());
        const Store<Mat> &s = *w.stores[ch[c].shard];
        leaves.push_back(s.leaf_mask(ch[c].ref));
        if constexpr (Mat) {
          const u8 *v = s.leaves.items[ch[c].ref - World<Mat>::kU].v;
          mats.insert(mats.end(), v, v + 64);
        }
      } else {
        word = (1u << 30) | visit(level + 1, ch[c]);
      }
      nodes[size_t(id) * 8 + c] = word;
    }
    return id;
  }
};

// A canonical DAG dump, kept so that the size query and the copy-out calls
// share one traversal.
struct DagDump {
  u32 root = 0;
  std::vector<u64> counts;
  std::vector<u32> nodes;
  std::vector<u64> leaves;
};

struct Handle {
  bool mats;
  std::unique_ptr<World<false>> occ;
  std::unique_ptr<World<true>> mat;
  std::unique_ptr<DagDump> dag;
};

template <bool Mat>
std::unique_ptr<World<Mat>> make_world(u32 depth, const vx_terrain *t, const vx_primitive *p,
                                       u64 n, u32 base, const u32 cell[3], u32 shard_levels,
                                       int threads) {
  auto w = std::make_unique<World<Mat>>();
  w->depth = depth;
  w->base = base;
  const i64 s = i64(4) << (depth - base);
  for (int a = 0; a < 3; ++a) w->origin[a] = (i64(cell[a]) / s) * s;
  w->shard_level = std::min(depth, base + shard_levels);
  w->run(t, p, n, threads);
  return w;
}

template <bool Mat> std::unique_ptr<DagDump> dump_dag(const World<Mat> &w) {
  DagCanon<Mat> d(w);
  auto out = std::make_unique<DagDump>();
  out->root = d.visit(w.base, w.root);
  const u32 L = w.depth - w.base;
  for (u32 l = 0; l < L; ++l) {
    out->counts.push_back(d.levels[l].items.size());
    for (const Node &ids : d.levels[l].items) {
      u32 cm = 0, fm = 0;
      for (u32 c = 0; c < 8; ++c) {
        if (ids[c] >= 2) cm |= 1u << c;
        if (ids[c] == 1) fm |= 1u << c;
      }
      out->nodes.push_back(cm);
      out->nodes.push_back(fm);
      out->nodes.insert(out->nodes.end(), ids.begin(), ids.end());
    }
    std::vector<Node>().swap(d.levels[l].items); // release as we go
  }
  out->counts.push_back(d.leaves.items.size());
  out->leaves = d.leaves.items;
  return out;
}

int export_dag(const DagDump &d, u32 *root, u64 *counts, u32 *nodes, u64 cap_words,
               u64 *leaves, u64 cap_leaves) {
  if (root) *root = d.root;
  if (counts) std::copy(d.counts.begin(), d.counts.end(), counts);
  if (nodes) {
    if (d.nodes.size() > cap_words) return 2;
    std::copy(d.nodes.begin(), d.nodes.end(), nodes);
  }
  if (leaves) {
    if (d.leaves.size() > cap_leaves) return 2;
    std::copy(d.leaves.begin(), d.leaves.end(), leaves);
  }
  return 0;
}

template <bool Mat>
int export_svo(const World<Mat> &w, u64 *node_count, u64 *leaf_count, u32 *nodes, u64 cap_nodes,
               u64 *leaves, u8 *mats, u64 cap_leaves) {
  SvoCanon<Mat> d(w);
  d.visit(w.base, w.root);
  const u64 nn = d.nodes.size() / 8, nl = d.leaves.size();
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
  if (mats && Mat) std::copy(d.mats.begin(), d.mats.end(), mats);
  return 0;
}

// Occupancy masks of the leaves in a box of leaves (leaf coordinates
// [lo, lo + n) inside the region), x fastest.
template <bool Mat>
void leaf_block(const World<Mat> &w, const u32 lo[3], const u32 n[3], u64 *out) {
  const u64 total = u64(n[0]) * n[1] * n[2];
  for (u64 i = 0; i < total; ++i) {
    const u32 l[3] = {lo[0] + u32(i % n[0]), lo[1] + u32((i / n[0]) % n[1]),
                      lo[2] + u32(i / (u64(n[0]) * n[1]))};
    GRef g = w.root;
    u64 m = 0;
    bool done = false;
    for (u32 level = w.base; level < w.depth && !done; ++level) {
      if (g.shard < 0 && g.ref < World<Mat>::kU) {
        m = g.ref ? ~0ull : 0ull;
        done = true;
        break;
      }
      const u32 sh = w.depth - level - 1; // child bit of leaf coordinates
      const u32 c = ((l[0] >> sh) & 1u) | (((l[1] >> sh) & 1u) << 1) | (((l[2] >> sh) & 1u) << 2);
      g = w.children(level, g)[c];
    }
    if (!done) {
      if (g.shard < 0) m = g.ref < World<Mat>::kU ? (g.ref ? ~0ull : 0ull) : 0ull;
      else m = w.stores[g.shard]->leaf_mask(g.ref);
    }
    out[i] = m;
  }
}

// First solid voxel along a ray (the semantics of vx_dag_raycast, restated
// over the sparse world): the ray is clipped to the world box, then it steps
// from cell to cell, each step finding the largest uniform cell (or leaf
// voxel) that holds the current voxel; a solid one is the hit, otherwise the
// ray leaves it through the side with the smallest exit parameter (ties x,
// y, z) into the next voxel, whose other coordinates are floor(o + t d) kept
// inside the cell and not moving backwards.  Single-precision operations,
// each rounded once (no contraction), in the order of the GPU code.
// Output: voxel x, y, z, face (0 X+ .. 5 Z-, 6 no hit), t as float bits.
template <bool Mat>
void raycast(const World<Mat> &w, const float *ray, u32 out[5]) {
  const float *o = ray, *d = ray + 3;
  const float t_max = ray[6];
  const u32 no_hit[5] = {~0u, ~0u, ~0u, 6u, 0xbf800000u}; // t = -1.0f
  std::memcpy(out, no_hit, sizeof(no_hit));
  const u32 D = w.depth;
  const int32_t W = 4 << D;
  const float Wf = static_cast<float>(W);
  float t0 = 0.0f, t1 = std::numeric_limits<float>::infinity();
  int entry = -1;
  for (int a = 0; a < 3; ++a) {
    if (d[a] == 0.0f) {
      if (!(o[a] >= 0.0f && o[a] < Wf)) return;
      continue;
    }
    const float ta = (0.0f - o[a]) / d[a];
    const float tb = (Wf - o[a]) / d[a];
    const float tn = ta < tb ? ta : tb, tf = ta < tb ? tb : ta;
    if (tn > t0) {
      t0 = tn;
      entry = a;
    }
    if (tf < t1) t1 = tf;
  }
  if (!(t0 < t1) || !(t0 <= t_max)) return;
  int32_t vox[3];
  for (int a = 0; a < 3; ++a) {
    if (a == entry) {
      vox[a] = d[a] > 0.0f ? 0 : W - 1;
    } else {
      const float prod = t0 * d[a];
      float f = std::floor(o[a] + prod);
      f = f < 0.0f ? 0.0f : (f > Wf - 1.0f ? Wf - 1.0f : f);
      vox[a] = static_cast<int32_t>(f);
    }
  }
  u32 face = entry < 0 ? 0u : (d[entry] > 0.0f ? 2u * entry + 1u : 2u * entry);
  float t = t0;
  const u32 limit = 3u * static_cast<u32>(W) + 8u;
  for (u32 step = 0; step < limit; ++step) {
    // the largest uniform cell or the leaf holding vox
    GRef g = w.root;
    u32 level = 0;
    bool uniform = g.shard < 0 && g.ref < World<Mat>::kU;
    while (!uniform && level < D) {
      const u32 sh = D + 1 - level;
      const u32 c = ((u32(vox[0]) >> sh) & 1u) | (((u32(vox[1]) >> sh) & 1u) << 1) |
                    (((u32(vox[2]) >> sh) & 1u) << 2);
      g = w.children(level, g)[c];
      ++level;
      uniform = g.shard < 0 && g.ref < World<Mat>::kU;
    }
    int32_t side;
    if (uniform) {
      side = g.ref != 0 ? 0 : (4 << (D - level));
    } else {
      const u64 m = w.stores[g.shard]->leaf_mask(g.ref);
      const u32 bit = u32(vox[0] & 3) + 4u * u32(vox[1] & 3) + 16u * u32(vox[2] & 3);
      side = ((m >> bit) & 1u) ? 0 : 1;
    }
    if (side == 0) {
      out[0] = u32(vox[0]);
      out[1] = u32(vox[1]);
      out[2] = u32(vox[2]);
      out[3] = face;
      std::memcpy(&out[4], &t, 4);
      return;
    }
    int32_t cmin[3];
    for (int a = 0; a < 3; ++a) cmin[a] = vox[a] & ~(side - 1);
    float tx = 0.0f;
    int ax = -1;
    for (int a = 0; a < 3; ++a) {
      if (d[a] == 0.0f) continue;
      const float b = static_cast<float>(d[a] > 0.0f ? cmin[a] + side : cmin[a]);
      const float ta = (b - o[a]) / d[a];
      if (ax < 0 || ta < tx) {
        tx = ta;
        ax = a;
      }
    }
    if (ax < 0 || !(tx <= t_max)) return;
    const int32_t nv = d[ax] > 0.0f ? cmin[ax] + side : cmin[ax] - 1;
    if (nv < 0 || nv >= W) return;
    for (int b = 0; b < 3; ++b) {
      if (b == ax || d[b] == 0.0f) continue;
      const float lo = static_cast<float>(d[b] > 0.0f ? vox[b] : cmin[b]);
      const float hi = static_cast<float>(d[b] > 0.0f ? cmin[b] + side - 1 : vox[b]);
      const float prod = tx * d[b];
      float f = std::floor(o[b] + prod);
      f = f < lo ? lo : (f > hi ? hi : f);
      vox[b] = static_cast<int32_t>(f);
    }
    vox[ax] = nv;
    t = tx;
    face = d[ax] > 0.0f ? 2u * ax + 1u : 2u * ax;
  }
}

} // namespace

extern "C" {

// Rays (8 floats each: origin, dir, t_max, unused) through the whole world
// (base 0); hits: 5 words each (see raycast above).
void orc_sparse_raycast(void *hp, const float *rays, u64 n, u32 *hits) {
  const Handle &h = *static_cast<Handle *>(hp);
  for (u64 i = 0; i < n; ++i) {
    if (h.mats) raycast(*h.mat, rays + 8 * i, hits + 5 * i);
    else raycast(*h.occ, rays + 8 * i, hits + 5 * i);
  }
}

// Build the terrain (t may be null: empty world) of a 4 << depth world and
// apply n primitives in order, restricted to the cell at level `base` that
// contains voxel `cell` (base 0: the whole world).  The region is split into
// 8^shard_levels shards handled by up to `threads` threads.
void *orc_sparse_run(u32 depth, const vx_terrain *t, const vx_primitive *p, u64 n, int materials,
                     u32 base, const u32 *cell, u32 shard_levels, int threads) {
  if (base > depth) return nullptr;
  vx_terrain tt{};
  if (t) {
    tt = *t;
    tt.world_exp = depth + 2;
  }
  const u32 zero[3] = {0, 0, 0};
  const u32 *c = cell ? cell : zero;
  auto *h = new Handle{materials != 0, nullptr, nullptr};
  if (h->mats)
    h->mat = make_world<true>(depth, t ? &tt : nullptr, p, n, base, c, shard_levels, threads);
  else
    h->occ = make_world<false>(depth, t ? &tt : nullptr, p, n, base, c, shard_levels, threads);
  return h;
}

void orc_sparse_free(void *h) { delete static_cast<Handle *>(h); }

// Canonical Hash DAG dump of the region (counts has depth - base + 1 entries).
int orc_sparse_export_dag(void *hp, u32 *root, u64 *counts, u32 *nodes, u64 cap_words,
                          u64 *leaves, u64 cap_leaves) {
  Handle &h = *static_cast<Handle *>(hp);
  if (!h.dag) h.dag = h.mats ? dump_dag(*h.mat) : dump_dag(*h.occ);
  return export_dag(*h.dag, root, counts, nodes, cap_words, leaves, cap_leaves);
}

// Canonical SVO dump of the region (mats: 64 bytes per leaf, materials only).
int orc_sparse_export_svo(void *hp, u64 *node_count, u64 *leaf_count, u32 *nodes, u64 cap_nodes,
                          u64 *leaves, u8 *mats, u64 cap_leaves) {
  const Handle &h = *static_cast<Handle *>(hp);
  return h.mats ? export_svo(*h.mat, node_count, leaf_count, nodes, cap_nodes, leaves, mats,
                             cap_leaves)
                : export_svo(*h.occ, node_count, leaf_count, nodes, cap_nodes, leaves, mats,
                             cap_leaves);
}

// Leaf occupancy masks of the leaf box [lo, lo + n) (leaf coordinates of the
// whole world), x fastest; the box must lie inside the region.
void orc_sparse_leaf_block(void *hp, const u32 *lo, const u32 *n, u64 *out) {
  const Handle &h = *static_cast<Handle *>(hp);
  if (h.mats) leaf_block(*h.mat, lo, n, out);
  else leaf_block(*h.occ, lo, n, out);
}

// Self-check of the terrain evaluation of the sparse build: the number of
// voxels of the leaves at the given origins where the cached-lattice
// evaluation differs from vx_terrain_solid / vx_terrain_material, plus the
// number of cubes (the leaf and its aligned ancestors up to the cached side)
// whose cached classification differs from vx_terrain_classify.
u64 orc_terrain_leaf_mismatches(const vx_terrain *t, const u32 *origins, u64 count, int mats) {
  TerrainEval e(*t);
  u64 bad = 0;
  for (u64 i = 0; i < count; ++i) {
    const u32 *o = origins + 3 * i;
    Lattice L;
    e.fetch(o[0], o[1], o[2], L);
    u8 v[64];
    e.leaf(L, o[0], o[1], o[2], mats != 0, v);
    for (int b = 0; b < 64; ++b) {
      const u32 x = o[0] + (b & 3), y = o[1] + ((b >> 2) & 3), z = o[2] + (b >> 4);
      const u32 want = vx_terrain_solid(t, x, y, z)
                           ? (mats ? vx_terrain_material(t, z) : 1u)
                           : 0u;
      bad += v[b] != want;
    }
    for (i64 n = 4; n <= e.cached_side(); n *= 2) {
      const i64 q[3] = {o[0] / n * n, o[1] / n * n, o[2] / n * n};
      Lattice Lq;
      e.fetch(q[0], q[1], q[2], Lq);
      bad += e.classify(Lq, q[0], q[1], q[2], n) !=
             vx_terrain_classify(t, u32(q[0]), u32(q[1]), u32(q[2]), u32(n));
    }
  }
  return bad;
}

// Self-check of the terrain classification used to prune the build: for each
// cube (x, y, z, n), 1 if a FULL / EMPTY answer contradicts a voxel of the
// cube (evaluated one by one), else 0.
u64 orc_terrain_classify_mismatches(const vx_terrain *t, const u32 *cubes, u64 count) {
  u64 bad = 0;
  for (u64 i = 0; i < count; ++i) {
    const u32 *q = cubes + 4 * i;
    const u32 c = vx_terrain_classify(t, q[0], q[1], q[2], q[3]);
    if (c == VX_CELL_MIXED) continue;
    bool wrong = false;
    for (u32 z = 0; z < q[3] && !wrong; ++z)
      for (u32 y = 0; y < q[3] && !wrong; ++y)
        for (u32 x = 0; x < q[3] && !wrong; ++x)
          wrong = vx_terrain_solid(t, q[0] + x, q[1] + y, q[2] + z) != (c == VX_CELL_FULL);
    bad += wrong;
  }
  return bad;
}

} // extern "C"

extern "C" {

// The seeded workload generators of vx_workload.h, compiled into the oracle
// so that CPU-only users (the timed reference baseline) need no GPU library.
void orc_generate_primitives(const vx_edit_mix *mix, u64 seed, u64 stream, u64 count,
                             vx_primitive *out) {
  vx_generate_primitives_host(mix, seed, stream, count, out);
}

u64 orc_generate_requests(const vx_edit_mix *mix, u64 seed, double rate, double seconds,
                          double zipf_s, u32 max_size, u64 max_requests, u64 *arrival_ns,
                          u32 *sizes, u64 max_prims, vx_primitive *prims, u64 *total_prims) {
  return vx_generate_requests_host(mix, seed, rate, seconds, zipf_s, max_size, max_requests,
                                   arrival_ns, sizes, max_prims, prims, total_prims);
}

} // extern "C"
