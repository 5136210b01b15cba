// Terminal edits: whole octree cells and 4^3 bricks, moved by voxel offsets,
// placed or destroyed as one union (svt/cuda/terminal/detail/pipeline.cuh:
// 27-222).
//
// The reference turns its inputs into sorted, pruned cell and brick write
// requests and runs its own allocation / release / collapse passes.  Here
// one kernel turns every input into primitives of fixed count -- a node input
// into one half-open box (an aligned cell, or an unaligned cube when the
// offset is not a multiple of the cell size), a brick into the up to 8 aligned
// leaf masks it straddles -- and the batched edit of the SVO or the Hash DAG
// applies them.  All primitives of a call share one op, so their order does
// not matter and covered or duplicated inputs need no pruning; the batched
// edit already collapses uniform regions and frees what they replace.  The
// primitive count is known on the host, so nothing synchronises before the
// final status read.
#include "common.cuh"
#include "edit_common.cuh"
#include "profile.cuh"

namespace vx::terminal {

constexpr uint32_t kBrickSlots = 8;
constexpr uint32_t kMaxTerminalDepth = 10;

static_assert(sizeof(vx_terminal_node) == 20, "TerminalNodeInput layout");
static_assert(sizeof(vx_terminal_leaf) == 32, "TerminalLeafInput layout");

// A primitive that touches nothing (a leaf mask outside the world).
__device__ __forceinline__ vx_primitive nothing() {
  vx_primitive p{};
  p.c[0] = p.c[1] = p.c[2] = -4;
  p.flags = vx_make_flags(edit::kShapeLeafMask, VX_OP_ADD, 0);
  return p;
}

// Leaf coordinates (in leaves) of the cell at `depth` with path `prefix`, in a
// structure of `depth_max` levels; false for an invalid input.
__device__ __forceinline__ bool cell_origin(uint32_t depth, uint32_t prefix,
                                            uint32_t depth_max, uint32_t &lx,
                                            uint32_t &ly, uint32_t &lz) {
  if (depth > depth_max) return false;
  if (depth < 11u && (prefix >> (3u * depth)) != 0u) return false;
  lx = ly = lz = 0;
  for (uint32_t i = 0; i < depth; ++i) {
    const uint32_t c = (prefix >> (3u * (depth - 1u - i))) & 7u;
    lx = (lx << 1) | (c & 1u);
    ly = (ly << 1) | ((c >> 1) & 1u);
    lz = (lz << 1) | ((c >> 2) & 1u);
  }
  lx <<= depth_max - depth;
  ly <<= depth_max - depth;
  lz <<= depth_max - depth;
  return true;
}

__global__ void to_primitives_kernel(const vx_terminal_node *nodes, uint32_t node_count,
                                     const vx_terminal_leaf *leaves, uint32_t leaf_count,
                                     uint32_t depth_max, uint32_t flags_op,
                                     vx_primitive *out) {
  const int64_t world = int64_t(4) << depth_max;
  const uint64_t total = node_count + static_cast<uint64_t>(leaf_count) * kBrickSlots;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    vx_primitive p = nothing();
    if (i < node_count) {
      const vx_terminal_node in = nodes[i];
      uint32_t lx, ly, lz;
      if (cell_origin(in.depth, in.prefix, depth_max, lx, ly, lz)) {
        const uint32_t side = 4u << (depth_max - in.depth);
        const int64_t o[3] = {int64_t(lx) * 4 + in.offset[0], int64_t(ly) * 4 + in.offset[1],
                              int64_t(lz) * 4 + in.offset[2]};
        // Clip to the world so the box fits the 32-bit primitive fields.
        int64_t lo[3], hi[3];
        bool empty = false;
        for (int a = 0; a < 3; ++a) {
          lo[a] = o[a] < 0 ? 0 : o[a];
          hi[a] = o[a] + side > world ? world : o[a] + side;
          empty |= hi[a] <= lo[a];
        }
        if (!empty) {
          for (int a = 0; a < 3; ++a) {
            p.c[a] = static_cast<int32_t>(lo[a]);
            p.r[a] = static_cast<uint32_t>(hi[a] - lo[a]);
          }
          p.flags = VX_SHAPE_AABB | flags_op;
        }
      }
    } else {
      const uint64_t j = i - node_count;
      const vx_terminal_leaf in = leaves[j / kBrickSlots];
      const uint32_t slot = static_cast<uint32_t>(j % kBrickSlots);
      uint32_t lx, ly, lz;
      if (in.mask64 != 0 && cell_origin(depth_max, in.leaf_prefix, depth_max, lx, ly, lz)) {
        // The moved brick starts at o; slot s is the aligned leaf at
        // floor(o / 4) + (s & 1, s >> 1 & 1, s >> 2 & 1).
        const int64_t o[3] = {int64_t(lx) * 4 + in.offset[0], int64_t(ly) * 4 + in.offset[1],
                              int64_t(lz) * 4 + in.offset[2]};
        int64_t base[3], sh[3];
        for (int a = 0; a < 3; ++a) {
          base[a] = o[a] >= 0 ? o[a] / 4 : -((-o[a] + 3) / 4);
          sh[a] = o[a] - base[a] * 4; // 0..3
        }
        const int64_t leaf[3] = {base[0] + (slot & 1u), base[1] + ((slot >> 1) & 1u),
                                 base[2] + ((slot >> 2) & 1u)};
        uint64_t m = 0;
        bool inside = true;
        for (int a = 0; a < 3; ++a) inside &= leaf[a] >= 0 && leaf[a] * 4 < world;
        if (inside) {
          for (uint32_t b = 0; b < 64; ++b) {
            if (!((in.mask64 >> b) & 1ull)) continue;
            const int64_t v[3] = {(b & 3u) + sh[0], ((b >> 2) & 3u) + sh[1],
                                  ((b >> 4) & 3u) + sh[2]};
            // v is the bit's position relative to leaf `base`; keep the
            // bits that land in this slot's leaf.
            const int64_t q[3] = {v[0] - 4 * int64_t(slot & 1u),
                                  v[1] - 4 * int64_t((slot >> 1) & 1u),
                                  v[2] - 4 * int64_t((slot >> 2) & 1u)};
            if (q[0] < 0 || q[0] > 3 || q[1] < 0 || q[1] > 3 || q[2] < 0 || q[2] > 3) continue;
            m |= 1ull << (q[0] + 4 * q[1] + 16 * q[2]);
          }
        }
        if (m) {
          for (int a = 0; a < 3; ++a) p.c[a] = static_cast<int32_t>(leaf[a] * 4);
          p.r[0] = static_cast<uint32_t>(m);
          p.r[1] = static_cast<uint32_t>(m >> 32);
          p.r[2] = 0;
          p.flags = edit::kShapeLeafMask | flags_op;
        }
      }
    }
    out[i] = p;
  }
}

// Validates and converts; on success *prims / *count describe the batch.
vx_status prepare(uint32_t depth, const vx_terminal_node *nodes, uint32_t node_count,
                  const vx_terminal_leaf *leaves, uint32_t leaf_count, uint32_t op,
                  uint32_t material, void *ws, size_t ws_bytes, cudaStream_t s,
                  vx_primitive **prims, uint32_t *count) {
  if ((nodes == nullptr && node_count != 0) || (leaves == nullptr && leaf_count != 0) || op > 1)
    return VX_ERR_INVALID_VALUE;
  if (ws == nullptr || ws_bytes < vx_terminal_workspace_size(node_count, leaf_count))
    return VX_ERR_INVALID_VALUE;
  if (depth > kMaxTerminalDepth) return VX_ERR_INVALID_VALUE;
  const uint64_t total = node_count + static_cast<uint64_t>(leaf_count) * kBrickSlots;
  if (total > 0xffffffffull) return VX_ERR_INVALID_VALUE;
  *count = static_cast<uint32_t>(total);
  *prims = reinterpret_cast<vx_primitive *>(static_cast<char *>(ws) + 256);
  if (total == 0) return VX_OK;
  const uint32_t flags_op = vx_make_flags(0, op == VX_EDIT_PLACE ? VX_OP_ADD : VX_OP_REMOVE,
                                          op == VX_EDIT_PLACE ? material : 0u);
  const uint32_t grid = static_cast<uint32_t>(
      std::min<uint64_t>((total + edit::kBlock - 1) / edit::kBlock, uint64_t(sm_count()) * 16));
  prof::Scope sc("terminal_to_primitives", s);
  to_primitives_kernel<<<grid, edit::kBlock, 0, s>>>(nodes, node_count, leaves, leaf_count,
                                                     depth, flags_op, *prims);
  return from_cuda(cudaGetLastError());
}

} // namespace vx::terminal

extern "C" {

size_t vx_terminal_workspace_size(uint32_t node_count, uint32_t leaf_count) {
  return 256 + (node_count + static_cast<size_t>(leaf_count) * vx::terminal::kBrickSlots) *
                   sizeof(vx_primitive);
}

vx_status vx_svo_apply_terminal(vx_svo *svo, const vx_terminal_node *nodes,
                                uint32_t node_count, const vx_terminal_leaf *leaves,
                                uint32_t leaf_count, uint32_t op, uint32_t material,
                                void *workspace, size_t workspace_bytes, vx_stream stream) {
  if (svo == nullptr || material > 255) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx_primitive *prims = nullptr;
  uint32_t count = 0;
  VX_TRY(vx::terminal::prepare(vx_svo_depth(svo), nodes, node_count, leaves, leaf_count, op,
                               material ? material : 1u, workspace, workspace_bytes, s,
                               &prims, &count));
  if (count == 0) return VX_OK;
  VX_TRY(vx_svo_apply_primitives(svo, prims, count, stream));
  return vx_svo_status(svo, stream);
}

vx_status vx_dag_apply_terminal(vx_dag *dag, const vx_terminal_node *nodes,
                                uint32_t node_count, const vx_terminal_leaf *leaves,
                                uint32_t leaf_count, uint32_t op, void *workspace,
                                size_t workspace_bytes, vx_stream stream) {
  if (dag == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  vx_primitive *prims = nullptr;
  uint32_t count = 0;
  VX_TRY(vx::terminal::prepare(vx_dag_depth(dag), nodes, node_count, leaves, leaf_count, op,
                               0u, workspace, workspace_bytes, s, &prims, &count));
  if (count == 0) return VX_OK;
  VX_TRY(vx_dag_apply_primitives(dag, prims, count, stream));
  return vx_dag_status(dag, stream);
}

} // extern "C"
