// Internal hooks of the Hash DAG used by the serving loop.
#pragma once

#include "common.cuh"

namespace vx::dag {
// Device address of the DAG's edit header (root, status, counters).
const void *device_header(const vx_dag *d);
// Size of that header in bytes.
size_t header_bytes();
// Root and status in a host copy of the header.
uint32_t header_root(const void *host_header);
uint32_t header_status(const void *host_header);
// Highest fill fraction over all tables (index slots, pools, leaf set) in a
// host copy of the header.
double fill_fraction(const vx_dag *d, const void *host_header);
// Room and use of the tables, per level l = 0..depth (depth = the leaf set):
// nodes an index can hold (half its slots), words a pool can hold (0 for the
// leaf set), and, from a host copy of the header, the nodes and words used.
struct TableRoom {
  uint32_t depth;
  uint64_t node_cap[16], word_cap[16];
  uint64_t nodes[16], words[16];
};
TableRoom table_room(const vx_dag *d, const void *host_header);
// Synchronous copy of the device header into host memory.
vx_status read_header(const vx_dag *d, void *host_header, cudaStream_t s);
// vx_dag_graph_primitives with an explicit grid (blocks per SM) for the item
// kernels: small served batches want fewer blocks than large edits.
vx_status graph_primitives_grid(vx_dag *d, const vx_primitive *prims, const uint32_t *d_count,
                                uint32_t capacity, uint32_t blocks_per_sm, vx_graph **out);
} // namespace vx::dag
