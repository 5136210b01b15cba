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
// vx_dag_graph_primitives with an explicit grid (blocks per SM) for the item
// kernels: small served batches want fewer blocks than large edits.
vx_status graph_primitives_grid(vx_dag *d, const vx_primitive *prims, const uint32_t *d_count,
                                uint32_t capacity, uint32_t blocks_per_sm, vx_graph **out);
} // namespace vx::dag
