"""Torch-facing wrappers over the C ABI (mirror of the reference operators).

Each function takes CUDA tensors, allocates the workspace the C call asks for
(the reference's ``*_workspace_size`` + caller-owned workspace contract),
launches on the current torch stream and raises VoxelError on failure.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import check, lib

__all__ = [
    "stream_handle", "ptr", "exclusive_sum", "inclusive_sum", "sort_pairs",
    "workspace_status", "SlabHashSet", "SlabHashMap", "CuckooMap", "ItemSet", "PRIM_DTYPE",
    "make_flags", "prims_to_device", "voxels_to_device", "HashDag",
    "generate_primitives", "config_c1_edits", "config_c3_edits",
    "config_c4_edits", "rasterize", "Svo", "Server", "generate_requests",
    "COMPLETION_DTYPE", "TERMINAL_NODE_DTYPE", "TERMINAL_LEAF_DTYPE", "cell_prefix",
    "terminal_nodes", "terminal_leaves", "records_to_device",
    "tuning", "tuning_options", "set_tuning", "reset_tuning", "Graph", "LEAF_COMMAND_DTYPE", "RAY_DTYPE", "HIT_DTYPE",
]


def tuning() -> dict:
    """Current launch-shape knobs {name: value} (vx_tuning_*)."""
    out = {}
    for i in range(lib().vx_tuning_count()):
        name = lib().vx_tuning_name(i)
        v = C.c_int64()
        check(lib().vx_tuning_get(name, C.byref(v)), "vx_tuning_get")
        out[name.decode()] = v.value
    return out


def tuning_options(name: str) -> list[int]:
    n = C.c_uint32()
    check(lib().vx_tuning_options(name.encode(), None, 0, C.byref(n)), "vx_tuning_options")
    vals = (C.c_int64 * n.value)()
    check(lib().vx_tuning_options(name.encode(), vals, n.value, C.byref(n)),
          "vx_tuning_options")
    return list(vals)


def set_tuning(name: str, value: int) -> None:
    check(lib().vx_tuning_set(name.encode(), int(value)), f"vx_tuning_set({name}={value})")


def reset_tuning() -> None:
    check(lib().vx_tuning_reset(), "vx_tuning_reset")


# The current stream's raw handle without building a torch.cuda.Stream object
# (a few microseconds per call, which per-call edits feel).
_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_device = getattr(torch._C, "_cuda_getDevice", None)


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    if stream is None and _raw_stream is not None and _cur_device is not None:
        return _raw_stream(_cur_device())
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def _scan(data: torch.Tensor, inclusive: bool,
          workspace: torch.Tensor | None = None) -> torch.Tensor:
    n = data.numel()
    need = lib().vx_scan_workspace_size(n)
    ws = workspace if workspace is not None else _workspace(need, data.device)
    if data.dtype in (torch.int32, torch.uint32):
        fn = (lib().vx_scan_inclusive_sum_u32 if inclusive
              else lib().vx_scan_exclusive_sum_u32)
    elif data.dtype in (torch.int64, torch.uint64) and not inclusive:
        fn = lib().vx_scan_exclusive_sum_u64
    else:
        raise TypeError(f"unsupported scan dtype {data.dtype}")
    check(fn(ptr(data), n, ptr(ws), ws.numel(), stream_handle()),
          "scan")
    return data


def exclusive_sum(data: torch.Tensor,
                  workspace: torch.Tensor | None = None) -> torch.Tensor:
    """In-place exclusive prefix sum with wrapping u32/u64 arithmetic
    (algo::cuda::scan::exclusive_sum, cuda/scan/scan.cuh:139-151)."""
    return _scan(data, False, workspace)


def inclusive_sum(data: torch.Tensor,
                  workspace: torch.Tensor | None = None) -> torch.Tensor:
    """In-place inclusive prefix sum (cuda/scan/scan.cuh:123-135)."""
    return _scan(data, True, workspace)


def sort_pairs(keys: torch.Tensor, values: torch.Tensor | None = None,
               key_bits: int | None = None,
               workspace: torch.Tensor | None = None):
    """Stable in-place radix sort by the low ``key_bits`` bits of ``keys``
    (u32 / u64 stored in int32 / int64 tensors), permuting ``values`` (u32)
    alongside (algo::cuda::sort::sort_by_key, cuda/sort/sort.cuh:118-128)."""
    n = keys.numel()
    kb = keys.element_size()
    if key_bits is None:
        key_bits = 8 * kb
    if values is not None and (values.numel() != n or values.element_size() != 4):
        raise ValueError("values must be a u32 array of the same length")
    need = lib().vx_sort_workspace_size(n, kb)
    ws = workspace if workspace is not None else _workspace(need, keys.device)
    fn = lib().vx_sort_pairs_u64 if kb == 8 else lib().vx_sort_pairs_u32
    check(fn(ptr(keys), ptr(values), n, key_bits, ptr(ws), ws.numel(),
             stream_handle()), "sort_pairs")
    return keys, values


def workspace_status(workspace: torch.Tensor) -> int:
    """Synchronise and return the device status a scan/sort left in its
    workspace (0 = ok, VX_ERR_TIMEOUT if a bounded wait gave up)."""
    return lib().vx_workspace_status(ptr(workspace), stream_handle())


class SlabHashSet:
    """u64 slab hash set (BasicSlabHashSetU32 widened to u64 keys,
    cuda/hash_table/slab_hash/set/host.cuh:13-121)."""

    def __init__(self, bucket_count: int, slab_capacity: int):
        h = C.c_void_p()
        check(lib().vx_slab_set_create(bucket_count, slab_capacity, C.byref(h)),
              "vx_slab_set_create")
        self._h = h
        self._free = lib().vx_slab_set_destroy
        self.bucket_count = bucket_count
        self.slab_capacity = slab_capacity

    def device_view(self):
        """View for user kernels (voxel_b200_device.cuh vx_slab_set_contains_warp)."""
        from . import vx_slab_set_view
        v = vx_slab_set_view()
        check(lib().vx_slab_set_device_view(self._h, C.byref(v)), "vx_slab_set_device_view")
        return v

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    @property
    def nbytes(self) -> int:
        return lib().vx_slab_set_bytes(self._h)

    def clear(self):
        check(lib().vx_slab_set_clear(self._h, stream_handle()), "slab clear")

    def insert(self, keys: torch.Tensor, statuses: torch.Tensor | None = None):
        check(lib().vx_slab_set_insert(self._h, ptr(keys), keys.numel(),
                                       ptr(statuses), stream_handle()),
              "slab insert")
        return statuses

    def contains(self, keys: torch.Tensor, out: torch.Tensor | None = None,
                 statuses: torch.Tensor | None = None):
        if out is None:
            out = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
        check(lib().vx_slab_set_contains(self._h, ptr(keys), keys.numel(),
                                         ptr(out), ptr(statuses),
                                         stream_handle()), "slab contains")
        return out

    def erase(self, keys: torch.Tensor, statuses: torch.Tensor | None = None):
        check(lib().vx_slab_set_erase(self._h, ptr(keys), keys.numel(),
                                      ptr(statuses), stream_handle()),
              "slab erase")
        return statuses


class SlabHashMap:
    """u32 -> u32 slab hash map (SlabHashMapU32,
    cuda/hash_table/slab_hash/map/host.cuh)."""

    def __init__(self, bucket_count: int, slab_capacity: int):
        h = C.c_void_p()
        check(lib().vx_slab_map_create(bucket_count, slab_capacity, C.byref(h)),
              "vx_slab_map_create")
        self._h = h
        self._free = lib().vx_slab_map_destroy

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    @property
    def nbytes(self) -> int:
        return lib().vx_slab_map_bytes(self._h)

    def clear(self):
        check(lib().vx_slab_map_clear(self._h, stream_handle()), "slab map clear")

    def insert_or_replace(self, keys: torch.Tensor, values: torch.Tensor,
                          statuses: torch.Tensor | None = None):
        check(lib().vx_slab_map_insert_or_replace(self._h, ptr(keys), ptr(values),
                                                  keys.numel(), ptr(statuses),
                                                  stream_handle()), "slab map insert")
        return statuses

    def find(self, keys: torch.Tensor, out: torch.Tensor | None = None,
             statuses: torch.Tensor | None = None):
        if out is None:
            out = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
        check(lib().vx_slab_map_find(self._h, ptr(keys), keys.numel(), ptr(out),
                                     ptr(statuses), stream_handle()), "slab map find")
        return out

    def erase_all(self, keys: torch.Tensor, statuses: torch.Tensor | None = None):
        check(lib().vx_slab_map_erase_all(self._h, ptr(keys), keys.numel(), ptr(statuses),
                                          stream_handle()), "slab map erase")
        return statuses


class ItemSet:
    """Content-addressed fixed-width item store (AccelerationHashSet32,
    cuda/hash_table/acceleration_hash/set/host.cuh); pointers = index + 1."""

    def __init__(self, width: int, max_items: int):
        h = C.c_void_p()
        check(lib().vx_itemset_create(width, max_items, C.byref(h)), "vx_itemset_create")
        self._h = h
        self._free = lib().vx_itemset_destroy
        self.width = width

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    def _op(self, fn, items, name):
        n = items.numel() // self.width
        ptrs = torch.empty(n, dtype=torch.int32, device=items.device)
        st = torch.empty(n, dtype=torch.int32, device=items.device)
        check(fn(self._h, ptr(items), n, ptr(ptrs), ptr(st), stream_handle()), name)
        return ptrs, st

    def find(self, items: torch.Tensor):
        return self._op(lib().vx_itemset_find, items, "itemset find")

    def find_or_insert(self, items: torch.Tensor):
        return self._op(lib().vx_itemset_find_or_insert, items, "itemset find_or_insert")

    def insert_unique_unchecked(self, items: torch.Tensor):
        return self._op(lib().vx_itemset_insert_unique_unchecked, items, "itemset insert")

    def read(self, ptrs: torch.Tensor):
        n = ptrs.numel()
        out = torch.empty(n * self.width, dtype=torch.int32, device=ptrs.device)
        st = torch.empty(n, dtype=torch.int32, device=ptrs.device)
        check(lib().vx_itemset_read(self._h, ptr(ptrs), n, ptr(out), ptr(st), stream_handle()),
              "itemset read")
        return out, st

    def count(self) -> int:
        v = C.c_uint64(0)
        check(lib().vx_itemset_count(self._h, C.byref(v), stream_handle()), "itemset count")
        return v.value


class CuckooMap:
    """u64 -> u32 cuckoo map with 4 hash functions and bounded eviction
    (cuda/cuckoo_hash.cuh:54-120 widened to inline u64 keys)."""

    def __init__(self, slot_count: int, max_evictions: int = 1000):
        h = C.c_void_p()
        check(lib().vx_cuckoo_create(slot_count, max_evictions, C.byref(h)),
              "vx_cuckoo_create")
        self._h = h
        self._free = lib().vx_cuckoo_destroy
        self.slot_count = slot_count

    def device_view(self):
        """View for user kernels (voxel_b200_device.cuh vx_cuckoo_find)."""
        from . import vx_cuckoo_view
        v = vx_cuckoo_view()
        check(lib().vx_cuckoo_device_view(self._h, C.byref(v)), "vx_cuckoo_device_view")
        return v

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    @property
    def nbytes(self) -> int:
        return lib().vx_cuckoo_bytes(self._h)

    def clear(self):
        check(lib().vx_cuckoo_clear(self._h, stream_handle()), "cuckoo clear")

    def insert(self, keys: torch.Tensor, values: torch.Tensor | None = None,
               statuses: torch.Tensor | None = None):
        check(lib().vx_cuckoo_insert(self._h, ptr(keys), ptr(values),
                                     keys.numel(), ptr(statuses),
                                     stream_handle()), "cuckoo insert")
        return statuses

    def find(self, keys: torch.Tensor, out: torch.Tensor | None = None):
        if out is None:
            out = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
        check(lib().vx_cuckoo_find(self._h, ptr(keys), keys.numel(), ptr(out),
                                   stream_handle()), "cuckoo find")
        return out

    def dropped(self) -> int:
        v = C.c_uint64(0)
        check(lib().vx_cuckoo_dropped(self._h, C.byref(v), stream_handle()),
              "cuckoo dropped")
        return v.value


PRIM_DTYPE = np.dtype([("c", "<i4", 3), ("r", "<u4", 3), ("flags", "<u4"),
                       ("reserved", "<u4")])
# Rays and hits of vx_dag_raycast (the hit is the engine's raycast result words).
RAY_DTYPE = np.dtype([("origin", "<f4", 3), ("dir", "<f4", 3), ("t_max", "<f4"),
                      ("reserved", "<u4")])
HIT_DTYPE = np.dtype([("voxel", "<u4", 3), ("face", "<u4"), ("t", "<f4")])
# The voxel engine's LeafEditCommand (20 bytes, #[repr(C)]).
LEAF_COMMAND_DTYPE = np.dtype([("leaf_x", "<u4"), ("leaf_y", "<u4"), ("leaf_z", "<u4"),
                               ("voxel_data_low", "<u4"), ("voxel_data_high", "<u4")])


def make_flags(shape: int, op: int, material: int = 0) -> int:
    return shape | (op << 8) | (material << 16)


def prims_to_device(prims: np.ndarray, device) -> torch.Tensor:
    """vx_primitive records (PRIM_DTYPE) -> int32 [n, 8] CUDA tensor."""
    a = np.ascontiguousarray(prims, PRIM_DTYPE)
    return torch.from_numpy(a.view(np.int32).reshape(-1, 8).copy()).to(device)


def voxels_to_device(xyz: np.ndarray, device) -> torch.Tensor:
    a = np.ascontiguousarray(xyz, np.uint32).reshape(-1, 3)
    return torch.from_numpy(a.view(np.int32)).to(device)


# Terminal edit inputs (TerminalNodeInput / TerminalLeafInput,
# svt/cuda/terminal/types.cuh:15-31).
TERMINAL_NODE_DTYPE = np.dtype([("depth", "<u4"), ("prefix", "<u4"), ("offset", "<i4", 3)])
TERMINAL_LEAF_DTYPE = np.dtype([("leaf_prefix", "<u4"), ("pad0", "<u4"), ("mask64", "<u8"),
                                ("offset", "<i4", 3), ("pad1", "<u4")])
assert TERMINAL_NODE_DTYPE.itemsize == 20 and TERMINAL_LEAF_DTYPE.itemsize == 32


def cell_prefix(x: int, y: int, z: int, level: int) -> int:
    """Path of the cell (x, y, z) at `level` (cell units): 3 bits per level,
    the root's child in the highest triple, child = x | y << 1 | z << 2
    (make_leaf_key, svt/cuda/detail/geometry.cuh:12-24, at any level)."""
    p = 0
    for i in range(level - 1, -1, -1):
        p = (p << 3) | ((x >> i) & 1) | (((y >> i) & 1) << 1) | (((z >> i) & 1) << 2)
    return p


def terminal_nodes(rows) -> np.ndarray:
    """[(depth, prefix, ox, oy, oz), ...] -> TERMINAL_NODE_DTYPE records."""
    a = np.zeros(len(rows), TERMINAL_NODE_DTYPE)
    for i, (d, p, ox, oy, oz) in enumerate(rows):
        a[i] = (d, p, (ox, oy, oz))
    return a


def terminal_leaves(rows) -> np.ndarray:
    """[(leaf_prefix, mask64, ox, oy, oz), ...] -> TERMINAL_LEAF_DTYPE records."""
    a = np.zeros(len(rows), TERMINAL_LEAF_DTYPE)
    for i, (p, m, ox, oy, oz) in enumerate(rows):
        a[i] = (p, 0, m, (ox, oy, oz), 0)
    return a


def records_to_device(records: np.ndarray, device) -> torch.Tensor:
    """Any record array -> uint8 CUDA tensor holding its bytes."""
    a = np.ascontiguousarray(records)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(device)


def _apply_terminal(fn, h, nodes, leaves, extra, workspace, device):
    nn = 0 if nodes is None else nodes.numel() // TERMINAL_NODE_DTYPE.itemsize
    nl = 0 if leaves is None else leaves.numel() // TERMINAL_LEAF_DTYPE.itemsize
    ws = workspace
    if ws is None:
        ws = torch.empty(lib().vx_terminal_workspace_size(nn, nl), dtype=torch.uint8,
                         device=device)
    return fn(h, ptr(nodes) if nn else None, nn, ptr(leaves) if nl else None, nl, *extra,
              ptr(ws), ws.numel(), stream_handle())


class Graph:
    """A captured edit (vx_*_graph_*): launch() replays it with one launch.
    Keeps the captured buffers alive; the structure must outlive it."""

    def __init__(self, handle, keep):
        self._h = handle
        self._keep = keep

    def launch(self) -> None:
        check(lib().vx_graph_launch(self._h, stream_handle()), "vx_graph_launch")

    @property
    def kernels(self) -> int:
        n = C.c_uint64()
        check(lib().vx_graph_kernels(self._h, C.byref(n)), "vx_graph_kernels")
        return n.value

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().vx_graph_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _graph_primitives(fn, owner, prims, device_count, capacity):
    n = prims.numel() // 8
    cap = capacity if capacity is not None else n
    if cap > n:
        raise ValueError("capacity exceeds the primitive buffer")
    h = C.c_void_p()
    check(fn(owner._h, ptr(prims), ptr(device_count), cap, C.byref(h)), "graph capture")
    return Graph(h, (owner, prims, device_count))


class HashDag:
    """Hash DAG resident on the GPU (HashDagGpu / DeviceHashDagGpu,
    hash_dag_gpu/storage.cuh:16-105, widened to depth 1..14)."""

    def __init__(self, depth: int, max_nodes: int = 1 << 20, arena_bytes: int = 0):
        from . import vx_dag_config
        cfg = vx_dag_config(depth, 0, max_nodes, arena_bytes)
        h = C.c_void_p()
        check(lib().vx_dag_create(C.byref(cfg), C.byref(h)), "vx_dag_create")
        self._h = h
        self._free = lib().vx_dag_destroy
        self.depth = depth

    def device_view(self):
        """View for user kernels (voxel_b200_device.cuh vx_dag_get_voxel)."""
        from . import vx_dag_view
        v = vx_dag_view()
        check(lib().vx_dag_device_view(self._h, C.byref(v)), "vx_dag_device_view")
        return v

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    @property
    def world(self) -> int:
        return 4 << self.depth

    def reset(self):
        check(lib().vx_dag_reset(self._h, stream_handle()), "vx_dag_reset")

    def workspace_size(self, count: int) -> int:
        return lib().vx_dag_voxel_workspace_size(count)

    def apply_voxels(self, voxels: torch.Tensor, op: int,
                     workspace: torch.Tensor | None = None) -> int:
        """Plain path: place (op=1) or destroy (op=0) a voxel list
        (hash_dag_gpu::apply_voxel_edits, hash_dag_gpu/edit.cuh:21-41).
        Returns the status (0 or an error code) like the reference."""
        n = voxels.numel() // 3
        ws = workspace
        if ws is None and n:
            ws = torch.empty(self.workspace_size(n), dtype=torch.uint8,
                             device=voxels.device)
        return lib().vx_dag_apply_voxels(self._h, ptr(voxels) if n else None, n,
                                         op, ptr(ws) if n else None,
                                         ws.numel() if n else 0, stream_handle())

    def apply_terminal(self, nodes: torch.Tensor | None, leaves: torch.Tensor | None,
                       op: int, workspace: torch.Tensor | None = None,
                       device="cuda") -> int:
        """Terminal edit (place_/destroy_terminal_edits): byte tensors of
        TERMINAL_NODE_DTYPE / TERMINAL_LEAF_DTYPE records; returns the status."""
        return _apply_terminal(lib().vx_dag_apply_terminal, self._h, nodes, leaves, (op,),
                               workspace, device)

    def graph_primitives(self, prims: torch.Tensor, device_count: torch.Tensor | None = None,
                         capacity: int | None = None) -> "Graph":
        """Capture the batched edit of `prims` (int32 [n, 8]) as a CUDA graph;
        with device_count (one int32 on the device) each launch edits that
        many primitives (at most capacity)."""
        return _graph_primitives(lib().vx_dag_graph_primitives, self, prims, device_count,
                                 capacity)

    def graph_voxels(self, voxels: torch.Tensor, op: int,
                     workspace: torch.Tensor | None = None) -> "Graph":
        """Capture the plain path (sort, merge, rebuild) for a voxel list."""
        n = voxels.numel() // 3
        ws = workspace if workspace is not None else torch.empty(
            self.workspace_size(n), dtype=torch.uint8, device=voxels.device)
        h = C.c_void_p()
        check(lib().vx_dag_graph_voxels(self._h, ptr(voxels), n, op, ptr(ws), ws.numel(),
                                        C.byref(h)), "vx_dag_graph_voxels")
        return Graph(h, (self, voxels, ws))

    def save(self, path) -> None:
        """Checkpoint: the canonical dump as a file (vx_dag_save)."""
        check(lib().vx_dag_save(self._h, str(path).encode(), stream_handle()), "vx_dag_save")

    def load(self, path) -> int:
        """Resume from a file written by save(); returns the status."""
        return lib().vx_dag_load(self._h, str(path).encode(), stream_handle())

    def apply_primitives(self, prims: torch.Tensor) -> None:
        """Batched path: primitives applied as if in order; asynchronous
        (check with status())."""
        n = prims.numel() // 8
        check(lib().vx_dag_apply_primitives(self._h, ptr(prims) if n else None,
                                            n, stream_handle()),
              "vx_dag_apply_primitives")

    def status(self) -> int:
        return lib().vx_dag_status(self._h, stream_handle())

    def build_terrain(self, seed: int, scale: int, caves: bool) -> None:
        from . import vx_terrain
        t = vx_terrain(seed, scale, int(caves), self.depth + 2)
        check(lib().vx_dag_build_terrain(self._h, C.byref(t), stream_handle()),
              "vx_dag_build_terrain")

    def query(self, voxels: torch.Tensor) -> torch.Tensor:
        n = voxels.numel() // 3
        out = torch.empty(n, dtype=torch.uint8, device=voxels.device)
        check(lib().vx_dag_query(self._h, ptr(voxels), n, ptr(out), stream_handle()),
              "vx_dag_query")
        return out

    def compact(self) -> None:
        """Drop superseded nodes (copy-on-write garbage); content unchanged."""
        check(lib().vx_dag_compact(self._h, stream_handle()), "vx_dag_compact")

    def copy_from(self, other: "HashDag") -> None:
        """Device-side snapshot restore: take other's complete table state."""
        check(lib().vx_dag_copy(self._h, other._h, stream_handle()), "vx_dag_copy")

    def stats(self):
        from . import vx_dag_stats
        st = vx_dag_stats()
        check(lib().vx_dag_get_stats(self._h, C.byref(st), stream_handle()),
              "vx_dag_get_stats")
        return st

    def apply_leaf_commands(self, cmds: torch.Tensor, op: int,
                            workspace: torch.Tensor | None = None) -> int:
        """The voxel engine's leaf edit commands (LEAF_COMMAND_DTYPE records
        in a device tensor): masks OR-merged per leaf, then placed (op=1) or
        cleared (op=0).  Returns the status."""
        n = cmds.numel() * cmds.element_size() // LEAF_COMMAND_DTYPE.itemsize
        ws = workspace
        if ws is None:
            ws = torch.empty(max(lib().vx_leaf_command_workspace_size(n), 1),
                             dtype=torch.uint8, device=cmds.device)
        return lib().vx_dag_apply_leaf_commands(self._h, ptr(cmds), n, op, ptr(ws), ws.numel(),
                                                stream_handle())

    def raycast(self, rays: torch.Tensor) -> torch.Tensor:
        """First solid voxel of each ray (RAY_DTYPE records in a device tensor):
        HIT_DTYPE records (voxel, face, t) as a uint8 device tensor."""
        n = rays.numel() * rays.element_size() // RAY_DTYPE.itemsize
        out = torch.empty(max(n, 1) * HIT_DTYPE.itemsize, dtype=torch.uint8, device=rays.device)
        check(lib().vx_dag_raycast(self._h, ptr(rays), n, ptr(out), stream_handle()),
              "vx_dag_raycast")
        return out[:n * HIT_DTYPE.itemsize]

    def read_leaves(self, lo, n, out: torch.Tensor | None = None) -> torch.Tensor:
        """Occupancy masks of the leaf box [lo, lo + n) (leaf coordinates),
        x fastest, as an int64 device tensor."""
        count = int(n[0]) * int(n[1]) * int(n[2])
        if out is None:
            out = torch.empty(max(count, 1), dtype=torch.int64, device="cuda")
        check(lib().vx_dag_read_leaves(self._h, int(lo[0]), int(lo[1]), int(lo[2]), int(n[0]),
                                       int(n[1]), int(n[2]), ptr(out), stream_handle()),
              "vx_dag_read_leaves")
        return out[:count]

    def canonical(self, at_root: int = 0xFFFFFFFF):
        """(root, counts, nodes, leaves): DFS first-visit canonical dump of the
        current root, or of an earlier root ref still held by the tables."""
        root = C.c_uint32(0)
        counts = np.zeros(self.depth + 1, np.uint64)
        f = lib().vx_dag_export_canonical_at
        check(f(self._h, at_root, C.byref(root), counts.ctypes.data, None, 0, None, 0,
                stream_handle()), "export sizes")
        words = int(counts[:self.depth].sum()) * 10
        nodes = np.zeros(max(words, 1), np.uint32)
        nl = int(counts[self.depth])
        leaves = np.zeros(max(nl, 1), np.uint64)
        check(f(self._h, at_root, C.byref(root), counts.ctypes.data, nodes.ctypes.data,
                words, leaves.ctypes.data, nl, stream_handle()), "export")
        return root.value, counts, nodes[:words], leaves[:nl]


def generate_primitives(world_exp: int, count: int, seed: int, *,
                        sphere_permille: int = 1000, add_permille: int = 500,
                        r_min: int = 1, r_max: int = 16, log_uniform: bool = False,
                        material_min: int = 1, material_max: int = 255,
                        stream: int = 0) -> np.ndarray:
    """Seeded primitive list (PRIM_DTYPE) from the library's generator."""
    from . import vx_edit_mix
    mix = vx_edit_mix(world_exp, sphere_permille, add_permille, r_min, r_max,
                      int(log_uniform), material_min, material_max)
    out = np.zeros(count, PRIM_DTYPE)
    check(lib().vx_generate_primitives(C.byref(mix), seed, stream, count,
                                       out.ctypes.data if count else None),
          "vx_generate_primitives")
    return out


# The benchmark configurations' edit mixes.
def config_c1_edits(count: int = 1000, seed: int = 1) -> np.ndarray:
    """Plain SVO: 256^3, spheres r in U{2..16}, 50/50, materials U{1..255}."""
    return generate_primitives(8, count, seed, r_min=2, r_max=16)


def config_c3_edits(count: int = 65536, seed: int = 6, world_exp: int = 12) -> np.ndarray:
    """Batched SVO: 70% spheres / 30% boxes, r log-uniform [1, 64], 50/50."""
    return generate_primitives(world_exp, count, seed, sphere_permille=700,
                               r_min=1, r_max=64, log_uniform=True)


def config_c4_edits(count: int = 16384, seed: int = 7, world_exp: int = 14) -> np.ndarray:
    """Batched Hash DAG: spheres r log-uniform [1, 256], 60% add."""
    return generate_primitives(world_exp, count, seed, add_permille=600,
                               r_min=1, r_max=256, log_uniform=True)


def rasterize(prims: torch.Tensor, world_exp: int):
    """Voxel lists of primitives (clipped to the world): returns
    (voxels int32 [total, 3], offsets int64 [n + 1])."""
    n = prims.numel() // 8
    dev = prims.device
    counts = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    if n == 0:
        return torch.zeros((0, 3), dtype=torch.int32, device=dev), counts
    check(lib().vx_rasterize_count(ptr(prims), n, world_exp, ptr(counts),
                                   stream_handle()), "vx_rasterize_count")
    offsets = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    offsets[1:] = torch.cumsum(counts[:n], 0)
    total = int(offsets[-1].item())
    out = torch.empty((max(total, 1), 3), dtype=torch.int32, device=dev)
    check(lib().vx_rasterize(ptr(prims), n, world_exp, ptr(offsets), ptr(out),
                             stream_handle()), "vx_rasterize")
    return out[:total], offsets


class Svo:
    """Pointer sparse voxel octree on the GPU (GpuSvo / DeviceGpuSvo,
    svt/cuda/storage.cuh:12-122, widened to depth 1..12 and optional uint8
    materials)."""

    def __init__(self, depth: int, max_nodes: int = 1 << 20, max_leaves: int = 1 << 20,
                 materials: bool = False, arena_bytes: int = 0):
        from . import vx_svo_config
        cfg = vx_svo_config(depth, int(materials), max_nodes, max_leaves, arena_bytes)
        h = C.c_void_p()
        check(lib().vx_svo_create(C.byref(cfg), C.byref(h)), "vx_svo_create")
        self._h = h
        self._free = lib().vx_svo_destroy
        self.depth = depth
        self.materials = materials

    def device_view(self):
        """View for user kernels (voxel_b200_device.cuh vx_svo_get_voxel)."""
        from . import vx_svo_view
        v = vx_svo_view()
        check(lib().vx_svo_device_view(self._h, C.byref(v)), "vx_svo_device_view")
        return v

    def __del__(self):
        # the destroy function bound at creation: at interpreter exit the
        # module's globals may already be gone
        h, free = getattr(self, "_h", None), getattr(self, "_free", None)
        if h is not None and h.value and free is not None:
            free(h)
        self._h = None

    @property
    def world(self) -> int:
        return 4 << self.depth

    def reset(self):
        check(lib().vx_svo_reset(self._h, stream_handle()), "vx_svo_reset")

    def apply_voxels(self, voxels: torch.Tensor, op: int, material: int = 1,
                     workspace: torch.Tensor | None = None) -> int:
        """Plain path (svt::cuda::{place,destroy}_voxel_edits,
        svt/cuda/voxel/edit.cuh:76-92); returns the status."""
        n = voxels.numel() // 3
        ws = workspace
        if ws is None and n:
            ws = torch.empty(lib().vx_svo_voxel_workspace_size(n), dtype=torch.uint8,
                             device=voxels.device)
        return lib().vx_svo_apply_voxels(self._h, ptr(voxels) if n else None, n, op,
                                         material, ptr(ws) if n else None,
                                         ws.numel() if n else 0, stream_handle())

    def apply_terminal(self, nodes: torch.Tensor | None, leaves: torch.Tensor | None,
                       op: int, material: int = 1, workspace: torch.Tensor | None = None,
                       device="cuda") -> int:
        """Terminal edit (svt::cuda::place_/destroy_terminal_edits,
        svt/cuda/terminal/detail/pipeline.cuh:200-222); returns the status."""
        return _apply_terminal(lib().vx_svo_apply_terminal, self._h, nodes, leaves,
                               (op, material), workspace, device)

    def graph_primitives(self, prims: torch.Tensor, device_count: torch.Tensor | None = None,
                         capacity: int | None = None) -> "Graph":
        return _graph_primitives(lib().vx_svo_graph_primitives, self, prims, device_count,
                                 capacity)

    def apply_primitives(self, prims: torch.Tensor) -> None:
        n = prims.numel() // 8
        check(lib().vx_svo_apply_primitives(self._h, ptr(prims) if n else None, n,
                                            stream_handle()), "vx_svo_apply_primitives")

    def status(self) -> int:
        return lib().vx_svo_status(self._h, stream_handle())

    def build_terrain(self, seed: int, scale: int, caves: bool) -> None:
        from . import vx_terrain
        t = vx_terrain(seed, scale, int(caves), self.depth + 2)
        check(lib().vx_svo_build_terrain(self._h, C.byref(t), stream_handle()),
              "vx_svo_build_terrain")

    def apply_leaf_commands(self, cmds: torch.Tensor, op: int, material: int = 1,
                            workspace: torch.Tensor | None = None) -> int:
        """Leaf edit commands (see HashDag.apply_leaf_commands); placed voxels
        get `material` in a material SVO.  Returns the status."""
        n = cmds.numel() * cmds.element_size() // LEAF_COMMAND_DTYPE.itemsize
        ws = workspace
        if ws is None:
            ws = torch.empty(max(lib().vx_leaf_command_workspace_size(n), 1),
                             dtype=torch.uint8, device=cmds.device)
        return lib().vx_svo_apply_leaf_commands(self._h, ptr(cmds), n, op, material, ptr(ws),
                                                ws.numel(), stream_handle())

    def query(self, voxels: torch.Tensor) -> torch.Tensor:
        n = voxels.numel() // 3
        out = torch.empty(n, dtype=torch.uint8, device=voxels.device)
        check(lib().vx_svo_query(self._h, ptr(voxels), n, ptr(out), stream_handle()),
              "vx_svo_query")
        return out

    def counters(self):
        from . import vx_svo_counters
        c = vx_svo_counters()
        check(lib().vx_svo_get_counters(self._h, C.byref(c), stream_handle()),
              "vx_svo_get_counters")
        return c

    def collect(self) -> None:
        """Return the storage of every unreachable subtree to the free lists
        now (edits collect only when they would not fit otherwise)."""
        check(lib().vx_svo_collect(self._h, stream_handle()), "vx_svo_collect")

    def canonical(self):
        """(nodes [8 words each], leaves, materials or None): DFS pre-order."""
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        f = lib().vx_svo_export_canonical
        check(f(self._h, C.byref(nn), C.byref(nl), None, 0, None, None, 0,
                stream_handle()), "export sizes")
        nodes = np.zeros(max(nn.value * 8, 1), np.uint32)
        leaves = np.zeros(max(nl.value, 1), np.uint64)
        mats = np.zeros(max(nl.value * 64, 1), np.uint8) if self.materials else None
        check(f(self._h, C.byref(nn), C.byref(nl), nodes.ctypes.data, nn.value,
                leaves.ctypes.data, None if mats is None else mats.ctypes.data,
                nl.value, stream_handle()), "export")
        return (nodes[:nn.value * 8], leaves[:nl.value],
                None if mats is None else mats[:nl.value * 64])


COMPLETION_DTYPE = np.dtype([("request_id", "<u8"), ("arrival_ns", "<u8"),
                             ("commit_ns", "<u8"), ("status", "<u4"), ("root", "<u4")])


def generate_requests(world_exp: int, rate: float, seconds: float, seed: int, *,
                      zipf_s: float = 1.2, max_size: int = 4096,
                      sphere_permille: int = 500, add_permille: int = 500,
                      r_min: int = 1, r_max: int = 128, log_uniform: bool = True,
                      max_requests: int = 1 << 40):
    """Served request stream: (arrival_ns [n], sizes [n], prims [total])."""
    from . import vx_edit_mix
    mix = vx_edit_mix(world_exp, sphere_permille, add_permille, r_min, r_max,
                      int(log_uniform), 1, 255)
    nreq, nprim = C.c_uint64(0), C.c_uint64(0)
    f = lib().vx_generate_requests
    check(f(C.byref(mix), seed, rate, seconds, zipf_s, max_size, max_requests,
            None, None, 0, None, C.byref(nreq), C.byref(nprim)), "count requests")
    arr = np.zeros(max(nreq.value, 1), np.uint64)
    sizes = np.zeros(max(nreq.value, 1), np.uint32)
    prims = np.zeros(max(nprim.value, 1), PRIM_DTYPE)
    check(f(C.byref(mix), seed, rate, seconds, zipf_s, max_size, max_requests,
            arr.ctypes.data, sizes.ctypes.data, prims.size, prims.ctypes.data,
            C.byref(nreq), C.byref(nprim)), "generate requests")
    return arr[:nreq.value], sizes[:nreq.value], prims[:nprim.value]


class Server:
    """Request loop over a resident HashDag with continuous batching."""

    def __init__(self, dag: HashDag, max_batch_prims: int = 0, max_batch_requests: int = 0,
                 compact_at_fill: float = 0.0, max_inflight: int = 0, graphs: bool = True):
        from . import vx_serve_config
        cfg = vx_serve_config(max_batch_prims, max_batch_requests, compact_at_fill,
                              max_inflight, 0 if graphs else 1)
        h = C.c_void_p()
        check(lib().vx_serve_create(dag._h, C.byref(cfg), C.byref(h)), "vx_serve_create")
        self._h = h
        self.dag = dag

    @staticmethod
    def now_ns() -> int:
        return lib().vx_serve_now_ns()

    def submit(self, request_id: int, prims: np.ndarray, arrival_ns: int) -> None:
        p = np.ascontiguousarray(prims, PRIM_DTYPE)
        check(lib().vx_serve_submit(self._h, request_id, p.ctypes.data if p.size else None,
                                    p.size, arrival_ns), "vx_serve_submit")

    def poll(self, capacity: int = 1 << 16) -> np.ndarray:
        out = np.zeros(capacity, COMPLETION_DTYPE)
        n = C.c_uint32(0)
        check(lib().vx_serve_poll(self._h, out.ctypes.data, capacity, C.byref(n)),
              "vx_serve_poll")
        return out[:n.value]

    def drain(self) -> None:
        check(lib().vx_serve_drain(self._h), "vx_serve_drain")

    def stats(self):
        from . import vx_serve_stats
        st = vx_serve_stats()
        check(lib().vx_serve_get_stats(self._h, C.byref(st)), "vx_serve_get_stats")
        return st

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            check(lib().vx_serve_destroy(h), "vx_serve_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
