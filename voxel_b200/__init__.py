"""voxel_b200 - B200-native voxel-editing path (scan, radix sort, hash tables,
sparse voxel octree and Hash DAG editing) behind a C ABI.

This module binds ``libvoxel_b200.so`` (built in-tree by
``python -m voxel_b200.build``) with ctypes and mirrors the reference's
operator interface (``algo::cuda::scan``, ``algo::cuda::sort``, the hash
tables, ``algo::svt::cuda`` and ``algo::svt::hash_dag_gpu``) for Python
callers: device buffers are torch CUDA tensors, streams are torch streams,
and every failure raises :class:`VoxelError` with the library status code.
There is no CPU fallback: importing works without a GPU, but every compute
call requires the CUDA library and a device.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libvoxel_b200.so"

VX_OK = 0
VX_ERR_INVALID_VALUE = 1
# hash-table statuses (the reference's kSlabHashStatus* values) and keys
VX_HASH_NOT_FOUND, VX_HASH_INSERTED, VX_HASH_REPLACED, VX_HASH_ERASED = 0, 1, 2, 3
VX_HASH_OVERFLOW, VX_HASH_INVALID_KEY, VX_HASH_FOUND, VX_HASH_ALREADY_PRESENT = 4, 5, 6, 7
VX_HASH_NOT_FOUND_VALUE = 0xFFFFFFFF
VX_MAP_EMPTY_KEY = 0xFFFFFFFF
VX_MAP_DELETED_KEY = 0xFFFFFFFE
VX_ERR_MEMORY_ALLOCATION = 2
VX_ERR_TIMEOUT = 1001
VX_ERR_CAPACITY = 1002
VX_ERR_NO_DEVICE = 1003
VX_ERR_IO = 1004

HASH_NOT_FOUND = 0
HASH_INSERTED = 1
HASH_REPLACED = 2
HASH_ERASED = 3
HASH_OVERFLOW = 4
HASH_INVALID_KEY = 5
HASH_FOUND = 6
HASH_ALREADY_PRESENT = 7
HASH_NOT_FOUND_VALUE = 0xFFFFFFFF
HASH_EMPTY_KEY = 0xFFFFFFFFFFFFFFFF
HASH_DELETED_KEY = 0xFFFFFFFFFFFFFFFE

EDIT_DESTROY = 0
EDIT_PLACE = 1
SHAPE_SPHERE = 0
SHAPE_BOX = 1
OP_REMOVE = 0
OP_ADD = 1


class VoxelError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)})")


class vx_voxel(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("z", C.c_uint32)]


class vx_primitive(C.Structure):
    _fields_ = [("c", C.c_int32 * 3), ("r", C.c_uint32 * 3),
                ("flags", C.c_uint32), ("reserved", C.c_uint32)]


class vx_terrain(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("scale", C.c_uint32),
                ("caves", C.c_uint32), ("world_exp", C.c_uint32)]


class vx_edit_mix(C.Structure):
    _fields_ = [("world_exp", C.c_uint32), ("sphere_permille", C.c_uint32),
                ("add_permille", C.c_uint32), ("r_min", C.c_uint32),
                ("r_max", C.c_uint32), ("log_uniform", C.c_uint32),
                ("material_min", C.c_uint32), ("material_max", C.c_uint32)]


class vx_dag_config(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("reserved0", C.c_uint32),
                ("max_nodes", C.c_uint64), ("arena_bytes", C.c_uint64)]


class vx_dag_stats(C.Structure):
    _fields_ = [("nodes_per_level", C.c_uint64 * 16),
                ("words_per_level", C.c_uint64 * 16),
                ("items_per_level", C.c_uint32 * 16),
                ("pairs_per_level", C.c_uint32 * 16),
                ("bytes_reserved", C.c_uint64), ("root", C.c_uint32),
                ("status", C.c_uint32)]


class vx_dag_view(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("reserved", C.c_uint32), ("root", C.c_void_p),
                ("pool", C.c_void_p * 14), ("leaves", C.c_void_p)]


class vx_svo_view(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("materials", C.c_uint32), ("nodes", C.c_void_p),
                ("leaves", C.c_void_p), ("materials_data", C.c_void_p)]


class vx_slab_set_view(C.Structure):
    _fields_ = [("slabs", C.c_void_p), ("bucket_count", C.c_uint32), ("capacity", C.c_uint32)]


class vx_cuckoo_view(C.Structure):
    _fields_ = [("slots", C.c_void_p), ("slot_count", C.c_uint32), ("reserved", C.c_uint32)]


class vx_serve_config(C.Structure):
    _fields_ = [("max_batch_prims", C.c_uint32), ("max_batch_requests", C.c_uint32),
                ("compact_at_fill", C.c_double), ("max_inflight", C.c_uint32),
                ("launch_mode", C.c_uint32)]


class vx_serve_stats(C.Structure):
    _fields_ = [("batches", C.c_uint64), ("requests", C.c_uint64),
                ("prims", C.c_uint64), ("compactions", C.c_uint64),
                ("recoveries", C.c_uint64), ("compact_ms", C.c_double)]


class vx_svo_config(C.Structure):
    _fields_ = [("depth", C.c_uint32), ("materials", C.c_uint32),
                ("max_nodes", C.c_uint32), ("max_leaves", C.c_uint32),
                ("arena_bytes", C.c_uint64)]


class vx_svo_counters(C.Structure):
    _fields_ = [("node_count", C.c_uint32), ("leaf_count", C.c_uint32),
                ("free_node_count", C.c_uint32),
                ("free_leaf_count", C.c_uint32)]


_P = C.c_void_p
_U32 = C.c_uint32
_U64 = C.c_uint64
_SZ = C.c_size_t
_ST = C.c_int32

# name -> (restype, argtypes).  Every symbol declared in include/voxel_b200.h
# that the library exports is listed here; missing symbols are tolerated at
# load time (so a partial build can still be inspected) and fail on use.
_SIGS = {
    "vx_version": (_U32, []),
    "vx_status_string": (C.c_char_p, [_ST]),
    "vx_workspace_status": (_ST, [_P, _P]),
    "vx_profile_enable": (None, [_U32]),
    "vx_profile_reset": (None, []),
    "vx_profile_launches": (_U64, []),
    "vx_profile_query": (_ST, [C.c_char_p, C.POINTER(C.c_double),
                               C.POINTER(_U64)]),
    "vx_generate_primitives": (_ST, [C.POINTER(vx_edit_mix), _U64, _U64, _U64, _P]),
    "vx_scan_workspace_size": (_SZ, [_U32]),
    "vx_scan_exclusive_sum_u32": (_ST, [_P, _U32, _P, _SZ, _P]),
    "vx_scan_inclusive_sum_u32": (_ST, [_P, _U32, _P, _SZ, _P]),
    "vx_scan_exclusive_sum_u64": (_ST, [_P, _U32, _P, _SZ, _P]),
    "vx_scan_exclusive_sum_u32_noalloc": (_ST, [_P, _U32, _P]),
    "vx_scan_noalloc_status": (_ST, [_P]),
    "vx_sort_workspace_size": (_SZ, [_U32, _U32]),
    "vx_sort_pairs_u32": (_ST, [_P, _P, _U32, _U32, _P, _SZ, _P]),
    "vx_sort_pairs_u64": (_ST, [_P, _P, _U32, _U32, _P, _SZ, _P]),
    "vx_sort_words_workspace_size": (_SZ, [_U32, _U32]),
    "vx_sort_words": (_ST, [_P, _U32, _U32, _U32, _P, _P, _SZ, _P]),
    "vx_gather": (_ST, [_P, _P, _P, _U32, _U32, _P]),
    "vx_slab_set_create": (_ST, [_U32, _U32, C.POINTER(_P)]),
    "vx_slab_set_destroy": (_ST, [_P]),
    "vx_slab_set_clear": (_ST, [_P, _P]),
    "vx_slab_set_insert": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_slab_set_contains": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_slab_set_erase": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_slab_set_bytes": (_SZ, [_P]),
    "vx_slab_map_create": (_ST, [_U32, _U32, C.POINTER(_P)]),
    "vx_slab_map_destroy": (_ST, [_P]),
    "vx_slab_map_clear": (_ST, [_P, _P]),
    "vx_slab_map_insert_or_replace": (_ST, [_P, _P, _P, _U32, _P, _P]),
    "vx_slab_map_find": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_slab_map_erase_all": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_slab_map_bytes": (_SZ, [_P]),
    "vx_itemset_create": (_ST, [_U32, _U32, C.POINTER(_P)]),
    "vx_itemset_destroy": (_ST, [_P]),
    "vx_itemset_clear": (_ST, [_P, _P]),
    "vx_itemset_find": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_itemset_find_or_insert": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_itemset_insert_unique_unchecked": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_itemset_read": (_ST, [_P, _P, _U32, _P, _P, _P]),
    "vx_itemset_count": (_ST, [_P, C.POINTER(_U64), _P]),
    "vx_cuckoo_create": (_ST, [_U32, _U32, C.POINTER(_P)]),
    "vx_cuckoo_destroy": (_ST, [_P]),
    "vx_cuckoo_clear": (_ST, [_P, _P]),
    "vx_cuckoo_insert": (_ST, [_P, _P, _P, _U32, _P, _P]),
    "vx_cuckoo_find": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_cuckoo_bytes": (_SZ, [_P]),
    "vx_cuckoo_dropped": (_ST, [_P, C.POINTER(_U64), _P]),
    "vx_dag_create": (_ST, [C.POINTER(vx_dag_config), C.POINTER(_P)]),
    "vx_dag_destroy": (_ST, [_P]),
    "vx_dag_reset": (_ST, [_P, _P]),
    "vx_dag_depth": (_U32, [_P]),
    "vx_dag_voxel_workspace_size": (_SZ, [_U32]),
    "vx_dag_apply_voxels": (_ST, [_P, _P, _U32, _U32, _P, _SZ, _P]),
    "vx_dag_apply_primitives": (_ST, [_P, _P, _U32, _P]),
    "vx_dag_status": (_ST, [_P, _P]),
    "vx_dag_build_terrain": (_ST, [_P, C.POINTER(vx_terrain), _P]),
    "vx_dag_query": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_dag_raycast": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_leaf_command_workspace_size": (_SZ, [_U32]),
    "vx_dag_apply_leaf_commands": (_ST, [_P, _P, _U32, _U32, _P, _SZ, _P]),
    "vx_svo_apply_leaf_commands": (_ST, [_P, _P, _U32, _U32, _U32, _P, _SZ, _P]),
    "vx_dag_read_leaves": (_ST, [_P, _U32, _U32, _U32, _U32, _U32, _U32, _P, _P]),
    "vx_dag_export_canonical": (_ST, [_P, C.POINTER(_U32), _P,
                                      _P, _U64, _P, _U64, _P]),
    "vx_dag_get_stats": (_ST, [_P, C.POINTER(vx_dag_stats), _P]),
    "vx_dag_export_canonical_at": (_ST, [_P, _U32, C.POINTER(_U32), _P, _P, _U64,
                                         _P, _U64, _P]),
    "vx_serve_now_ns": (_U64, []),
    "vx_serve_create": (_ST, [_P, C.POINTER(vx_serve_config), C.POINTER(_P)]),
    "vx_serve_submit": (_ST, [_P, _U64, _P, _U32, _U64]),
    "vx_serve_poll": (_ST, [_P, _P, _U32, C.POINTER(_U32)]),
    "vx_serve_drain": (_ST, [_P]),
    "vx_serve_get_stats": (_ST, [_P, C.POINTER(vx_serve_stats)]),
    "vx_serve_destroy": (_ST, [_P]),
    "vx_generate_requests": (_ST, [C.POINTER(vx_edit_mix), _U64, C.c_double, C.c_double,
                                   C.c_double, _U32, _U64, _P, _P, _U64, _P,
                                   C.POINTER(_U64), C.POINTER(_U64)]),
    "vx_dag_copy": (_ST, [_P, _P, _P]),
    "vx_dag_compact": (_ST, [_P, _P]),
    "vx_svo_create": (_ST, [C.POINTER(vx_svo_config), C.POINTER(_P)]),
    "vx_svo_destroy": (_ST, [_P]),
    "vx_svo_reset": (_ST, [_P, _P]),
    "vx_svo_voxel_workspace_size": (_SZ, [_U32]),
    "vx_svo_apply_voxels": (_ST, [_P, _P, _U32, _U32, _U32, _P, _SZ, _P]),
    "vx_svo_apply_primitives": (_ST, [_P, _P, _U32, _P]),
    "vx_svo_status": (_ST, [_P, _P]),
    "vx_svo_build_terrain": (_ST, [_P, C.POINTER(vx_terrain), _P]),
    "vx_svo_query": (_ST, [_P, _P, _U32, _P, _P]),
    "vx_svo_export_canonical": (_ST, [_P, C.POINTER(_U32), C.POINTER(_U32),
                                      _P, _U32, _P, _P, _U32, _P]),
    "vx_svo_get_counters": (_ST, [_P, C.POINTER(vx_svo_counters), _P]),
    "vx_svo_collect": (_ST, [_P, _P]),
    "vx_svo_depth": (_U32, [_P]),
    "vx_terminal_workspace_size": (_SZ, [_U32, _U32]),
    "vx_svo_apply_terminal": (_ST, [_P, _P, _U32, _P, _U32, _U32, _U32, _P, _SZ, _P]),
    "vx_dag_apply_terminal": (_ST, [_P, _P, _U32, _P, _U32, _U32, _P, _SZ, _P]),
    "vx_rasterize_count": (_ST, [_P, _U32, _U32, _P, _P]),
    "vx_rasterize": (_ST, [_P, _U32, _U32, _P, _P, _P]),
    "vx_dag_graph_primitives": (_ST, [_P, _P, _P, _U32, C.POINTER(_P)]),
    "vx_dag_graph_voxels": (_ST, [_P, _P, _U32, _U32, _P, _SZ, C.POINTER(_P)]),
    "vx_svo_graph_primitives": (_ST, [_P, _P, _P, _U32, C.POINTER(_P)]),
    "vx_graph_launch": (_ST, [_P, _P]),
    "vx_graph_kernels": (_ST, [_P, C.POINTER(_U64)]),
    "vx_graph_destroy": (_ST, [_P]),
    "vx_dag_device_view": (_ST, [_P, C.POINTER(vx_dag_view)]),
    "vx_svo_device_view": (_ST, [_P, C.POINTER(vx_svo_view)]),
    "vx_slab_set_device_view": (_ST, [_P, C.POINTER(vx_slab_set_view)]),
    "vx_cuckoo_device_view": (_ST, [_P, C.POINTER(vx_cuckoo_view)]),
    "vx_dag_import_canonical": (_ST, [_P, _U32, _P, _P, _P, _P]),
    "vx_dag_save": (_ST, [_P, C.c_char_p, _P]),
    "vx_dag_load": (_ST, [_P, C.c_char_p, _P]),
    "vx_tuning_count": (_U32, []),
    "vx_tuning_name": (C.c_char_p, [_U32]),
    "vx_tuning_options": (_ST, [C.c_char_p, C.POINTER(C.c_int64), _U32, C.POINTER(_U32)]),
    "vx_tuning_get": (_ST, [C.c_char_p, C.POINTER(C.c_int64)]),
    "vx_tuning_set": (_ST, [C.c_char_p, C.c_int64]),
    "vx_tuning_reset": (_ST, []),
}

_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: run `python -m voxel_b200.build` "
                "(there is no CPU fallback)")
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(l, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = l
        _apply_saved_tuning()
    return _lib


TUNING_DIR = Path(__file__).resolve().parent / "tuning"


def tuning_file(device_name: str) -> Path:
    """Where the autotuner keeps the knob settings for one kind of device."""
    safe = "".join(ch if ch.isalnum() else "_" for ch in device_name).strip("_")
    return TUNING_DIR / f"{safe}.json"


def _apply_saved_tuning() -> None:
    """Apply the autotuner's settings for the current device, if it has any
    (voxel_b200/tuning/<device>.json, written by voxel_b200.autotune)."""
    try:
        import torch
        if not torch.cuda.is_available():
            return
        path = tuning_file(torch.cuda.get_device_name())
    except Exception:
        return
    if not path.exists():
        return
    import json
    knobs = json.loads(path.read_text()).get("knobs", {})
    for name, value in knobs.items():
        _lib.vx_tuning_set(name.encode(), int(value))


def exported_symbols() -> list[str]:
    """Names from the signature table that the loaded library exports."""
    l = lib()
    return [n for n in _SIGS if hasattr(l, n)]


def status_string(status: int) -> str:
    try:
        return lib().vx_status_string(status).decode()
    except Exception:  # library not loadable
        return "unknown"


def check(status: int, what: str) -> None:
    if status != VX_OK:
        raise VoxelError(status, what)


from .api import *  # noqa: E402,F401,F403
