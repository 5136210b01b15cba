"""Torch-facing wrappers over the C ABI (mirror of the reference operators).

Each function takes CUDA tensors, allocates the workspace the C call asks for
(the reference's ``*_workspace_size`` + caller-owned workspace contract),
launches on the current torch stream and raises VoxelError on failure.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import check, lib

__all__ = [
    "stream_handle", "ptr", "exclusive_sum", "inclusive_sum", "sort_pairs",
    "workspace_status", "SlabHashSet", "CuckooMap",
]


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
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
        self.bucket_count = bucket_count
        self.slab_capacity = slab_capacity

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().vx_slab_set_destroy(h)
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


class CuckooMap:
    """u64 -> u32 cuckoo map with 4 hash functions and bounded eviction
    (cuda/cuckoo_hash.cuh:54-120 widened to inline u64 keys)."""

    def __init__(self, slot_count: int, max_evictions: int = 1000):
        h = C.c_void_p()
        check(lib().vx_cuckoo_create(slot_count, max_evictions, C.byref(h)),
              "vx_cuckoo_create")
        self._h = h
        self.slot_count = slot_count

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().vx_cuckoo_destroy(h)
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
