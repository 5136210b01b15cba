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
    "workspace_status",
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
