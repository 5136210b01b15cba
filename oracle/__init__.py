"""ORACLE - test infrastructure only.

A CPU restatement of the reference's algorithms for the voxel-editing path
(oracle_*.cpp), plus a shim over the reference's own CPU HashDAG / SVO
compiled from its headers (ref_shim.cpp -> _ref/libvxref.so).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this package,
and only as the checker or the timed baseline; the product library never
links, imports or calls it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libvxref.so"

_P = C.c_void_p
_U32 = C.c_uint32
_U64 = C.c_uint64
_I = C.c_int

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from . import build
            build.build_oracle()
        _lib = C.CDLL(str(LIB))
        for name, res, args in _SIGS:
            fn = getattr(_lib, name, None)
            if fn is not None:
                fn.restype = res
                fn.argtypes = args
    return _lib


def ref_available() -> bool:
    return REF_LIB.exists()


def ref():
    """The reference's own CPU HashDAG / SVO (requires oracle/_ref built)."""
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (needs the reference tree)")
        _ref = C.CDLL(str(REF_LIB))
        for name, res, args in _REF_SIGS:
            fn = getattr(_ref, name)
            fn.restype = res
            fn.argtypes = args
    return _ref


_SIGS = [
    ("orc_scan_u32", None, [_P, _P, _U64, _I]),
    ("orc_scan_u64", None, [_P, _P, _U64, _I]),
    ("orc_exclusive_scan_u32_mt", None, [_P, _P, _U64, _I]),
    ("orc_stable_sort_pairs_u32", None, [_P, _P, _U64, _U32]),
    ("orc_stable_sort_pairs_u64", None, [_P, _P, _U64, _U32]),
    ("orc_radix_sort_pairs_u32_mt", None, [_P, _P, _U64, _U32, _I]),
    ("orc_radix_sort_pairs_u64_mt", None, [_P, _P, _U64, _U32, _I]),
    ("orc_hash_set_u64", _U64, [_P, _U64, _P, _P, _U64, _P]),
]

_REF_SIGS = [
    ("ref_dag_new", _P, [_U32]),
    ("ref_dag_free", None, [_P]),
    ("ref_dag_edit_box", _I, [_P, _U32, _U32, _U32, _U32, _U32, _U32, _I]),
    ("ref_dag_set_voxel", _I, [_P, _U32, _U32, _U32, _I]),
    ("ref_dag_get_voxel", _I, [_P, _U32, _U32, _U32]),
    ("ref_dag_node_count", _U64, [_P]),
    ("ref_dag_export", _I, [_P, C.POINTER(_U32), _P, _P, _U64, _P, _U64]),
    ("ref_svo_new", _P, [_U32]),
    ("ref_svo_free", None, [_P]),
    ("ref_svo_set_voxel", _I, [_P, _U32, _U32, _U32, _I]),
    ("ref_svo_get_voxel", _I, [_P, _U32, _U32, _U32]),
    ("ref_svo_node_count", _U64, [_P]),
    ("ref_svo_leaf_count", _U64, [_P]),
    ("ref_svo_export", _I, [_P, C.POINTER(_U32), C.POINTER(_U32), _P, _U32,
                            _P, _U32]),
]


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------- primitives --

def exclusive_sum(a: np.ndarray) -> np.ndarray:
    out = np.empty_like(a)
    fn = lib().orc_scan_u64 if a.dtype.itemsize == 8 else lib().orc_scan_u32
    fn(_p(np.ascontiguousarray(a)), _p(out), a.size, 0)
    return out


def inclusive_sum(a: np.ndarray) -> np.ndarray:
    out = np.empty_like(a)
    fn = lib().orc_scan_u64 if a.dtype.itemsize == 8 else lib().orc_scan_u32
    fn(_p(np.ascontiguousarray(a)), _p(out), a.size, 1)
    return out


def stable_sort_pairs(keys: np.ndarray, values: np.ndarray | None,
                      key_bits: int):
    k = np.ascontiguousarray(keys).copy()
    v = None if values is None else np.ascontiguousarray(values, np.uint32).copy()
    fn = (lib().orc_stable_sort_pairs_u64 if k.dtype.itemsize == 8
          else lib().orc_stable_sort_pairs_u32)
    fn(_p(k), _p(v), k.size, key_bits)
    return k, v


def hash_set(inserts: np.ndarray, queries: np.ndarray):
    ins = np.ascontiguousarray(inserts, np.uint64)
    q = np.ascontiguousarray(queries, np.uint64)
    st = np.empty(ins.size, np.uint32)
    found = np.empty(q.size, np.uint32)
    lib().orc_hash_set_u64(_p(ins), ins.size, _p(st), _p(q), q.size, _p(found))
    return st, found
