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
    ("ref_dag_apply_prim", C.c_longlong, [_P, _I] + [C.c_longlong] * 6 + [_I]),
    ("ref_dag_apply_prim_clipped", C.c_longlong, [_P, _I] + [C.c_longlong] * 6 + [_I, _P, _P]),
    ("ref_dag_get_voxel", _I, [_P, _U32, _U32, _U32]),
    ("ref_dag_node_count", _U64, [_P]),
    ("ref_dag_export", _I, [_P, C.POINTER(_U32), _P, _P, _U64, _P, _U64]),
    ("ref_dag_import_region", _I, [_P, _U32, _U32, _U32, _U32, _U32, _P, _P, _P]),
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


# --------------------------------------------------------------- voxels --

_VOXEL_SIGS = [
    ("orc_grid_new", _P, [_U32, _I]),
    ("orc_grid_free", None, [_P]),
    ("orc_grid_terrain", None, [_P, _P]),
    ("orc_grid_apply_prims", None, [_P, _P, _U64]),
    ("orc_grid_apply_voxels", None, [_P, _P, _U64, _I, _U32]),
    ("orc_grid_apply_terminal", None, [_P, _P, _U64, _P, _U64, _I, _U32]),
    ("orc_grid_count", _U64, [_P]),
    ("orc_grid_get", _I, [_P, _U32, _U32, _U32]),
    ("orc_grid_export_dag", _I, [_P, C.POINTER(_U32), _P, _P, _U64, _P, _U64]),
    ("orc_grid_export_svo", _I, [_P, C.POINTER(_U32), C.POINTER(_U32), _P, _U32,
                                 _P, _P, _U32]),
    ("orc_eval_voxels", None, [_P, _U32, _P, _U64, _P, _U64, _P, _I]),
    ("orc_sparse_run", _P, [_U32, _P, _P, _U64, _I, _U32, _P, _U32, _I]),
    ("orc_sparse_free", None, [_P]),
    ("orc_sparse_export_dag", _I, [_P, C.POINTER(_U32), _P, _P, _U64, _P, _U64]),
    ("orc_sparse_export_svo", _I, [_P, C.POINTER(_U64), C.POINTER(_U64), _P, _U64, _P, _P,
                                   _U64]),
    ("orc_sparse_leaf_block", None, [_P, _P, _P, _P]),
    ("orc_terrain_leaf_mismatches", _U64, [_P, _P, _U64, _I]),
    ("orc_terrain_classify_mismatches", _U64, [_P, _P, _U64]),
    ("orc_generate_primitives", None, [_P, _U64, _U64, _U64, _P]),
    ("orc_sparse_raycast", None, [_P, _P, _U64, _P]),
    ("orc_generate_requests", _U64, [_P, _U64, C.c_double, C.c_double, C.c_double, _U32,
                                     _U64, _P, _P, _U64, _P, C.POINTER(_U64)]),
]
_SIGS.extend(_VOXEL_SIGS)

PRIM_DTYPE = np.dtype([("c", "<i4", 3), ("r", "<u4", 3), ("flags", "<u4"),
                       ("reserved", "<u4")])
TERRAIN_DTYPE = np.dtype([("seed", "<u4"), ("scale", "<u4"), ("caves", "<u4"),
                          ("world_exp", "<u4")])


EDIT_MIX_DTYPE = np.dtype([(k, "<u4") for k in (
    "world_exp", "sphere_permille", "add_permille", "r_min", "r_max", "log_uniform",
    "material_min", "material_max")])


def _mix(world_exp, sphere_permille, add_permille, r_min, r_max, log_uniform,
         material_min, material_max) -> np.ndarray:
    m = np.zeros(1, EDIT_MIX_DTYPE)
    m[0] = (world_exp, sphere_permille, add_permille, r_min, r_max, int(log_uniform),
            material_min, material_max)
    return m


def generate_primitives(world_exp: int, count: int, seed: int, *,
                        sphere_permille: int = 1000, add_permille: int = 500,
                        r_min: int = 1, r_max: int = 16, log_uniform: bool = False,
                        material_min: int = 1, material_max: int = 255,
                        stream: int = 0) -> np.ndarray:
    """The seeded primitive lists of vx_workload.h (same draws as the
    library's vx_generate_primitives)."""
    m = _mix(world_exp, sphere_permille, add_permille, r_min, r_max, log_uniform,
             material_min, material_max)
    out = np.zeros(max(count, 1), PRIM_DTYPE)
    lib().orc_generate_primitives(m.ctypes.data, seed, stream, count, out.ctypes.data)
    return out[:count]


def config_c4_edits(count: int = 16384, seed: int = 7, world_exp: int = 14) -> np.ndarray:
    """The batched Hash DAG benchmark's spheres: r log-uniform [1, 256], 60 % add."""
    return generate_primitives(world_exp, count, seed, add_permille=600, r_min=1, r_max=256,
                               log_uniform=True)


def config_c3_edits(count: int = 65536, seed: int = 6, world_exp: int = 12) -> np.ndarray:
    """The batched SVO benchmark's mix: 70 % spheres / 30 % boxes, r log-uniform [1, 64]."""
    return generate_primitives(world_exp, count, seed, sphere_permille=700, r_min=1, r_max=64,
                               log_uniform=True)


def generate_requests(world_exp: int, rate: float, seconds: float, seed: int, *,
                      zipf_s: float = 1.2, max_size: int = 4096, sphere_permille: int = 500,
                      add_permille: int = 500, r_min: int = 1, r_max: int = 128,
                      log_uniform: bool = True, max_requests: int = 1 << 40):
    """A served request stream (arrival_ns, sizes, prims) of vx_workload.h."""
    m = _mix(world_exp, sphere_permille, add_permille, r_min, r_max, log_uniform, 1, 255)
    total = C.c_uint64(0)
    f = lib().orc_generate_requests
    n = f(m.ctypes.data, seed, rate, seconds, zipf_s, max_size, max_requests, None, None, 0,
          None, C.byref(total))
    arr = np.zeros(max(n, 1), np.uint64)
    sizes = np.zeros(max(n, 1), np.uint32)
    prims = np.zeros(max(total.value, 1), PRIM_DTYPE)
    f(m.ctypes.data, seed, rate, seconds, zipf_s, max_size, max_requests, arr.ctypes.data,
      sizes.ctypes.data, prims.size, prims.ctypes.data, C.byref(total))
    return arr[:n], sizes[:n], prims[:total.value]


def terrain(seed: int, scale: int, caves: bool, world_exp: int = 0) -> np.ndarray:
    t = np.zeros(1, TERRAIN_DTYPE)
    t[0] = (seed, scale, int(caves), world_exp)
    return t


class DagCanon:
    """A canonical Hash DAG dump: root id, per-level node records
    (10 words: child_mask, fill_mask, 8 child ids) and leaf masks."""

    def __init__(self, root, counts, nodes, leaves):
        self.root = int(root)
        self.counts = [int(c) for c in counts]
        self.nodes = np.asarray(nodes, np.uint32)
        self.leaves = np.asarray(leaves, np.uint64)

    def __eq__(self, other):
        return (self.root == other.root and self.counts == other.counts
                and np.array_equal(self.nodes, other.nodes)
                and np.array_equal(self.leaves, other.leaves))

    def __repr__(self):
        return f"DagCanon(root={self.root}, counts={self.counts})"


class SvoCanon:
    def __init__(self, nodes, leaves, mats=None):
        self.nodes = np.asarray(nodes, np.uint32)
        self.leaves = np.asarray(leaves, np.uint64)
        self.mats = None if mats is None else np.asarray(mats, np.uint8)

    def __eq__(self, other):
        if not (np.array_equal(self.nodes, other.nodes)
                and np.array_equal(self.leaves, other.leaves)):
            return False
        if self.mats is None or other.mats is None:
            return True
        return np.array_equal(self.mats, other.mats)

    def __repr__(self):
        return f"SvoCanon(nodes={self.nodes.size // 8}, leaves={self.leaves.size})"


def _dump_dag(fn, h, depth):
    root = C.c_uint32(0)
    counts = np.zeros(depth + 1, np.uint64)
    fn(h, C.byref(root), counts.ctypes.data, None, 0, None, 0)
    words = int(counts[:depth].sum()) * 10
    nodes = np.zeros(max(words, 1), np.uint32)
    leaves = np.zeros(max(int(counts[depth]), 1), np.uint64)
    rc = fn(h, C.byref(root), counts.ctypes.data, nodes.ctypes.data, words,
            leaves.ctypes.data, int(counts[depth]))
    assert rc == 0
    return DagCanon(root.value, counts, nodes[:words], leaves[:int(counts[depth])])


class Grid:
    """Dense voxel grid of a 4 << depth world with sequential edit semantics."""

    def __init__(self, depth: int, materials: bool = False):
        self.depth = depth
        self.materials = materials
        self._h = lib().orc_grid_new(depth, int(materials))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_grid_free(self._h)
            self._h = None

    def terrain(self, t: np.ndarray):
        lib().orc_grid_terrain(self._h, t.ctypes.data)
        return self

    def apply_prims(self, prims: np.ndarray):
        p = np.ascontiguousarray(prims, PRIM_DTYPE)
        lib().orc_grid_apply_prims(self._h, p.ctypes.data, p.size)
        return self

    def apply_terminal(self, nodes, leaves, op: int, material: int = 1):
        """Terminal edit semantics: nodes / leaves are record arrays with the
        TerminalNodeInput (20 B) / TerminalLeafInput (32 B) layouts."""
        n = np.ascontiguousarray(nodes) if nodes is not None and len(nodes) else None
        lv = np.ascontiguousarray(leaves) if leaves is not None and len(leaves) else None
        assert n is None or n.dtype.itemsize == 20
        assert lv is None or lv.dtype.itemsize == 32
        lib().orc_grid_apply_terminal(self._h, None if n is None else n.ctypes.data,
                                      0 if n is None else n.size,
                                      None if lv is None else lv.ctypes.data,
                                      0 if lv is None else lv.size, op, material)
        return self

    def apply_voxels(self, xyz: np.ndarray, op: int, material: int = 1):
        v = np.ascontiguousarray(xyz, np.uint32).reshape(-1, 3)
        lib().orc_grid_apply_voxels(self._h, v.ctypes.data, v.shape[0], op, material)
        return self

    def count(self) -> int:
        return lib().orc_grid_count(self._h)

    def get(self, x, y, z) -> int:
        return lib().orc_grid_get(self._h, x, y, z)

    def dag(self) -> DagCanon:
        return _dump_dag(lib().orc_grid_export_dag, self._h, self.depth)

    def svo(self) -> SvoCanon:
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        f = lib().orc_grid_export_svo
        f(self._h, C.byref(nn), C.byref(nl), None, 0, None, None, 0)
        nodes = np.zeros(max(nn.value * 8, 1), np.uint32)
        leaves = np.zeros(max(nl.value, 1), np.uint64)
        mats = np.zeros(max(nl.value * 64, 1), np.uint8) if self.materials else None
        rc = f(self._h, C.byref(nn), C.byref(nl), nodes.ctypes.data, nn.value,
               leaves.ctypes.data, None if mats is None else mats.ctypes.data, nl.value)
        assert rc == 0
        return SvoCanon(nodes[:nn.value * 8], leaves[:nl.value],
                        None if mats is None else mats[:nl.value * 64])


def eval_voxels(t, world_exp, prims, xyz, materials=False) -> np.ndarray:
    p = np.ascontiguousarray(prims, PRIM_DTYPE)
    v = np.ascontiguousarray(xyz, np.uint32).reshape(-1, 3)
    out = np.zeros(v.shape[0], np.uint8)
    lib().orc_eval_voxels(None if t is None else t.ctypes.data, world_exp,
                          p.ctypes.data, p.size, v.ctypes.data, v.shape[0],
                          out.ctypes.data, int(materials))
    return out


class Sparse:
    """Sequential editing on a sparse, hash-consed CPU DAG (oracle_sparse.cpp):
    the terrain of a 4 << depth world (or an empty world), then every
    primitive in order.  With base > 0 only the cell of that level containing
    voxel `cell` is built (a region); the work is split into 8^shard_levels
    shards over `threads` threads.  Dumps use the canonical forms of Grid."""

    def __init__(self, depth: int, terrain_: np.ndarray | None = None, prims=None,
                 materials: bool = False, base: int = 0, cell=(0, 0, 0),
                 shard_levels: int = 3, threads: int | None = None):
        import os
        self.depth, self.base, self.materials = depth, base, materials
        p = np.ascontiguousarray(np.zeros(0, PRIM_DTYPE) if prims is None else prims, PRIM_DTYPE)
        c = np.ascontiguousarray(cell, np.uint32)
        self._h = lib().orc_sparse_run(depth, None if terrain_ is None else terrain_.ctypes.data,
                                       p.ctypes.data if p.size else None, p.size, int(materials),
                                       base, c.ctypes.data, shard_levels,
                                       threads or os.cpu_count() or 1)
        assert self._h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_sparse_free(self._h)
            self._h = None

    def dag(self) -> DagCanon:
        return _dump_dag(lib().orc_sparse_export_dag, self._h, self.depth - self.base)

    def svo(self) -> SvoCanon:
        nn, nl = C.c_uint64(0), C.c_uint64(0)
        f = lib().orc_sparse_export_svo
        f(self._h, C.byref(nn), C.byref(nl), None, 0, None, None, 0)
        nodes = np.zeros(max(nn.value * 8, 1), np.uint32)
        leaves = np.zeros(max(nl.value, 1), np.uint64)
        mats = np.zeros(max(nl.value * 64, 1), np.uint8) if self.materials else None
        rc = f(self._h, C.byref(nn), C.byref(nl), nodes.ctypes.data, nn.value,
               leaves.ctypes.data, None if mats is None else mats.ctypes.data, nl.value)
        assert rc == 0
        return SvoCanon(nodes[:nn.value * 8], leaves[:nl.value],
                        None if mats is None else mats[:nl.value * 64])

    def raycast(self, rays: np.ndarray) -> np.ndarray:
        """First solid voxel of each ray (records of 8 floats: origin, dir,
        t_max, unused), as records of 5 words (voxel, face, t bits); the
        world must be whole (base 0)."""
        assert self.base == 0
        r = np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)
        out = np.zeros((r.shape[0], 5), np.uint32)
        lib().orc_sparse_raycast(self._h, r.ctypes.data, r.shape[0], out.ctypes.data)
        return out

    def leaf_block(self, lo, n) -> np.ndarray:
        """Occupancy masks of the leaves [lo, lo + n) (leaf coordinates), x fastest."""
        lo_ = np.ascontiguousarray(lo, np.uint32)
        n_ = np.ascontiguousarray(n, np.uint32)
        out = np.zeros(int(np.prod(n_.astype(np.uint64))), np.uint64)
        lib().orc_sparse_leaf_block(self._h, lo_.ctypes.data, n_.ctypes.data, out.ctypes.data)
        return out


def terrain_leaf_mismatches(t: np.ndarray, origins: np.ndarray, materials: bool) -> int:
    o = np.ascontiguousarray(origins, np.uint32).reshape(-1, 3)
    return lib().orc_terrain_leaf_mismatches(t.ctypes.data, o.ctypes.data, o.shape[0],
                                             int(materials))


def terrain_classify_mismatches(t: np.ndarray, cubes: np.ndarray) -> int:
    q = np.ascontiguousarray(cubes, np.uint32).reshape(-1, 4)
    return lib().orc_terrain_classify_mismatches(t.ctypes.data, q.ctypes.data, q.shape[0])


class RefDag:
    """The reference's own CPU HashDAG (algorithm/lib/include/algo/svt/hash_dag.hpp)."""

    def __init__(self, depth: int):
        self.depth = depth
        self._h = ref().ref_dag_new(depth)
        assert self._h

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_dag_free(self._h)
            self._h = None

    def box(self, lo, hi, fill: bool):
        """Half-open box [lo, hi) like HashDAG::Box."""
        rc = ref().ref_dag_edit_box(self._h, *map(int, lo), *map(int, hi), int(fill))
        assert rc == 0

    def set_voxel(self, x, y, z, v: bool):
        assert ref().ref_dag_set_voxel(self._h, x, y, z, int(v)) == 0

    def get_voxel(self, x, y, z) -> int:
        return ref().ref_dag_get_voxel(self._h, x, y, z)

    def apply_prim_runs(self, p):
        """Apply one sphere / box primitive as x-runs of boxes."""
        world = 4 << self.depth
        add = ((int(p["flags"]) >> 8) & 0xFF) == 1
        c = [int(v) for v in p["c"]]
        r = [int(v) for v in p["r"]]
        if (int(p["flags"]) & 0xFF) == 1:  # box
            lo = [max(0, c[a] - r[a]) for a in range(3)]
            hi = [min(world, c[a] + r[a] + 1) for a in range(3)]
            if all(hi[a] > lo[a] for a in range(3)):
                self.box(lo, hi, add)
            return
        rad = r[0]
        for z in range(max(0, c[2] - rad), min(world, c[2] + rad + 1)):
            for y in range(max(0, c[1] - rad), min(world, c[1] + rad + 1)):
                rem = rad * rad - (z - c[2]) ** 2 - (y - c[1]) ** 2
                if rem < 0:
                    continue
                dx = int(np.floor(np.sqrt(rem)))
                while dx * dx > rem:
                    dx -= 1
                while (dx + 1) * (dx + 1) <= rem:
                    dx += 1
                x0, x1 = max(0, c[0] - dx), min(world, c[0] + dx + 1)
                if x1 > x0:
                    self.box((x0, y, z), (x1, y + 1, z + 1), add)

    def canon(self) -> DagCanon:
        return _dump_dag(ref().ref_dag_export, self._h, self.depth)

    def import_region(self, base: int, cell, dump: DagCanon) -> None:
        """Load the canonical dump of the cell at level `base` containing voxel
        `cell` (e.g. Sparse(..., base=base, cell=cell).dag()) into this empty
        HashDAG with its own find_or_append_node / _leaf; the rest stays empty."""
        counts = np.ascontiguousarray(dump.counts, np.uint64)
        nodes = np.ascontiguousarray(dump.nodes, np.uint32)
        leaves = np.ascontiguousarray(dump.leaves, np.uint64)
        rc = ref().ref_dag_import_region(self._h, base, *map(int, cell), dump.root,
                                         counts.ctypes.data,
                                         nodes.ctypes.data if nodes.size else None,
                                         leaves.ctypes.data if leaves.size else None)
        if rc != 0:
            raise RuntimeError("reference HashDAG bucket capacity exceeded on import")


class RefSvo:
    """The reference's own CPU SVO (algorithm/lib/include/algo/svt/svo.hpp)."""

    def __init__(self, depth: int):
        self.depth = depth
        self._h = ref().ref_svo_new(depth)
        assert self._h

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_svo_free(self._h)
            self._h = None

    def set_voxel(self, x, y, z, v: bool):
        assert ref().ref_svo_set_voxel(self._h, x, y, z, int(v)) == 0

    def get_voxel(self, x, y, z) -> int:
        return ref().ref_svo_get_voxel(self._h, x, y, z)

    def canon(self) -> SvoCanon:
        nn, nl = C.c_uint32(0), C.c_uint32(0)
        f = ref().ref_svo_export
        f(self._h, C.byref(nn), C.byref(nl), None, 0, None, 0)
        nodes = np.zeros(max(nn.value * 8, 1), np.uint32)
        leaves = np.zeros(max(nl.value, 1), np.uint64)
        assert f(self._h, C.byref(nn), C.byref(nl), nodes.ctypes.data, nn.value,
                 leaves.ctypes.data, nl.value) == 0
        return SvoCanon(nodes[:nn.value * 8], leaves[:nl.value])
