"""The C-ABI library loads without a GPU and exports exactly what the public
header declares (no compute calls here)."""
import re
from pathlib import Path

import voxel_b200

HEADER = Path(__file__).resolve().parent.parent / "include" / "voxel_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(vx_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = voxel_b200.lib()
    declared = declared_functions()
    assert declared, "header parse found no declarations"
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_every_declared_symbol():
    sigs = set(voxel_b200._SIGS)
    missing = [n for n in declared_functions() if n not in sigs]
    assert not missing, f"no ctypes signature for: {missing}"


def test_status_strings_and_workspace_sizes_need_no_device():
    lib = voxel_b200.lib()
    assert lib.vx_version() > 0
    assert voxel_b200.status_string(voxel_b200.VX_ERR_TIMEOUT).startswith("a bounded")
    assert lib.vx_scan_workspace_size(0) == 0
    assert lib.vx_scan_workspace_size(1 << 20) > 0
    assert lib.vx_sort_workspace_size(1, 4) == 0
    assert lib.vx_sort_workspace_size(1 << 20, 8) > lib.vx_sort_workspace_size(1 << 20, 4)


def test_scan_workspace_covers_the_smallest_tile():
    """The scan workspace holds one look-back record per tile of the
    smallest tile shape the "scan.tile_kb" knob offers (8 KB = 1024 u64
    elements): a u64 record is an aggregate, an inclusive value and a state
    word (20 B), plus the tile counter and status (8 B)."""
    lib = voxel_b200.lib()
    smallest_kb = min(voxel_b200.tuning_options("scan.tile_kb"))
    per_tile = smallest_kb * 1024 // 8  # u64 elements per tile
    for n in (1, 1023, 1024, 1025, 1 << 20, 5_000_011, 1 << 28):
        tiles = -(-n // per_tile)
        assert lib.vx_scan_workspace_size(n) >= 8 + 20 * tiles, n
