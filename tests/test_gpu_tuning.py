"""Every allowed value of every launch-shape knob computes the same result:
radix sorts of each partition variant against the oracle's stable sort
(partial tiles, unaligned arrays, duplicates), batched DAG / SVO edits under
each edit setting against the oracle's canonical dumps; and a quick autotune
run writes a valid settings file."""
import itertools
import json

import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx
from test_tuning import EXPECTED

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _defaults():
    vx.reset_tuning()
    yield
    vx.reset_tuning()


def to_dev(a, device):
    return torch.from_numpy(a.view(np.int64 if a.dtype == np.uint64 else np.int32)).to(device)


@pytest.mark.parametrize("key_bytes,key_bits,n,offset", [
    (4, 32, 1_000_003, 0), (4, 32, 100_000, 1), (4, 20, 3072 * 5, 0),
    (8, 60, 700_001, 0), (8, 64, 65_537, 1), (8, 40, 2048 * 7, 0), (8, 40, 2560 * 7, 0)])
def test_sort_variants_match_oracle(cuda, key_bytes, key_bits, n, offset):
    rng = np.random.default_rng(n + key_bits)
    dt = np.uint64 if key_bytes == 8 else np.uint32
    keys = rng.integers(0, 2**63, n, dtype=np.uint64).astype(dt)
    keys[::5] = keys[3]
    vals = np.arange(n, dtype=np.uint32)
    ek, ev = oracle.stable_sort_pairs(keys, vals, key_bits)
    knob = "sort.items_u32" if key_bytes == 4 else "sort.items_u64"
    for items, early, ballots, radix in itertools.product(
            vx.tuning_options(knob), vx.tuning_options("sort.early_counts"),
            vx.tuning_options("sort.rank_ballots"), vx.tuning_options("sort.radix_bits")):
        vx.set_tuning(knob, items)
        vx.set_tuning("sort.early_counts", early)
        vx.set_tuning("sort.rank_ballots", ballots)
        vx.set_tuning("sort.radix_bits", radix)
        # offset 1: the arrays start one element into a buffer (not 16-byte aligned)
        kbuf = to_dev(np.concatenate([np.zeros(offset, dt), keys]), cuda)
        vbuf = to_dev(np.concatenate([np.zeros(offset, np.uint32), vals]), cuda)
        dk, dv = kbuf[offset:], vbuf[offset:]
        vx.sort_pairs(dk, dv, key_bits)
        assert np.array_equal(dk.cpu().numpy().view(dt), ek), (items, early, ballots, radix)
        assert np.array_equal(dv.cpu().numpy().view(np.uint32), ev), (items, early, ballots, radix)
        dk = to_dev(keys.copy(), cuda)
        vx.sort_pairs(dk, None, key_bits)
        assert np.array_equal(dk.cpu().numpy().view(dt), ek), (items, early, ballots, radix, "keys only")


@pytest.mark.parametrize("n", [1, 1023, 1024, 1025, 2048 * 5 + 3, 4096 * 3, 1_000_003])
def test_scan_tile_shapes_match_oracle(cuda, n):
    """Every prefix-sum tile shape: u32 exclusive / inclusive (aligned and
    4 bytes into a buffer) and u64 exclusive, against the oracle, with one
    workspace reused across shapes (its size covers the smallest tile)."""
    rng = np.random.default_rng(n + 5)
    x32 = rng.integers(0, 2**32, n + 1, dtype=np.uint64).astype(np.uint32)
    x64 = rng.integers(0, 2**63, n, dtype=np.uint64)
    ws = torch.empty(vx.lib().vx_scan_workspace_size(n + 1), dtype=torch.uint8, device=cuda)
    for kb in vx.tuning_options("scan.tile_kb"):
        vx.set_tuning("scan.tile_kb", kb)
        for off in (0, 1):
            d = to_dev(x32, cuda)[off:off + n]
            vx.exclusive_sum(d, ws)
            assert np.array_equal(d.cpu().numpy().view(np.uint32),
                                  oracle.exclusive_sum(x32[off:off + n])), (kb, off)
            assert vx.workspace_status(ws) == 0
            d = to_dev(x32, cuda)[off:off + n]
            vx.inclusive_sum(d, ws)
            assert np.array_equal(d.cpu().numpy().view(np.uint32),
                                  np.cumsum(x32[off:off + n], dtype=np.uint32)), (kb, off, "inc")
        d = to_dev(x64, cuda)
        vx.exclusive_sum(d, ws)
        assert np.array_equal(d.cpu().numpy().view(np.uint64), oracle.exclusive_sum(x64)), (kb, "u64")


def rand_prims(rng, n, world, rmax):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = int(rng.random() < 0.4)
        op = int(rng.random() < 0.55)
        r = rng.integers(0, rmax + 1, 3)
        p[i] = (rng.integers(-3, world + 3, 3), (r[0], r[1] if shape else 0, r[2] if shape else 0),
                shape | (op << 8) | ((1 if op else 0) << 16), 0)
    return p


def test_edit_settings_match_oracle(cuda):
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(21)
    prims = rand_prims(rng, 300, world, world // 4)
    # a long primitive list at the root exercises the block-per-item path
    t = oracle.terrain(seed=4, scale=1, caves=True)
    expect = oracle.Grid(depth).terrain(t).apply_prims(prims)
    for big, bps, lpb, lanes, pf in [(16, 2, 4, 4, 0), (64, 8, 5, 8, 0), (512, 16, 6, 4, 0),
                                     (32, 32, 4, 8, 0), (32, 32, 5, 4, 0), (16, 32, 4, 2, 0),
                                     (32, 16, 5, 2, 0), (16, 8, 6, 2, 0), (32, 32, 5, 4, 1),
                                     (16, 2, 4, 4, 1), (64, 16, 6, 4, 1), (32, 32, 5, 8, 1)]:
        vx.set_tuning("edit.big_item", big)
        vx.set_tuning("edit.blocks_per_sm", bps)
        vx.set_tuning("edit.leafparent_blocks", lpb)
        vx.set_tuning("edit.leafparent_lanes", lanes)
        vx.set_tuning("edit.leafparent_prefetch", pf)
        d = vx.HashDag(depth, 1 << 18, 64 << 20)
        d.build_terrain(4, 1, True)
        d.apply_primitives(vx.prims_to_device(prims, cuda))
        assert d.status() == 0
        assert oracle.DagCanon(*d.canonical()) == expect.dag(), (big, bps, lpb, lanes, pf)
        s = vx.Svo(depth, 1 << 18, 1 << 18, arena_bytes=64 << 20)
        s.build_terrain(4, 1, True)
        s.apply_primitives(vx.prims_to_device(prims, cuda))
        assert s.status() == 0
        assert oracle.SvoCanon(*s.canonical()) == expect.svo(), (big, bps, lpb, lanes, pf)


def test_quick_autotune_writes_settings(cuda, tmp_path):
    from voxel_b200 import autotune
    out = tmp_path / "tune.json"
    res = autotune.main(["--quick", "--quiet", "--out", str(out)])
    saved = json.loads(out.read_text())
    assert saved["knobs"] == res["knobs"]
    for name, value in saved["knobs"].items():
        assert value in vx.tuning_options(name)
    # the run leaves the compiled-in defaults in force
    assert vx.tuning() == EXPECTED


def test_small_edit_kernel_matches_oracle(cuda):
    """The single cooperative kernel for small edits (edit.small_*) computes
    what the multi-launch pipeline does: a primitive batch whose root list
    takes the block-per-item expansion, and plain voxel lists, on the DAG and
    the SVO, at every allowed residency."""
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(33)
    prims = rand_prims(rng, 300, world, world // 4)
    vox = rng.integers(0, world, (3000, 3)).astype(np.uint32)
    t = oracle.terrain(seed=4, scale=1, caves=True)
    expect = oracle.Grid(depth).terrain(t).apply_prims(prims)
    expect.apply_voxels(vox, 1)
    vx.set_tuning("edit.small_max_prims", 4096)
    vx.set_tuning("edit.small_max_voxels", 16384)
    try:
        for blocks in vx.tuning_options("edit.small_blocks_per_sm"):
            vx.set_tuning("edit.small_blocks_per_sm", blocks)
            d = vx.HashDag(depth, 1 << 18, 64 << 20)
            d.build_terrain(4, 1, True)
            d.apply_primitives(vx.prims_to_device(prims, cuda))
            assert d.status() == 0
            assert d.apply_voxels(torch.from_numpy(vox.view(np.int32)).to(cuda), 1) == 0
            assert oracle.DagCanon(*d.canonical()) == expect.dag(), blocks
            s = vx.Svo(depth, 1 << 18, 1 << 18, arena_bytes=64 << 20)
            s.build_terrain(4, 1, True)
            s.apply_primitives(vx.prims_to_device(prims, cuda))
            assert s.status() == 0
            assert s.apply_voxels(torch.from_numpy(vox.view(np.int32)).to(cuda), 1) == 0
            assert oracle.SvoCanon(*s.canonical()) == expect.svo(), blocks
    finally:
        vx.reset_tuning()
