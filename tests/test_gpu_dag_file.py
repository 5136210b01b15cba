"""Checkpoint / resume of a Hash DAG: save the canonical dump to a file, load
it into fresh DAGs (same depth, other capacities) and get the same content;
editing continues after a load; malformed files and too-small DAGs are
rejected with the old state reported, not a fault."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def rand_prims(rng, n, world, rmax):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = int(rng.random() < 0.4)
        op = int(rng.random() < 0.55)
        r = rng.integers(0, rmax + 1, 3)
        p[i] = (rng.integers(-3, world + 3, 3), (r[0], r[1] if shape else 0, r[2] if shape else 0),
                shape | (op << 8) | ((1 if op else 0) << 16), 0)
    return p


def canon(d):
    return oracle.DagCanon(*d.canonical())


def test_save_load_round_trip(cuda, tmp_path):
    depth = 7
    world = 4 << depth
    rng = np.random.default_rng(61)
    a = vx.HashDag(depth, 1 << 20, 128 << 20)
    a.build_terrain(5, 2, True)
    p1 = rand_prims(rng, 300, world, world // 6)
    a.apply_primitives(vx.prims_to_device(p1, cuda))
    assert a.status() == 0
    path = tmp_path / "dag.vxdag"
    a.save(path)
    b = vx.HashDag(depth, 1 << 19, 64 << 20)  # other capacity, same depth
    assert b.load(path) == 0
    assert canon(b) == canon(a)
    g = torch.Generator(device=cuda)
    g.manual_seed(3)
    pts = torch.randint(0, world, (500_000, 3), dtype=torch.int32, device=cuda, generator=g)
    assert torch.equal(a.query(pts), b.query(pts))
    # editing continues on the loaded DAG exactly as on the original
    p2 = rand_prims(rng, 200, world, world // 6)
    for d in (a, b):
        d.apply_primitives(vx.prims_to_device(p2, cuda))
        assert d.status() == 0
    assert canon(a) == canon(b)
    t = oracle.terrain(5, 2, True)
    assert canon(b) == oracle.Grid(depth).terrain(t).apply_prims(p1).apply_prims(p2).dag()


def test_uniform_worlds_and_rejections(cuda, tmp_path):
    depth = 4
    full = vx.HashDag(depth, 1 << 16, 16 << 20)
    p = np.zeros(1, oracle.PRIM_DTYPE)
    p[0] = ((0, 0, 0), (1 << 10, 1 << 10, 1 << 10), 1 | (1 << 8) | (1 << 16), 0)  # covers all
    full.apply_primitives(vx.prims_to_device(p, cuda))
    assert full.status() == 0
    path = tmp_path / "full.vxdag"
    full.save(path)
    e = vx.HashDag(depth, 1 << 16, 16 << 20)
    assert e.load(path) == 0
    assert canon(e) == canon(full) and canon(e).root == 1
    # wrong depth, bad magic, missing file
    other = vx.HashDag(depth + 1, 1 << 16, 16 << 20)
    assert other.load(path) == vx.VX_ERR_INVALID_VALUE
    bad = tmp_path / "bad.vxdag"
    bad.write_bytes(b"NOTADAG!" + bytes(64))
    assert e.load(bad) == vx.VX_ERR_INVALID_VALUE
    assert e.load(tmp_path / "missing.vxdag") == vx.VX_ERR_IO
    # a DAG too small for the dump is refused before anything changes
    rng = np.random.default_rng(62)
    big = vx.HashDag(6, 1 << 18, 64 << 20)
    big.build_terrain(2, 1, True)
    big.save(tmp_path / "big.vxdag")
    small = vx.HashDag(6, 16, 16 << 20)
    before = canon(small)
    assert small.load(tmp_path / "big.vxdag") == vx.VX_ERR_CAPACITY
    assert canon(small) == before
