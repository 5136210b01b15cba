"""Batched edits captured as CUDA graphs: a replay computes what the direct
call computes (canonical dumps against the oracle), a graph with a device-side
count edits any number of primitives up to its capacity, rewriting the input
buffer between launches gives the next batch, an over-capacity count is
rejected with the old root kept, and the plain voxel path replays too."""
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


@pytest.mark.parametrize("cap", [256, 512])
def test_dag_graph_with_device_count(cuda, cap):
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(31)
    batches = [rand_prims(rng, n, world, world // 5) for n in (120, 7, 200, 0)]
    buf = torch.zeros((cap, 8), dtype=torch.int32, device=cuda)
    cnt = torch.zeros(1, dtype=torch.int32, device=cuda)
    dag = vx.HashDag(depth, 1 << 18, 64 << 20)
    dag.build_terrain(3, 1, True)
    g = dag.graph_primitives(buf, cnt, cap)
    # within the small-edit threshold the graph holds the single cooperative
    # kernel; above it, the level-by-level launches
    small = cap <= vx.tuning()["edit.small_max_prims"]
    assert g.kernels == 1 if small else g.kernels > depth
    t = oracle.terrain(seed=3, scale=1, caves=True)
    grid = oracle.Grid(depth).terrain(t)
    for b in batches:
        if len(b):
            buf[:len(b)] = vx.prims_to_device(b, cuda)
            grid.apply_prims(b)
        cnt.fill_(len(b))
        launches0 = vx.lib().vx_profile_launches()
        g.launch()
        assert vx.lib().vx_profile_launches() - launches0 == g.kernels
        assert dag.status() == 0
        assert oracle.DagCanon(*dag.canonical()) == grid.dag()
    # a count above the capacity is rejected and the old root stays
    before = oracle.DagCanon(*dag.canonical())
    cnt.fill_(cap + 1)
    g.launch()
    assert dag.status() == vx.VX_ERR_INVALID_VALUE
    assert oracle.DagCanon(*dag.canonical()) == before
    g.close()


def test_svo_graph_fixed_count(cuda):
    depth = 5
    world = 4 << depth
    rng = np.random.default_rng(32)
    prims = rand_prims(rng, 150, world, world // 4)
    d = vx.prims_to_device(prims, cuda)
    s = vx.Svo(depth, 1 << 16, 1 << 16, arena_bytes=32 << 20)
    g = s.graph_primitives(d)
    g.launch()
    assert s.status() == 0
    assert oracle.SvoCanon(*s.canonical()) == oracle.Grid(depth).apply_prims(prims).svo()
    # replay: the same edit again leaves the same content
    g.launch()
    assert s.status() == 0
    assert oracle.SvoCanon(*s.canonical()) == oracle.Grid(depth).apply_prims(prims).svo()


def test_dag_graph_voxels_matches_plain_call(cuda):
    depth = 6
    rng = np.random.default_rng(33)
    xyz = rng.integers(0, 4 << depth, (20000, 3)).astype(np.uint32)
    v = vx.voxels_to_device(xyz, cuda)
    a = vx.HashDag(depth, 1 << 18, 64 << 20)
    g = a.graph_voxels(v, 1)
    g.launch()
    assert a.status() == 0
    b = vx.HashDag(depth, 1 << 18, 64 << 20)
    assert b.apply_voxels(v, 1) == 0
    assert oracle.DagCanon(*a.canonical()) == oracle.DagCanon(*b.canonical())
    assert oracle.DagCanon(*a.canonical()) == oracle.Grid(depth).apply_voxels(xyz, 1).dag()
