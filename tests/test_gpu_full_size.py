"""The GPU edit paths against the sparse CPU oracle (sequential application,
oracle/oracle_sparse.cpp) at the benchmark configurations' full sizes and
depths: the batched Hash DAG on the 16384^3 cave terrain with the full
16,384-sphere batch, the batched SVO with materials on the 4096^3 terrain,
and the plain per-call voxel path at depths 11 and 12, whose 33- / 36-bit
leaf keys only exist there."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


@pytest.mark.slow
def test_c4_batch_full_size_matches_oracle(cuda):
    depth = 12
    prims = vx.config_c4_edits(16384, seed=7, world_exp=depth + 2)
    dag = vx.HashDag(depth, 1 << 27, 16 << 30)
    dag.build_terrain(7, 64, True)
    assert dag.status() == 0
    dag.apply_primitives(vx.prims_to_device(prims, cuda))
    assert dag.status() == 0
    got = oracle.DagCanon(*dag.canonical())
    del dag
    torch.cuda.empty_cache()
    assert got == oracle.Sparse(depth, oracle.terrain(7, 64, True), prims).dag()


@pytest.mark.slow
def test_c3_batch_full_size_matches_oracle(cuda):
    depth = 10
    prims = vx.config_c3_edits(65536, seed=6, world_exp=depth + 2)
    svo = vx.Svo(depth, 1 << 25, 1 << 27, materials=True, arena_bytes=8 << 30)
    svo.build_terrain(6, 16, True)
    svo.apply_primitives(vx.prims_to_device(prims, cuda))
    assert svo.status() == 0
    got = oracle.SvoCanon(*svo.canonical())
    del svo
    torch.cuda.empty_cache()
    want = oracle.Sparse(depth, oracle.terrain(6, 16, True), prims, materials=True).svo()
    assert got == want and np.array_equal(got.mats, want.mats)


def voxel_batches(rng, world, n_batches, per_batch):
    """Clustered and spread voxels over the whole world (so the leaf keys'
    top bits vary), with duplicates and out-of-world entries."""
    out = []
    for _ in range(n_batches):
        centres = rng.integers(0, world, (24, 3))
        near = (centres[rng.integers(0, 24, per_batch // 2)]
                + rng.integers(-40, 41, (per_batch // 2, 3)))
        spread = rng.integers(0, world, (per_batch // 2, 3))
        v = np.concatenate([near, spread, near[:500]])
        v[::97] = world + 5  # ignored
        out.append(np.clip(v, 0, world + 5).astype(np.uint32))
    return out


@pytest.mark.parametrize("depth", [11, 12])
def test_plain_voxel_path_deep_levels_matches_oracle(cuda, depth):
    world = 4 << depth
    rng = np.random.default_rng(depth)
    batches = voxel_batches(rng, world, 3, 40_000)
    ops = [1, 1, 0]
    dag = vx.HashDag(depth, 1 << 21, 1 << 30)
    prims = []
    for v, op in zip(batches, ops):
        assert dag.apply_voxels(torch.from_numpy(v.view(np.int32)).to(cuda), op) == 0
        inside = v[(v < world).all(axis=1)]
        p = np.zeros(len(inside), oracle.PRIM_DTYPE)
        p["c"] = inside
        p["r"] = 1
        p["flags"] = 4 | (op << 8)  # 1^3 half-open box
        prims.append(p)
    got = oracle.DagCanon(*dag.canonical())
    want = oracle.Sparse(depth, None, np.concatenate(prims), shard_levels=2).dag()
    assert got == want
    assert sum(got.counts) > 1000


@pytest.mark.parametrize("depth", [11, 12])
def test_region_leaf_read_matches_oracle(cuda, depth):
    """vx_dag_read_leaves over a region of an edited terrain DAG equals the
    oracle's leaf masks there."""
    scale = 32 if depth == 11 else 64
    prims = vx.config_c4_edits(2000, seed=3, world_exp=depth + 2)
    dag = vx.HashDag(depth, 1 << 27, 8 << 30)
    dag.build_terrain(8, scale, True)
    dag.apply_primitives(vx.prims_to_device(prims, cuda))
    assert dag.status() == 0
    base = 5
    side = 4 << (depth - base)
    cell = (side * 3, side * 7, 4096 * scale // 32)
    lo = [c // side * side // 4 for c in cell]
    n = side // 4
    got = dag.read_leaves(lo, (n, n, n)).cpu().numpy().view(np.uint64)
    want = oracle.Sparse(depth, oracle.terrain(8, scale, True), prims, base=base, cell=cell,
                         shard_levels=1).leaf_block(lo, (n, n, n))
    assert np.array_equal(got, want)
    assert 0 < np.count_nonzero(got) < got.size  # the region holds the surface
