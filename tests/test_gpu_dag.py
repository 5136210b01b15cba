"""GPU Hash DAG against the oracle: canonical dumps bit-exact after batched
primitive edits, the plain per-call voxel path and terrain builds; the
reference's test cases (test/cuda/test_cuda_hash_dag_gpu.cu) as known answers."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def canon(dag: vx.HashDag) -> oracle.DagCanon:
    return oracle.DagCanon(*dag.canonical())


def rand_prims(rng, n, world, rmax, sphere_frac=0.6, add_frac=0.55):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = 0 if rng.random() < sphere_frac else 1
        op = int(rng.random() < add_frac)
        r = rng.integers(0, rmax + 1, 3)
        p[i] = (rng.integers(-3, world + 3, 3), (r[0], r[1] if shape else 0, r[2] if shape else 0),
                shape | (op << 8), 0)
    return p


@pytest.mark.parametrize("depth,n,seed", [(1, 10, 0), (2, 30, 1), (3, 60, 2),
                                          (5, 200, 3), (6, 400, 4), (8, 300, 5)])
def test_batched_primitives_match_oracle(cuda, depth, n, seed):
    rng = np.random.default_rng(seed)
    world = 4 << depth
    prims = rand_prims(rng, n, world, max(2, world // 5))
    dag = vx.HashDag(depth, max_nodes=1 << 18, arena_bytes=64 << 20)
    dag.apply_primitives(vx.prims_to_device(prims, cuda))
    assert dag.status() == 0
    assert canon(dag) == oracle.Grid(depth).apply_prims(prims).dag()


def test_large_spheres_match_sparse_oracle(cuda):
    """Sphere leaf masks take single precision up to radius 1024 and 32-bit
    integers above: radii on both sides of the switch (and near the world's
    size), adds and removes, against the sparse CPU oracle at 4096^3."""
    depth = 10
    world = 4 << depth
    rng = np.random.default_rng(77)
    radii = [1, 2, 3, 700, 1020, 1023, 1024, 1025, 1026, 1100, 1500, 2047, 3000]
    p = np.zeros(len(radii), oracle.PRIM_DTYPE)
    for i, r in enumerate(radii):
        c = rng.integers(-r // 2, world + r // 2, 3)
        op = int(i % 3 != 2)
        p[i] = (c, (r, 0, 0), (op << 8), 0)
    dag = vx.HashDag(depth, max_nodes=1 << 22, arena_bytes=1 << 30)
    dag.apply_primitives(vx.prims_to_device(p, cuda))
    assert dag.status() == 0
    assert canon(dag) == oracle.Sparse(depth, None, p).dag()


@pytest.mark.parametrize("depth,caves", [(4, False), (5, True), (7, True)])
def test_terrain_build_matches_oracle(cuda, depth, caves):
    t = oracle.terrain(seed=1, scale=1 if depth <= 6 else 2, caves=caves)
    dag = vx.HashDag(depth, max_nodes=1 << 20, arena_bytes=128 << 20)
    dag.build_terrain(int(t["seed"][0]), int(t["scale"][0]), caves)
    assert dag.status() == 0
    assert canon(dag) == oracle.Grid(depth).terrain(t).dag()


def test_terrain_then_batches_then_queries(cuda):
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(11)
    t = oracle.terrain(seed=7, scale=1, caves=True)
    dag = vx.HashDag(depth, max_nodes=1 << 20, arena_bytes=128 << 20)
    dag.build_terrain(7, 1, True)
    g = oracle.Grid(depth).terrain(t)
    all_prims = []
    for b in range(3):  # three batches in a row, copy-on-write over shared nodes
        prims = rand_prims(rng, 150, world, 24)
        all_prims.append(prims)
        dag.apply_primitives(vx.prims_to_device(prims, cuda))
        g.apply_prims(prims)
        assert dag.status() == 0
        assert canon(dag) == g.dag()
    pts = rng.integers(0, world + 8, (5000, 3)).astype(np.uint32)
    got = dag.query(vx.voxels_to_device(pts, cuda)).cpu().numpy()
    inside = (pts < world).all(axis=1)
    expect = np.zeros(len(pts), np.uint8)
    expect[inside] = oracle.eval_voxels(t, depth + 2, np.concatenate(all_prims), pts[inside])
    assert np.array_equal(got, expect)


def test_batch_equals_two_halves(cuda):
    depth = 7
    rng = np.random.default_rng(3)
    prims = rand_prims(rng, 600, 4 << depth, 40)
    a = vx.HashDag(depth, max_nodes=1 << 20, arena_bytes=64 << 20)
    a.apply_primitives(vx.prims_to_device(prims, cuda))
    b = vx.HashDag(depth, max_nodes=1 << 20, arena_bytes=64 << 20)
    b.apply_primitives(vx.prims_to_device(prims[:250], cuda))
    b.apply_primitives(vx.prims_to_device(prims[250:], cuda))
    assert a.status() == 0 and b.status() == 0
    assert canon(a) == canon(b)


def spread_edits(count):
    """make_spread_edits (test/cuda/test_cuda_hash_dag_gpu.cu:142-156)."""
    out = []
    for i in range(count):
        if i % 19 == 0:
            out.append((1024 + i, 0, 0))
        else:
            out.append(((i * 37) & 1023, (i * 91 + 3) & 1023, (i * 53 + 7) & 1023))
    return np.array(out, np.uint32)


@pytest.mark.parametrize("count", [31, 32, 33, 255, 256, 257])
def test_plain_voxels_boundary_batches(cuda, count):
    """Boundary batch sizes with out-of-world edits ignored
    (test_cuda_hash_dag_gpu.cu:423-468)."""
    depth = 8  # 1024^3, the reference GPU DAG's world
    edits = spread_edits(count)
    dag = vx.HashDag(depth, max_nodes=1 << 16, arena_bytes=32 << 20)
    assert dag.apply_voxels(vx.voxels_to_device(edits, cuda), vx.EDIT_PLACE) == 0
    g = oracle.Grid(depth).apply_voxels(edits, 1)
    assert canon(dag) == g.dag()
    assert dag.apply_voxels(vx.voxels_to_device(edits[::3], cuda), vx.EDIT_DESTROY) == 0
    g.apply_voxels(edits[::3], 0)
    assert canon(dag) == g.dag()
    got = dag.query(vx.voxels_to_device(edits, cuda)).cpu().numpy()
    inside = (edits < 1024).all(axis=1)
    assert got[~inside].sum() == 0
    assert got[inside].tolist() == [g.get(*e) for e in edits[inside]]


def test_plain_voxels_duplicates_dedup_and_siblings(cuda):
    depth = 8
    dag = vx.HashDag(depth, max_nodes=1 << 16, arena_bytes=32 << 20)
    # in-batch duplicates, two identical leaves in different places (dedup),
    # sibling leaves of one parent, a full 4^3 leaf
    e = [(1, 2, 3), (1, 2, 3), (1, 2, 3), (101, 102, 103), (5, 2, 3), (1, 6, 3)]
    e += [(x, y, z) for x in range(8, 12) for y in range(4) for z in range(4)]
    e = np.array(e, np.uint32)
    assert dag.apply_voxels(vx.voxels_to_device(e, cuda), vx.EDIT_PLACE) == 0
    g = oracle.Grid(depth).apply_voxels(e, 1)
    assert canon(dag) == g.dag()


def test_plain_voxels_sphere_matches_batched_sphere(cuda):
    depth = 7
    world = 4 << depth
    c, r = np.array([200, 180, 230]), 37
    ax = np.arange(-r, r + 1)
    zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
    inside = xx ** 2 + yy ** 2 + zz ** 2 <= r * r
    vox = (np.stack([xx[inside], yy[inside], zz[inside]], 1) + c).astype(np.int64)
    vox = vox[(vox >= 0).all(1) & (vox < world).all(1)].astype(np.uint32)
    a = vx.HashDag(depth, max_nodes=1 << 18, arena_bytes=64 << 20)
    assert a.apply_voxels(vx.voxels_to_device(vox, cuda), vx.EDIT_PLACE) == 0
    p = np.zeros(1, oracle.PRIM_DTYPE)
    p[0] = (c, (r, 0, 0), 1 << 8, 0)
    b = vx.HashDag(depth, max_nodes=1 << 18, arena_bytes=64 << 20)
    b.apply_primitives(vx.prims_to_device(p, cuda))
    assert b.status() == 0
    assert canon(a) == canon(b)


def test_plain_api_rejections_leave_dag_intact(cuda):
    """test_cuda_hash_dag_gpu.cu:470-512: bad arguments return
    cudaErrorInvalidValue and change nothing; count 0 is a no-op."""
    depth = 8
    dag = vx.HashDag(depth, max_nodes=1 << 16, arena_bytes=32 << 20)
    e = vx.voxels_to_device(np.array([[5, 6, 7]], np.uint32), cuda)
    assert dag.apply_voxels(e, vx.EDIT_PLACE) == 0
    before = canon(dag)
    lib = vx.lib()
    ws = torch.empty(4, dtype=torch.uint8, device=cuda)
    s = vx.stream_handle()
    h = dag._h
    assert lib.vx_dag_apply_voxels(h, None, 3, 1, ws.data_ptr(), 4, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_voxels(h, e.data_ptr(), 1, 1, ws.data_ptr(), 4, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_voxels(h, e.data_ptr(), 1, 1, None, 0, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_voxels(h, None, 0, 1, None, 0, s) == vx.VX_OK
    assert canon(dag) == before


def test_capacity_overflow_keeps_previous_root(cuda):
    """A node table that runs out reports the capacity error and the previous
    root stays published (test_cuda_hash_dag_gpu.cu:514-535)."""
    depth = 6
    dag = vx.HashDag(depth, max_nodes=16, arena_bytes=16 << 20)
    small = np.array([[1, 1, 1]], np.uint32)
    assert dag.apply_voxels(vx.voxels_to_device(small, cuda), vx.EDIT_PLACE) == 0
    before = canon(dag)
    rng = np.random.default_rng(1)
    many = rng.integers(0, 4 << depth, (5000, 3)).astype(np.uint32)
    st = dag.apply_voxels(vx.voxels_to_device(many, cuda), vx.EDIT_PLACE)
    assert st == vx.VX_ERR_CAPACITY
    assert canon(dag) == before
    # the error was reported once: the next edit starts from a clear status
    assert dag.apply_voxels(vx.voxels_to_device(small, cuda), vx.EDIT_PLACE) == 0
    assert canon(dag) == before


def test_rasterize_matches_voxel_definition(cuda):
    rng = np.random.default_rng(21)
    depth = 5
    world = 4 << depth
    prims = rand_prims(rng, 40, world, 20)
    vox, off = vx.rasterize(vx.prims_to_device(prims, cuda), depth + 2)
    vox = vox.cpu().numpy().view(np.uint32)
    off = off.cpu().numpy()
    for i, p in enumerate(prims):
        got = {tuple(v) for v in vox[off[i]:off[i + 1]].tolist()}
        assert len(got) == off[i + 1] - off[i]
        single = np.zeros(1, oracle.PRIM_DTYPE)
        single[0] = p
        single[0]["flags"] = int(p["flags"]) | (1 << 8)
        g = oracle.Grid(depth).apply_prims(single)
        assert g.count() == len(got)
        assert all(g.get(*v) for v in list(got)[:200])


def test_copy_restores_snapshot(cuda):
    depth = 6
    rng = np.random.default_rng(5)
    a = vx.HashDag(depth, max_nodes=1 << 18, arena_bytes=32 << 20)
    a.build_terrain(2, 1, True)
    b = vx.HashDag(depth, max_nodes=1 << 18, arena_bytes=32 << 20)
    b.copy_from(a)
    assert canon(b) == canon(a)
    prims = rand_prims(rng, 80, 4 << depth, 20)
    b.apply_primitives(vx.prims_to_device(prims, cuda))
    assert b.status() == 0
    t = oracle.terrain(2, 1, True)
    assert canon(b) == oracle.Grid(depth).terrain(t).apply_prims(prims).dag()
    b.copy_from(a)
    assert canon(b) == canon(a)


def test_compaction_keeps_content_and_frees_garbage(cuda):
    depth = 7
    rng = np.random.default_rng(31)
    t = oracle.terrain(seed=4, scale=2, caves=True)
    dag = vx.HashDag(depth, max_nodes=1 << 20, arena_bytes=64 << 20)
    dag.build_terrain(4, 2, True)
    g = oracle.Grid(depth).terrain(t)
    for _ in range(5):  # several batches: plenty of superseded items
        prims = rand_prims(rng, 120, 4 << depth, 30)
        dag.apply_primitives(vx.prims_to_device(prims, cuda))
        g.apply_prims(prims)
    assert dag.status() == 0
    before = dag.stats()
    dag.compact()
    after = dag.stats()
    c = canon(dag)
    assert c == g.dag()
    # after compaction the tables hold exactly the live (canonical) nodes
    assert [int(after.nodes_per_level[l]) for l in range(depth + 1)] == c.counts
    assert sum(after.nodes_per_level) < sum(before.nodes_per_level)
    # editing continues normally on the compacted tables
    prims = rand_prims(rng, 60, 4 << depth, 30)
    dag.apply_primitives(vx.prims_to_device(prims, cuda))
    g.apply_prims(prims)
    assert dag.status() == 0
    assert canon(dag) == g.dag()
