"""Pin the sparse CPU oracle (oracle_sparse.cpp: sequential application on a
hash-consed DAG, the checker of the full-size configurations) against the
dense Grid oracle and the reference's own CPU HashDAG / SVO, and check the
terrain evaluation it prunes and caches with against the voxel-by-voxel
definition."""
import numpy as np
import pytest

import oracle
from test_oracle_voxel import rand_prims

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference shim not built (no reference tree)")


def gen_prims(world_exp, count, seed, **kw):
    return oracle.generate_primitives(world_exp, count, seed, **kw)


@pytest.mark.parametrize("depth,shards,caves,seed", [(3, 0, True, 1), (4, 1, True, 2),
                                                     (5, 2, True, 3), (6, 3, False, 4),
                                                     (6, 2, True, 5)])
def test_sparse_dag_and_svo_match_dense_grid(depth, shards, caves, seed):
    world = 4 << depth
    rng = np.random.default_rng(seed)
    prims = rand_prims(rng, 60, world, max(2, world // 5), sphere_frac=0.6)
    t = oracle.terrain(seed=7, scale=1, caves=caves)
    g = oracle.Grid(depth).terrain(t).apply_prims(prims)
    s = oracle.Sparse(depth, t, prims, shard_levels=shards, threads=3)
    assert s.dag() == g.dag()
    assert s.svo() == g.svo()


@pytest.mark.parametrize("depth,shards", [(4, 1), (5, 2)])
def test_sparse_svo_with_materials_matches_dense_grid(depth, shards):
    world = 4 << depth
    prims = gen_prims(depth + 2, 80, 6, sphere_permille=700, r_min=1, r_max=world // 6,
                      log_uniform=True)
    t = oracle.terrain(seed=7, scale=1, caves=True)
    g = oracle.Grid(depth, materials=True).terrain(t).apply_prims(prims)
    s = oracle.Sparse(depth, t, prims, materials=True, shard_levels=shards, threads=2)
    got, want = s.svo(), g.svo()
    assert got == want and np.array_equal(got.mats, want.mats)
    assert s.dag() == g.dag()  # occupancy of the material world


@needs_ref
@pytest.mark.parametrize("depth,n,seed", [(2, 20, 11), (4, 50, 12), (5, 30, 13)])
def test_sparse_dag_matches_reference_hashdag(depth, n, seed):
    """Primitives on an empty world, applied by the reference HashDAG as x-run
    boxes (fill_box / clear_box) and by the sparse oracle recursively."""
    rng = np.random.default_rng(seed)
    world = 4 << depth
    prims = rand_prims(rng, n, world, max(2, world // 4))
    ref = oracle.RefDag(depth)
    for p in prims:
        ref.apply_prim_runs(p)
    s = oracle.Sparse(depth, None, prims, shard_levels=min(2, depth), threads=2)
    assert s.dag() == ref.canon()


@needs_ref
def test_sparse_svo_matches_reference_svo():
    depth = 4
    rng = np.random.default_rng(21)
    world = 4 << depth
    ref = oracle.RefSvo(depth)
    vox = rng.integers(0, world, (700, 3))
    ops = rng.random(700) < 0.7
    prims = np.zeros(700, oracle.PRIM_DTYPE)
    for i, (v, on) in enumerate(zip(vox, ops)):
        ref.set_voxel(*map(int, v), bool(on))
        prims[i] = (v, (1, 1, 1), 4 | (int(on) << 8), 0)  # 1^3 half-open box
    s = oracle.Sparse(depth, None, prims, shard_levels=1, threads=2)
    assert s.svo() == ref.canon()


def test_sparse_plain_voxels_deep_keys():
    """Single voxels at depth 12 (16384^3): the plain path's 36-bit leaf keys;
    the region dump around them equals a dense Grid of the same region."""
    depth = 12
    rng = np.random.default_rng(3)
    base = 6  # 256^3 region
    cell = np.array([9000, 13000, 300], np.uint32)
    side = 4 << (depth - base)
    o = (cell // side) * side
    vox = o + rng.integers(0, side, (500, 3)).astype(np.uint32)
    prims = np.zeros(500, oracle.PRIM_DTYPE)
    prims["c"] = vox
    prims["r"] = 1
    prims["flags"] = 4 | (1 << 8)
    s = oracle.Sparse(depth, None, prims, base=base, cell=cell, shard_levels=1, threads=2)
    local = prims.copy()
    local["c"] -= o.astype(np.int32)
    g = oracle.Grid(depth - base).apply_prims(local)
    assert s.dag() == g.dag()


def test_sparse_region_equals_whole_world():
    """A region built alone equals the same cell of the whole world."""
    depth = 6
    t = oracle.terrain(seed=9, scale=1, caves=True)
    prims = gen_prims(depth + 2, 200, 8, sphere_permille=500, r_min=1, r_max=20,
                      log_uniform=True)
    whole = oracle.Sparse(depth, t, prims, shard_levels=2, threads=4)
    for base, cell in [(2, (70, 10, 200)), (3, (0, 250, 130)), (1, (200, 200, 0))]:
        part = oracle.Sparse(depth, t, prims, base=base, cell=cell, shard_levels=1, threads=2)
        n = 1 << (depth - base)
        lo = [(c // 4 // n) * n for c in cell]
        assert np.array_equal(part.leaf_block(lo, [n, n, n]), whole.leaf_block(lo, [n, n, n]))


def test_terrain_leaf_evaluation_matches_voxel_definition():
    rng = np.random.default_rng(0)
    for scale, caves in [(1, True), (16, True), (64, True), (32, False)]:
        t = oracle.terrain(seed=7, scale=scale, caves=caves, world_exp=14)
        side = 4 << 12
        xy = rng.integers(0, side // 4, (3000, 2)) * 4
        # near the surface band, where leaves are mixed
        z = (128 * scale + rng.integers(-60 * scale, 60 * scale, 3000)) // 4 * 4
        org = np.column_stack([xy, np.clip(z, 0, side - 4)]).astype(np.uint32)
        assert oracle.terrain_leaf_mismatches(t, org, False) == 0
        assert oracle.terrain_leaf_mismatches(t, org, True) == 0


def test_terrain_classification_is_exact_where_it_decides():
    """Cubes called full or empty by the classification really are (the
    sparse build prunes with it)."""
    rng = np.random.default_rng(1)
    for scale in (1, 64):
        t = oracle.terrain(seed=7, scale=scale, caves=True, world_exp=14)
        cubes = []
        for n in (4, 8, 16, 32):
            for _ in range(150):
                x, y = rng.integers(0, (4 << 12) - n, 2)
                z = int(np.clip(128 * scale + rng.integers(-50 * scale, 50 * scale),
                                0, (4 << 12) - n))
                cubes.append((x // n * n, y // n * n, z // n * n, n))
        assert oracle.terrain_classify_mismatches(t, np.array(cubes)) == 0


@needs_ref
def test_sparse_matches_reference_on_c4_terrain_cell():
    """The benchmark's reference sample: the reference HashDAG(12) loaded with
    the cave terrain (scale 64) of one 2048^3 cell of the C4 world through its
    own find_or_append_node, then edited with C4 spheres that reach the cell
    (x-runs clipped to it), equals the sparse oracle's sequential application
    on that cell."""
    depth, base, cell = 12, 3, (8192, 8192, 8192)
    t = oracle.terrain(7, 64, True)
    side = 4 << (depth - base)
    lo = np.array([c // side * side for c in cell], np.int64)
    hi = lo + side
    prims = oracle.config_c4_edits(16384)
    c = prims["c"].astype(np.int64)
    r = prims["r"][:, 0].astype(np.int64)
    reach = np.all((c + r[:, None] >= lo) & (c - r[:, None] < hi), axis=1)
    spheres = prims[reach][:6]
    ref = oracle.RefDag(depth)
    ref.import_region(base, cell, oracle.Sparse(depth, t, None, base=base, cell=cell,
                                                shard_levels=2).dag())
    f = oracle.ref().ref_dag_apply_prim_clipped
    for p in spheres:
        fl = int(p["flags"])
        assert f(ref._h, fl & 0xFF, *map(int, p["c"]), *map(int, p["r"]),
                 int(((fl >> 8) & 0xFF) == 1), lo.ctypes.data, hi.ctypes.data) >= 0
    want = oracle.Sparse(depth, t, spheres, base=base, cell=cell, shard_levels=2).dag()
    got = ref.canon()
    skip = int(sum(got.counts[:base])) * 10
    assert got.counts[base:] == want.counts
    assert np.array_equal(got.nodes[skip:], want.nodes)
    assert np.array_equal(got.leaves, want.leaves)


def test_oracle_generators_match_the_library():
    import voxel_b200 as vx
    assert np.array_equal(oracle.config_c4_edits(3000), vx.config_c4_edits(3000))
    assert np.array_equal(oracle.config_c3_edits(3000), vx.config_c3_edits(3000))
    a = oracle.generate_requests(13, 2000.0, 0.5, 8)
    b = vx.generate_requests(13, 2000.0, 0.5, 8)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
