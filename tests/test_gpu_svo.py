"""GPU SVO against the oracle (pinned to the reference's CPU SVO): canonical
node arrays, leaves and materials bit-exact after batched primitives, the
plain voxel path, terrain builds; queries; counters; capacity."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def canon(s: vx.Svo) -> oracle.SvoCanon:
    return oracle.SvoCanon(*s.canonical())


def rand_prims(rng, n, world, rmax, sphere_frac=0.6, add_frac=0.55, materials=True):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = 0 if rng.random() < sphere_frac else 1
        op = int(rng.random() < add_frac)
        r = rng.integers(0, rmax + 1, 3)
        mat = int(rng.integers(1, 256)) if (op and materials) else (1 if op else 0)
        p[i] = (rng.integers(-3, world + 3, 3), (r[0], r[1] if shape else 0, r[2] if shape else 0),
                shape | (op << 8) | (mat << 16), 0)
    return p


@pytest.mark.parametrize("depth,n,seed,mats", [(1, 12, 0, False), (2, 30, 1, False),
                                               (3, 80, 2, True), (5, 200, 3, False),
                                               (5, 200, 4, True), (6, 300, 5, True)])
def test_batched_primitives_match_oracle(cuda, depth, n, seed, mats):
    rng = np.random.default_rng(seed)
    world = 4 << depth
    prims = rand_prims(rng, n, world, max(2, world // 5), materials=mats)
    s = vx.Svo(depth, 1 << 18, 1 << 18, materials=mats, arena_bytes=64 << 20)
    s.apply_primitives(vx.prims_to_device(prims, cuda))
    assert s.status() == 0
    assert canon(s) == oracle.Grid(depth, materials=mats).apply_prims(prims).svo()


@pytest.mark.parametrize("depth,caves,mats", [(4, False, False), (5, True, True),
                                              (6, True, False)])
def test_terrain_build_matches_oracle(cuda, depth, caves, mats):
    t = oracle.terrain(seed=1, scale=1, caves=caves)
    s = vx.Svo(depth, 1 << 20, 1 << 20, materials=mats, arena_bytes=64 << 20)
    s.build_terrain(1, 1, caves)
    assert s.status() == 0
    assert canon(s) == oracle.Grid(depth, materials=mats).terrain(t).svo()


@pytest.mark.parametrize("mats", [False, True])
def test_terrain_then_batches_queries_and_gc(cuda, mats):
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(12)
    t = oracle.terrain(seed=7, scale=1, caves=True)
    s = vx.Svo(depth, 1 << 18, 1 << 18, materials=mats, arena_bytes=64 << 20)
    s.build_terrain(7, 1, True)
    g = oracle.Grid(depth, materials=mats).terrain(t)
    all_prims = []
    for _ in range(4):
        prims = rand_prims(rng, 120, world, 30, materials=mats)
        all_prims.append(prims)
        s.apply_primitives(vx.prims_to_device(prims, cuda))
        g.apply_prims(prims)
        assert s.status() == 0
        assert canon(s) == g.svo()
    pts = rng.integers(0, world + 8, (5000, 3)).astype(np.uint32)
    got = s.query(vx.voxels_to_device(pts, cuda)).cpu().numpy()
    inside = (pts < world).all(axis=1)
    expect = np.zeros(len(pts), np.uint8)
    expect[inside] = oracle.eval_voxels(t, depth + 2, np.concatenate(all_prims), pts[inside],
                                        materials=mats)
    assert np.array_equal(got, expect)
    # after a collection, live structure = counters minus free lists
    s.collect()
    c = s.counters()
    nodes, leaves, _ = s.canonical()
    assert c.node_count - c.free_node_count == nodes.size // 8
    assert c.leaf_count - c.free_leaf_count == leaves.size


def test_plain_voxels_match_reference_semantics(cuda):
    """The plain path (one op per voxel list) against the oracle, which is
    pinned to the reference SVO::set_voxel; config C1's 256^3 world."""
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(8)
    s = vx.Svo(depth, 1 << 16, 1 << 16, arena_bytes=32 << 20)
    g = oracle.Grid(depth)
    for i in range(12):
        c = rng.integers(0, world, 3)
        r = int(rng.integers(2, 17))
        ax = np.arange(-r, r + 1)
        zz, yy, xx = np.meshgrid(ax, ax, ax, indexing="ij")
        ins = xx ** 2 + yy ** 2 + zz ** 2 <= r * r
        vox = np.stack([xx[ins], yy[ins], zz[ins]], 1) + c
        vox = vox[(vox >= 0).all(1) & (vox < world).all(1)].astype(np.uint32)
        op = i % 2 == 0 or i % 3 == 0
        assert s.apply_voxels(vx.voxels_to_device(vox, cuda), int(op)) == 0
        g.apply_voxels(vox, int(op))
        assert canon(s) == g.svo()


def test_plain_out_of_world_and_rejections(cuda):
    depth = 4
    s = vx.Svo(depth, 1 << 12, 1 << 12, arena_bytes=8 << 20)
    e = np.array([[1, 2, 3], [70, 1, 1], [1, 999, 1], [4, 4, 4]], np.uint32)
    assert s.apply_voxels(vx.voxels_to_device(e, cuda), vx.EDIT_PLACE) == 0
    g = oracle.Grid(depth).apply_voxels(e, 1)
    assert canon(s) == g.svo()
    lib = vx.lib()
    st = vx.stream_handle()
    assert lib.vx_svo_apply_voxels(s._h, None, 3, 1, 1, None, 0, st) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_svo_apply_voxels(s._h, None, 0, 1, 1, None, 0, st) == vx.VX_OK
    assert canon(s) == g.svo()


def test_capacity_overflow_changes_nothing(cuda):
    depth = 6
    s = vx.Svo(depth, 64, 64, arena_bytes=8 << 20)
    small = np.array([[1, 1, 1]], np.uint32)
    assert s.apply_voxels(vx.voxels_to_device(small, cuda), vx.EDIT_PLACE) == 0
    before = canon(s)
    many = np.random.default_rng(2).integers(0, 4 << depth, (3000, 3)).astype(np.uint32)
    assert s.apply_voxels(vx.voxels_to_device(many, cuda), vx.EDIT_PLACE) == vx.VX_ERR_CAPACITY
    assert canon(s) == before
    # the error was reported once: the next edit starts from a clear status
    assert s.apply_voxels(vx.voxels_to_device(small, cuda), vx.EDIT_PLACE) == 0
    assert canon(s) == before


@pytest.mark.parametrize("small_max_prims", [256, 0])
def test_lazy_collection_reclaims_detached_subtrees(cuda, small_max_prims):
    """Edits collect garbage only when they would not fit otherwise: a cycle
    of (carve a sphere, fill the world) detaches every carved subtree, so 40
    cycles need about 40 spheres' storage without collection; in room for
    ten (the capacity check reserves a node per work item and 8 leaves per
    leaf-parent item, more than a sphere keeps) they all succeed, through the
    single cooperative kernel (256) and the level-by-level launches (0), and
    the content stays the oracle's."""
    vx.set_tuning("edit.small_max_prims", small_max_prims)
    try:
        depth = 5
        world = 4 << depth
        rng = np.random.default_rng(44)

        def sphere(c):
            p = np.zeros(1, oracle.PRIM_DTYPE)
            p[0] = (c, (20, 0, 0), 0, 0)  # remove a sphere of radius 20
            return p

        fill = np.zeros(1, oracle.PRIM_DTYPE)
        fill[0] = ((0, 0, 0), (world, world, world), 4 | (1 << 8) | (1 << 16), 0)  # whole world
        probe = vx.Svo(depth, 1 << 16, 1 << 16)
        probe.apply_primitives(vx.prims_to_device(fill, cuda))
        probe.apply_primitives(vx.prims_to_device(sphere((64, 64, 64)), cuda))
        assert probe.status() == 0
        used = probe.counters()
        s = vx.Svo(depth, 10 * used.node_count, 10 * used.leaf_count)
        g = oracle.Grid(depth)
        for i in range(40):
            c = tuple(int(v) for v in rng.integers(24, world - 24, 3))
            for prims in (fill, sphere(c)):
                s.apply_primitives(vx.prims_to_device(prims, cuda))
                g.apply_prims(prims)
                assert s.status() == 0, i
            assert canon(s) == g.svo()
        c = s.counters()
        s.collect()
        c = s.counters()
        nodes, leaves, _ = s.canonical()
        assert c.node_count - c.free_node_count == nodes.size // 8
        assert c.leaf_count - c.free_leaf_count == leaves.size
    finally:
        vx.reset_tuning()


def test_config_c1_full_size_plain_and_batched_bit_exact(cuda):
    """Configuration C1 at full size: 256^3 heightfield (materials by height
    band), 1,000 spheres r in [2, 16] applied in order through the plain
    per-call path (one voxel list and op per sphere) and through one batched
    call; both canonical dumps (nodes, leaves, materials) equal the oracle's
    sequential application."""
    depth = 6
    prims = vx.config_c1_edits(1000, seed=1)
    t = oracle.terrain(seed=1, scale=1, caves=False)
    g = oracle.Grid(depth, materials=True).terrain(t).apply_prims(prims)
    expect = g.svo()

    plain = vx.Svo(depth, 1 << 18, 1 << 18, materials=True, arena_bytes=64 << 20)
    plain.build_terrain(1, 1, False)
    assert plain.status() == 0
    dev_prims = vx.prims_to_device(prims, cuda)
    vox, off = vx.rasterize(dev_prims, depth + 2)
    off = off.cpu().numpy()
    for i, p in enumerate(prims):
        op = (int(p["flags"]) >> 8) & 0xFF
        mat = (int(p["flags"]) >> 16) & 0xFF
        assert plain.apply_voxels(vox[off[i]:off[i + 1]].contiguous(), op, mat) == 0
    assert canon(plain) == expect

    batched = vx.Svo(depth, 1 << 18, 1 << 18, materials=True, arena_bytes=64 << 20)
    batched.build_terrain(1, 1, False)
    batched.apply_primitives(dev_prims)
    assert batched.status() == 0
    assert canon(batched) == expect
