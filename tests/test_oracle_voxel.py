"""Pin the voxel oracle against the reference's own CPU implementations
(algorithm/lib/include/algo/svt/hash_dag.hpp and svo.hpp, compiled from the
reference headers into oracle/_ref by oracle/build.py): canonical Hash DAG and
SVO dumps must be identical after the same edit sequences."""
import numpy as np
import pytest

import oracle
import voxel_b200 as vx

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference shim not built (no reference tree)")


def rand_prims(rng, n, world, rmax, sphere_frac=0.6):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = 0 if rng.random() < sphere_frac else 1
        op = int(rng.random() < 0.55)
        r = rng.integers(0, rmax + 1, 3)
        p[i] = (rng.integers(-2, world + 2, 3), (r[0], r[1] if shape else 0, r[2] if shape else 0),
                shape | (op << 8) | (int(rng.integers(1, 256)) << 16 if op else 0), 0)
    return p


@needs_ref
@pytest.mark.parametrize("depth,n,seed", [(1, 6, 0), (2, 20, 1), (3, 40, 2), (4, 60, 3)])
def test_oracle_dag_matches_reference_hashdag(depth, n, seed):
    rng = np.random.default_rng(seed)
    world = 4 << depth
    prims = rand_prims(rng, n, world, max(2, world // 4))
    ref = oracle.RefDag(depth)
    for p in prims:
        ref.apply_prim_runs(p)
    g = oracle.Grid(depth).apply_prims(prims)
    assert g.dag() == ref.canon()
    # voxel-level agreement too
    for _ in range(200):
        x, y, z = rng.integers(0, world, 3)
        assert ref.get_voxel(x, y, z) == g.get(x, y, z)


@needs_ref
def test_oracle_dag_reference_known_cases():
    """Cases from test/svt/test_svt_hash_dag.cpp and
    test/cuda/test_cuda_hash_dag_gpu.cu, checked against the reference."""
    depth = 8
    # make_spread_edits (test_cuda_hash_dag_gpu.cu:142-156), batch 257, with
    # the out-of-world x = 1024 + i edits that the GPU path ignores
    edits = []
    for i in range(257):
        if i % 19 == 0:
            edits.append((1024 + i, 0, 0))
        else:
            edits.append(((i * 37) & 1023, (i * 91 + 3) & 1023, (i * 53 + 7) & 1023))
    ref = oracle.RefDag(depth)
    for e in edits:
        if max(e) < (4 << depth):
            ref.set_voxel(*e, True)
    g = oracle.Grid(depth).apply_voxels(np.array(edits), 1)
    assert g.dag() == ref.canon()
    # destroy half of them again
    for e in edits[::2]:
        if max(e) < (4 << depth):
            ref.set_voxel(*e, False)
    g.apply_voxels(np.array(edits[::2]), 0)
    assert g.dag() == ref.canon()


@needs_ref
def test_oracle_dag_full_volume_and_undo():
    """Filling the whole world uses the reserved full states; undoing an edit
    restores the root (test_svt_hash_dag.cpp:60-96)."""
    depth = 3
    world = 4 << depth
    ref = oracle.RefDag(depth)
    ref.box((0, 0, 0), (world,) * 3, True)
    g = oracle.Grid(depth)
    g.apply_voxels(np.array([(x, y, z) for x in range(world) for y in range(world)
                             for z in range(world)]), 1)
    assert g.dag() == ref.canon() and g.dag().root == 1
    before = ref.canon()
    ref.box((3, 4, 5), (9, 10, 11), False)
    ref.box((3, 4, 5), (9, 10, 11), True)
    assert ref.canon() == before


@needs_ref
@pytest.mark.parametrize("depth", [3, 4])
def test_oracle_terrain_matches_reference_columns(depth):
    world = 4 << depth
    t = oracle.terrain(seed=1, scale=1, caves=True)
    g = oracle.Grid(depth).terrain(t)
    ref = oracle.RefDag(depth)
    for x in range(world):
        for y in range(world):
            z = 0
            while z < world:
                if g.get(x, y, z):
                    z1 = z
                    while z1 < world and g.get(x, y, z1):
                        z1 += 1
                    ref.box((x, y, z), (x + 1, y + 1, z1), True)
                    z = z1
                else:
                    z += 1
    assert g.dag() == ref.canon()
    # the grid agrees with the terrain definition voxel by voxel
    pts = np.random.default_rng(0).integers(0, world, (500, 3)).astype(np.uint32)
    direct = oracle.eval_voxels(t, depth + 2, np.zeros(0, oracle.PRIM_DTYPE), pts)
    assert [g.get(*p) for p in pts] == direct.tolist()


@needs_ref
@pytest.mark.parametrize("depth,n,seed", [(1, 200, 0), (2, 500, 1), (3, 3000, 2), (4, 6000, 3)])
def test_oracle_svo_matches_reference_svo(depth, n, seed):
    rng = np.random.default_rng(seed)
    world = 4 << depth
    ref = oracle.RefSvo(depth)
    g = oracle.Grid(depth)
    # clustered edits so leaves fill up and collapse
    for _ in range(n):
        x, y, z = (rng.integers(0, world // 2, 3) if rng.random() < 0.7
                   else rng.integers(0, world, 3))
        v = bool(rng.random() < 0.7)
        ref.set_voxel(int(x), int(y), int(z), v)
        g.apply_voxels(np.array([[x, y, z]]), int(v))
    assert g.svo() == ref.canon()


@needs_ref
def test_oracle_svo_spheres_match_reference():
    depth = 6  # 256^3, the reference's SVO(6) of the plain SVO configuration
    prims = vx.config_c1_edits(40, seed=1)
    ref = oracle.RefSvo(depth)
    g = oracle.Grid(depth).apply_prims(prims)
    for p in prims:
        c = [int(v) for v in p["c"]]
        r = int(p["r"][0])
        add = ((int(p["flags"]) >> 8) & 0xFF) == 1
        for z in range(max(0, c[2] - r), min(256, c[2] + r + 1)):
            for y in range(max(0, c[1] - r), min(256, c[1] + r + 1)):
                for x in range(max(0, c[0] - r), min(256, c[0] + r + 1)):
                    if (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r:
                        ref.set_voxel(x, y, z, add)
    assert g.svo() == ref.canon()


def test_eval_voxels_matches_grid():
    rng = np.random.default_rng(9)
    depth = 4
    world = 4 << depth
    t = oracle.terrain(seed=3, scale=1, caves=True)
    prims = rand_prims(rng, 30, world, 12)
    g = oracle.Grid(depth).terrain(t).apply_prims(prims)
    pts = rng.integers(0, world, (2000, 3)).astype(np.uint32)
    direct = oracle.eval_voxels(t, depth + 2, prims, pts)
    assert [g.get(*p) for p in pts] == direct.tolist()
