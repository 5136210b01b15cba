"""Terminal edits (place_/destroy_terminal_edits) on the GPU SVO and Hash DAG:
the reference's own terminal-edit test cases at its depth 10 (query answers,
live node / leaf counts and free-list deltas), random cells and bricks with
offsets against the oracle's canonical dumps, and argument validation."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu

D = 10  # the reference GPU SVO's fixed depth (svt/cuda/config.cuh:17-31)


def dev(records):
    return vx.records_to_device(records, "cuda") if records is not None and len(records) else None


def place(s, nodes=None, leaves=None, op=1):
    n = vx.terminal_nodes(nodes) if nodes else None
    lv = vx.terminal_leaves(leaves) if leaves else None
    st = s.apply_terminal(dev(n), dev(lv), op)
    assert st == 0


def destroy(s, nodes=None, leaves=None):
    place(s, nodes, leaves, op=0)


def query(s, pts):
    return s.query(vx.voxels_to_device(np.array(pts, np.uint32), "cuda")).cpu().tolist()


def svo():
    # TestGpuSvo = GpuSvo<256, 64> (terminal_edit/cuda_terminal_edit_test_utils.cuh)
    return vx.Svo(D, 256, 64, arena_bytes=32 << 20)


def counters(s):
    """Counters after a collection: the reference frees a replaced subtree
    within the edit; this library collects lazily (when an edit would not fit
    otherwise, or on request), so free-list deltas are read after one."""
    s.collect()
    return s.counters()


def live(s):
    c = counters(s)
    return c.node_count - c.free_node_count, c.leaf_count - c.free_leaf_count


def key(x, y, z):
    return vx.cell_prefix(x, y, z, D)


def test_reference_place_cases(cuda):
    s = svo()
    place(s, leaves=[(0, 0b11, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (1, 0, 0), (2, 0, 0)]) == [1, 1, 0]
    s = svo()
    place(s, nodes=[(0, 0, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (2048, 2048, 2048), (4095, 4095, 4095)]) == [1, 1, 1]
    s = svo()
    place(s, nodes=[(0, 0, 0, 0, 0)], leaves=[(0, 1, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (4095, 4095, 4095)]) == [1, 1]
    s = svo()
    place(s, nodes=[(0, 0, 0, 0, 0), (9, 0, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (4095, 4095, 4095)]) == [1, 1]
    # LeavesExpectedSvoShapeAfterLeafAllocation
    s = svo()
    place(s, leaves=[(0, 1, 0, 0, 0)])
    assert live(s) == (D, 1)


def test_reference_destroy_and_collapse_cases(cuda):
    s = svo()
    place(s, nodes=[(10, 0, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (3, 3, 3), (4, 0, 0)]) == [1, 1, 0]
    assert live(s)[1] == 0  # CollapsesFullTerminalLeaf
    destroy(s, nodes=[(10, 0, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (3, 3, 3)]) == [0, 0]
    s = svo()
    place(s, nodes=[(0, 0, 0, 0, 0)], leaves=[(0, 1, 0, 0, 0)])
    destroy(s, nodes=[(0, 0, 0, 0, 0)], leaves=[(0, 1, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (4095, 4095, 4095)]) == [0, 0]
    s = svo()
    place(s, nodes=[(0, 0, 0, 0, 0), (9, 0, 0, 0, 0)])
    destroy(s, nodes=[(0, 0, 0, 0, 0), (9, 0, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (4095, 4095, 4095)]) == [0, 0]
    # AllocatesLeafWhenEditingUniformTerminalLeaf
    s = svo()
    place(s, nodes=[(10, 0, 0, 0, 0)])
    before = counters(s)
    assert before.free_leaf_count == 0
    destroy(s, leaves=[(0, 1, 0, 0, 0)])
    after = counters(s)
    assert after.leaf_count == before.leaf_count + 1 and after.free_leaf_count == 0
    assert query(s, [(0, 0, 0), (1, 0, 0)]) == [0, 1]


def test_reference_allocation_cases(cuda):
    s = svo()
    place(s, leaves=[(key(0, 0, 0), 0b1, 0, 0, 0), (key(512, 0, 0), 0b10, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (1, 0, 0), (2049, 0, 0), (2048, 0, 0)]) == [1, 0, 1, 0]
    s = svo()
    place(s, nodes=[(9, 0, 0, 0, 0)])
    destroy(s, leaves=[(0, 0b1, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (1, 0, 0), (7, 7, 7), (8, 0, 0)]) == [0, 1, 1, 0]
    s = svo()
    place(s, leaves=[(key(0, 0, 0), 0b1, 0, 0, 0), (key(1, 0, 0), 0b10, 0, 0, 0),
                     (key(2, 0, 0), 0b100, 0, 0, 0)])
    assert query(s, [(0, 0, 0), (5, 0, 0), (10, 0, 0), (11, 0, 0)]) == [1, 1, 1, 0]


def test_reference_release_cases(cuda):
    """Free-list deltas of release_tests.cuh: a cell overwriting a
    materialised subtree frees exactly its nodes and leaves."""
    s = svo()
    place(s, leaves=[(0, 1, 0, 0, 0)])
    b = counters(s)
    assert b.free_leaf_count == 0 and b.free_node_count == 0
    place(s, nodes=[(9, 0, 0, 0, 0)])
    a = counters(s)
    assert (a.free_leaf_count - b.free_leaf_count, a.free_node_count - b.free_node_count) == (1, 1)
    assert query(s, [(0, 0, 0), (7, 7, 7), (8, 0, 0)]) == [1, 1, 0]

    s = svo()
    place(s, nodes=[(9, 0, 0, 0, 0)])
    b = counters(s)
    place(s, nodes=[(8, 0, 0, 0, 0)])
    a = counters(s)
    assert (a.free_leaf_count - b.free_leaf_count, a.free_node_count - b.free_node_count) == (0, 1)
    assert query(s, [(0, 0, 0), (15, 15, 15), (16, 0, 0)]) == [1, 1, 0]

    s = svo()
    place(s, leaves=[(key(0, 0, 0), 1, 0, 0, 0), (key(16, 0, 0), 1, 0, 0, 0)])
    b = counters(s)
    assert b.free_leaf_count == 0 and b.free_node_count == 0
    place(s, nodes=[(5, 0, 0, 0, 0)])
    a = counters(s)
    assert (a.free_leaf_count - b.free_leaf_count, a.free_node_count - b.free_node_count) == (2, 9)
    assert query(s, [(0, 0, 0), (64, 0, 0), (127, 127, 127), (128, 0, 0)]) == [1, 1, 1, 0]


def rand_terminal(rng, depth, n_nodes, n_leaves):
    world = 4 << depth
    rows_n = []
    for _ in range(n_nodes):
        d = int(rng.integers(0, depth + 2))  # depth + 1 is invalid
        dd = min(d, depth)
        c = rng.integers(0, 1 << dd, 3)
        p = vx.cell_prefix(int(c[0]), int(c[1]), int(c[2]), dd)
        if rng.random() < 0.05 and dd < 10:
            p |= 1 << (3 * dd)  # invalid prefix
        off = rng.integers(-world // 4, world // 4, 3) if rng.random() < 0.5 else (0, 0, 0)
        rows_n.append((d, p, int(off[0]), int(off[1]), int(off[2])))
    rows_l = []
    for _ in range(n_leaves):
        c = rng.integers(0, 1 << depth, 3)
        m = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        if rng.random() < 0.1:
            m = 0
        off = rng.integers(-9, 10, 3) if rng.random() < 0.6 else (0, 0, 0)
        rows_l.append((vx.cell_prefix(int(c[0]), int(c[1]), int(c[2]), depth), m,
                       int(off[0]), int(off[1]), int(off[2])))
    return vx.terminal_nodes(rows_n), vx.terminal_leaves(rows_l)


@pytest.mark.parametrize("depth,seed,mats", [(3, 0, False), (5, 1, False), (6, 2, True),
                                             (6, 3, False)])
def test_random_terminal_edits_match_oracle(cuda, depth, seed, mats):
    rng = np.random.default_rng(seed)
    t = oracle.terrain(seed=3, scale=1, caves=True)
    s = vx.Svo(depth, 1 << 18, 1 << 18, materials=mats, arena_bytes=64 << 20)
    s.build_terrain(3, 1, True)
    dag = vx.HashDag(depth, 1 << 18, 64 << 20)
    dag.build_terrain(3, 1, True)
    g = oracle.Grid(depth, materials=mats).terrain(t)
    occ = oracle.Grid(depth).terrain(t)
    for step in range(4):
        nodes, leaves = rand_terminal(rng, depth, int(rng.integers(0, 12)),
                                      int(rng.integers(0, 40)))
        op = step % 2 if step < 3 else 1
        mat = int(rng.integers(1, 256)) if mats else 1
        assert s.apply_terminal(dev(nodes), dev(leaves), op, material=mat) == 0
        assert dag.apply_terminal(dev(nodes), dev(leaves), op) == 0
        g.apply_terminal(nodes, leaves, op, mat)
        occ.apply_terminal(nodes, leaves, op)
        assert oracle.SvoCanon(*s.canonical()) == g.svo()
        assert oracle.DagCanon(*dag.canonical()) == occ.dag()


def test_validation(cuda):
    s = svo()
    lib = vx.lib()
    ws = torch.empty(vx.lib().vx_terminal_workspace_size(1, 1), dtype=torch.uint8,
                     device=cuda)
    # EmptyApplyStillValidatesWorkspace: no inputs, no workspace
    assert lib.vx_svo_apply_terminal(s._h, None, 0, None, 0, 1, 1, None, 0,
                                     vx.stream_handle()) == 1
    assert lib.vx_svo_apply_terminal(s._h, None, 0, None, 0, 1, 1, vx.ptr(ws), ws.numel(),
                                     vx.stream_handle()) == 0
    # null inputs with a count, short workspace
    assert lib.vx_svo_apply_terminal(s._h, None, 1, None, 0, 1, 1, vx.ptr(ws), ws.numel(),
                                     vx.stream_handle()) == 1
    n = dev(vx.terminal_nodes([(0, 0, 0, 0, 0)]))
    assert lib.vx_svo_apply_terminal(s._h, vx.ptr(n), 1, None, 0, 1, 1, vx.ptr(ws), 100,
                                     vx.stream_handle()) == 1
    # prefixes are 32-bit: structures deeper than 10 are rejected
    deep = vx.HashDag(11, 1 << 16, 32 << 20)
    assert deep.apply_terminal(n, None, 1) == 1
    assert query(s, [(0, 0, 0)]) == [0]


def rand_aabb_mix(rng, n, world):
    p = np.zeros(n, oracle.PRIM_DTYPE)
    for i in range(n):
        shape = int(rng.choice([0, 1, 4]))
        op = int(rng.random() < 0.6)
        if shape == 4:
            c = rng.integers(-world // 4, world, 3)
            r = rng.integers(0, world // 2, 3)
        else:
            c = rng.integers(-3, world + 3, 3)
            r = rng.integers(0, world // 5 + 2, 3)
            if shape == 0:
                r[1:] = 0
        p[i] = (c, r, shape | (op << 8) | ((1 if op else 0) << 16), 0)
    return p


@pytest.mark.parametrize("depth,seed", [(4, 0), (6, 1)])
def test_aabb_primitives_match_oracle(cuda, depth, seed):
    """Half-open boxes (the shape terminal cells become) mixed with spheres
    and boxes in one batch, on both structures; rasterised counts too."""
    rng = np.random.default_rng(seed)
    world = 4 << depth
    prims = rand_aabb_mix(rng, 150, world)
    g = oracle.Grid(depth).apply_prims(prims)
    d = vx.HashDag(depth, 1 << 18, 64 << 20)
    d.apply_primitives(vx.prims_to_device(prims, cuda))
    assert d.status() == 0
    assert oracle.DagCanon(*d.canonical()) == g.dag()
    s = vx.Svo(depth, 1 << 18, 1 << 18, arena_bytes=64 << 20)
    s.apply_primitives(vx.prims_to_device(prims, cuda))
    assert s.status() == 0
    assert oracle.SvoCanon(*s.canonical()) == g.svo()
    adds = prims[(prims["flags"] & 0xff) == 4].copy()
    adds["flags"] = 4 | (1 << 8) | (1 << 16)
    vox, offsets = vx.rasterize(vx.prims_to_device(adds, cuda), depth + 2)
    counts = np.diff(offsets.cpu().numpy())
    for i, p in enumerate(adds):
        one = oracle.Grid(depth).apply_prims(np.array([p], oracle.PRIM_DTYPE))
        assert counts[i] == one.count()
