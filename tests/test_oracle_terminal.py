"""The oracle's terminal-edit semantics against the known answers of the
reference's terminal-edit tests (test/cuda/terminal_edit/{place,destroy,
collapse,allocation_policy,release}_tests.cuh).  The reference world is
fixed at depth 10 (4096^3); the dense oracle grid restates each case in a
smaller world with the same cell sizes (a cell `k` levels above the leaves
stays `k` levels above them), which is the same voxel set."""
import numpy as np

import oracle
import voxel_b200 as vx

REF_DEPTH = 10


def grid(depth=7):
    return oracle.Grid(depth)


def rel(depth, ref_cell_depth):
    """The reference cell depth, restated in a world of `depth` levels."""
    return depth - (REF_DEPTH - ref_cell_depth)


def nodes(*rows):
    return vx.terminal_nodes(rows)


def leaves(*rows):
    return vx.terminal_leaves(rows)


def q(g, pts):
    return [g.get(*p) for p in pts]


def key(x, y, z, depth=7):
    return vx.cell_prefix(x, y, z, depth)


def test_place_leaf_bits():  # PlacesTerminalLeafIntoWorldSvt
    g = grid().apply_terminal(None, leaves((0, 0b11, 0, 0, 0)), 1)
    assert q(g, [(0, 0, 0), (1, 0, 0), (2, 0, 0)]) == [1, 1, 0]


def test_place_root():  # PlacesRootWithoutLeafExpansion
    g = oracle.Grid(5).apply_terminal(nodes((0, 0, 0, 0, 0)), None, 1)
    w = 4 << 5
    assert q(g, [(0, 0, 0), (w // 2,) * 3, (w - 1,) * 3]) == [1, 1, 1]
    assert g.count() == w ** 3


def test_ancestor_and_descendant():  # HandlesAncestorAndDescendant{Batch,Cells}
    D = 5
    w = 4 << D
    g = oracle.Grid(D).apply_terminal(nodes((0, 0, 0, 0, 0)), leaves((0, 1, 0, 0, 0)), 1)
    assert q(g, [(0, 0, 0), (w - 1,) * 3]) == [1, 1]
    g.apply_terminal(nodes((0, 0, 0, 0, 0)), leaves((0, 1, 0, 0, 0)), 0)
    assert q(g, [(0, 0, 0), (w - 1,) * 3]) == [0, 0] and g.count() == 0
    g = oracle.Grid(D).apply_terminal(nodes((0, 0, 0, 0, 0), (rel(D, 9), 0, 0, 0, 0)), None, 1)
    assert q(g, [(0, 0, 0), (w - 1,) * 3]) == [1, 1]


def test_place_and_destroy_leaf_cell():  # PlacesAndDestroysFullTerminalCell
    D = 7
    cell = nodes((rel(D, 10), 0, 0, 0, 0))
    g = grid(D).apply_terminal(cell, None, 1)
    assert q(g, [(0, 0, 0), (3, 3, 3), (4, 0, 0)]) == [1, 1, 0]
    g.apply_terminal(cell, None, 0)
    assert q(g, [(0, 0, 0), (3, 3, 3)]) == [0, 0]


def test_destroy_bit_in_uniform_leaf():  # AllocatesLeafWhenEditingUniformTerminalLeaf
    D = 7
    g = grid(D).apply_terminal(nodes((rel(D, 10), 0, 0, 0, 0)), None, 1)
    g.apply_terminal(None, leaves((0, 1, 0, 0, 0)), 0)
    assert q(g, [(0, 0, 0), (1, 0, 0)]) == [0, 1]


def test_refine_cell_with_leaf():  # RefinesExistingTerminalNodeWithLeafEdit
    D = 7
    g = grid(D).apply_terminal(nodes((rel(D, 9), 0, 0, 0, 0)), None, 1)
    g.apply_terminal(None, leaves((0, 1, 0, 0, 0)), 0)
    assert q(g, [(0, 0, 0), (1, 0, 0), (7, 7, 7), (8, 0, 0)]) == [0, 1, 1, 0]


def test_three_leaf_siblings():  # PlacesThreeLeafSiblingsSharingNewParent
    D = 7
    g = grid(D).apply_terminal(None, leaves((key(0, 0, 0), 0b1, 0, 0, 0),
                                            (key(1, 0, 0), 0b10, 0, 0, 0),
                                            (key(2, 0, 0), 0b100, 0, 0, 0)), 1)
    assert q(g, [(0, 0, 0), (5, 0, 0), (10, 0, 0), (11, 0, 0)]) == [1, 1, 1, 0]


def test_cells_overwriting_subtrees():  # release_tests.cuh queries
    D = 7
    g = grid(D).apply_terminal(None, leaves((0, 1, 0, 0, 0)), 1)
    g.apply_terminal(nodes((rel(D, 9), 0, 0, 0, 0)), None, 1)
    assert q(g, [(0, 0, 0), (7, 7, 7), (8, 0, 0)]) == [1, 1, 0]
    g = grid(D).apply_terminal(nodes((rel(D, 9), 0, 0, 0, 0)), None, 1)
    g.apply_terminal(nodes((rel(D, 8), 0, 0, 0, 0)), None, 1)
    assert q(g, [(0, 0, 0), (15, 15, 15), (16, 0, 0)]) == [1, 1, 0]
    g = grid(D).apply_terminal(None, leaves((key(0, 0, 0), 1, 0, 0, 0),
                                            (key(16, 0, 0), 1, 0, 0, 0)), 1)
    g.apply_terminal(nodes((rel(D, 5), 0, 0, 0, 0)), None, 1)
    assert q(g, [(0, 0, 0), (64, 0, 0), (127, 127, 127), (128, 0, 0)]) == [1, 1, 1, 0]


def test_offsets_move_and_clip():
    """World offsets move inputs by voxels and the world clips them
    (common.cuh terminal_box_device / intersect_world_leaves_device,
    count_requests.cuh count_terminal_leaf_requests_device)."""
    D = 4
    w = 4 << D
    g = oracle.Grid(D).apply_terminal(nodes((D - 1, 0, 3, -2, w - 4)), None, 1)
    cell = 8
    xs, ys, zs = range(3, 3 + cell), range(0, cell - 2), range(w - 4, w)
    assert g.count() == len(xs) * len(ys) * len(zs)
    assert g.get(3, 0, w - 4) == 1 and g.get(2, 0, w - 4) == 0
    # a brick moved across a leaf corner lands in up to 8 leaves
    g = oracle.Grid(D).apply_terminal(None, leaves((0, ~0 & (2**64 - 1), 2, 3, 1)), 1)
    assert g.count() == 64
    assert g.get(2, 3, 1) == 1 and g.get(5, 6, 4) == 1 and g.get(6, 6, 4) == 0
    # bits moved outside the world are dropped
    g = oracle.Grid(D).apply_terminal(None, leaves((0, 2**64 - 1, -2, 0, 0)), 1)
    assert g.count() == 2 * 16


def test_invalid_inputs_are_ignored():
    D = 4
    g = oracle.Grid(D).apply_terminal(nodes((D + 1, 0, 0, 0, 0), (1, 8, 0, 0, 0)),
                                      leaves((1 << (3 * D), 1, 0, 0, 0)), 1)
    assert g.count() == 0
