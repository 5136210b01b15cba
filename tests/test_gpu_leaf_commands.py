"""The voxel engine's leaf edit commands (LeafEditCommand, voxel-engine/engine/
voxel/src/voxel/command.rs:8-52) through vx_dag_apply_leaf_commands /
vx_svo_apply_leaf_commands: masks of one leaf are OR-merged, then placed
(OrPolicy) or cleared (AndNotPolicy), against the oracle's per-voxel
application of the same bits."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def commands(rng, n, leaves_per_axis):
    c = np.zeros(n, vx.LEAF_COMMAND_DTYPE)
    xyz = rng.integers(0, leaves_per_axis, (n, 3))
    xyz[n // 2:] = xyz[rng.integers(0, n // 2, n - n // 2)]  # repeated leaves merge
    xyz[::53, 1] = leaves_per_axis + 3                     # outside the world: ignored
    c["leaf_x"], c["leaf_y"], c["leaf_z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    m = rng.integers(0, 2**64, n, dtype=np.uint64) & rng.integers(0, 2**64, n, dtype=np.uint64)
    c["voxel_data_low"] = (m & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    c["voxel_data_high"] = (m >> np.uint64(32)).astype(np.uint32)
    return c


def voxels_of(c, leaves_per_axis):
    """Every voxel a command's mask names (bit = x + 4y + 16z), in-world only."""
    out = []
    for r in c:
        if max(r["leaf_x"], r["leaf_y"], r["leaf_z"]) >= leaves_per_axis:
            continue
        m = int(r["voxel_data_low"]) | (int(r["voxel_data_high"]) << 32)
        for b in range(64):
            if (m >> b) & 1:
                out.append((4 * int(r["leaf_x"]) + (b & 3), 4 * int(r["leaf_y"]) + ((b >> 2) & 3),
                            4 * int(r["leaf_z"]) + (b >> 4)))
    return np.array(out, np.uint32).reshape(-1, 3)


def dev(c, cuda):
    return torch.from_numpy(c.view(np.uint8)).to(cuda)


def test_engine_merge_example(cuda):
    """command.rs merge_commands_preserves_high_bits: two commands on leaf
    (1, 2, 3) merge to low 0b0100, high 0b1010."""
    c = np.zeros(2, vx.LEAF_COMMAND_DTYPE)
    c[0] = (1, 2, 3, 0, 0b0010)
    c[1] = (1, 2, 3, 0b0100, 0b1000)
    dag = vx.HashDag(4, 1 << 16, 32 << 20)
    assert dag.apply_leaf_commands(dev(c, cuda), 1) == 0
    got = dag.read_leaves((1, 2, 3), (1, 1, 1)).cpu().numpy().view(np.uint64)
    assert int(got[0]) == 0b0100 | (0b1010 << 32)


@pytest.mark.parametrize("depth", [5, 8])
def test_dag_leaf_commands_match_oracle(cuda, depth):
    rng = np.random.default_rng(depth)
    leaves = 1 << depth
    t = oracle.terrain(seed=3, scale=1, caves=True)
    dag = vx.HashDag(depth, 1 << 20, 256 << 20)
    dag.build_terrain(3, 1, True)
    g = oracle.Grid(depth).terrain(t)
    for op in (1, 0, 1):
        c = commands(rng, 3000, leaves)
        assert dag.apply_leaf_commands(dev(c, cuda), op) == 0
        g.apply_voxels(voxels_of(c, leaves), op)
    assert oracle.DagCanon(*dag.canonical()) == g.dag()


def test_svo_leaf_commands_with_material_match_oracle(cuda):
    depth = 5
    rng = np.random.default_rng(9)
    leaves = 1 << depth
    svo = vx.Svo(depth, 1 << 16, 1 << 18, materials=True, arena_bytes=64 << 20)
    g = oracle.Grid(depth, materials=True)
    for op, mat in ((1, 7), (1, 200), (0, 0)):
        c = commands(rng, 1500, leaves)
        assert svo.apply_leaf_commands(dev(c, cuda), op, mat) == 0
        g.apply_voxels(voxels_of(c, leaves), op, mat)
    assert oracle.SvoCanon(*svo.canonical()) == g.svo()


def test_leaf_command_rejections(cuda):
    dag = vx.HashDag(4, 1 << 16, 32 << 20)
    lib = vx.lib()
    c = dev(np.zeros(4, vx.LEAF_COMMAND_DTYPE), cuda)
    ws = torch.empty(lib.vx_leaf_command_workspace_size(4), dtype=torch.uint8, device=cuda)
    h = dag._h
    assert lib.vx_dag_apply_leaf_commands(h, None, 4, 1, vx.ptr(ws), ws.numel(),
                                          vx.stream_handle()) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_leaf_commands(h, vx.ptr(c), 4, 2, vx.ptr(ws), ws.numel(),
                                          vx.stream_handle()) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_leaf_commands(h, vx.ptr(c), 4, 1, vx.ptr(ws), ws.numel() - 1,
                                          vx.stream_handle()) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_dag_apply_leaf_commands(h, None, 0, 1, None, 0, vx.stream_handle()) == 0
