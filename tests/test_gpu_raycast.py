"""vx_dag_raycast on the GPU against the oracle's ray cast over the same
world (sequential application on the sparse CPU DAG): every hit identical,
bit for bit (voxel, face and the float ray parameter)."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def rays_for(rng, n, world, surface_z):
    r = np.zeros(n, vx.RAY_DTYPE)
    kind = rng.integers(0, 3, n)
    o = rng.uniform(0, world, (n, 3))
    o[kind == 1, 2] = surface_z + rng.uniform(0, world / 8, (kind == 1).sum())   # above ground
    o[kind == 2] = rng.uniform(-world / 2, 1.5 * world, ((kind == 2).sum(), 3))  # often outside
    d = rng.normal(size=(n, 3))
    d[kind == 1, 2] = -np.abs(d[kind == 1, 2]) - 0.2                           # looking down
    d[::13, rng.integers(0, 3)] = 0.0
    d[::17] = np.eye(3)[rng.integers(0, 3)] * rng.choice([-1.0, 1.0])
    r["origin"] = o
    r["dir"] = d
    r["t_max"] = np.where(rng.random(n) < 0.15, rng.uniform(0, world / 4, n), 3.0e38)
    return r


@pytest.mark.parametrize("depth,scale,n_prims", [(6, 1, 300), (10, 16, 2000)])
def test_raycast_matches_oracle(cuda, depth, scale, n_prims):
    world = 4 << depth
    prims = vx.config_c4_edits(n_prims, seed=11, world_exp=depth + 2)
    prims["r"] = np.minimum(prims["r"], world // 8)
    dag = vx.HashDag(depth, 1 << 22, 1 << 30)
    dag.build_terrain(5, scale, True)
    dag.apply_primitives(vx.prims_to_device(prims, cuda))
    assert dag.status() == 0
    rng = np.random.default_rng(depth)
    rays = rays_for(rng, 60_000, world, 128 * scale)
    got = dag.raycast(torch.from_numpy(rays.view(np.uint8)).to(cuda)).cpu().numpy()
    got = got.view(np.uint32).reshape(-1, 5)
    want = oracle.Sparse(depth, oracle.terrain(5, scale, True), prims).raycast(rays)
    assert np.array_equal(got, want)
    hit = want[:, 3] != 6
    assert 0.1 < hit.mean() < 0.99
    assert len(set(want[hit, 3].tolist())) == 6  # every face occurs


def test_raycast_empty_and_full_worlds(cuda):
    dag = vx.HashDag(3, 1 << 16, 32 << 20)
    r = np.zeros(3, vx.RAY_DTYPE)
    r["origin"] = [(-5, 3.5, 4.25), (10, 10, 10), (40, 40, 40)]
    r["dir"] = [(1, 0, 0), (0, 0, -1), (1, 1, 1)]
    r["t_max"] = 1e30
    out = lambda: dag.raycast(torch.from_numpy(r.view(np.uint8)).to(cuda)).cpu().numpy().view(
        np.uint32).reshape(-1, 5)
    h = out()
    assert (h[:, 3] == 6).all() and (h[:, :3] == 0xFFFFFFFF).all()
    box = np.zeros(1, vx.PRIM_DTYPE)
    box[0] = ((0, 0, 0), (32, 32, 32), 4 | (1 << 8), 0)  # fill the whole 32^3 world
    dag.apply_primitives(vx.prims_to_device(box, cuda))
    h = out()
    assert h[0, :4].tolist() == [0, 3, 4, 1]          # entered through X- at x = 0
    assert np.array([h[0, 4]], np.uint32).view(np.float32)[0] == np.float32(5.0)
    assert h[1, :4].tolist() == [10, 10, 10, 0] and h[1, 4] == 0  # starts inside
    assert h[2, 3] == 6                               # points away from the world
