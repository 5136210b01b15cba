"""The oracle's ray cast (oracle_sparse.cpp raycast, the checker of
vx_dag_raycast) against the meaning of a ray hit, checked independently of
its stepping: the hit voxel is solid, the hit point lies on that voxel's
surface (on the face it names), and dense samples of the ray before the hit
meet no solid voxel; rays that report no hit meet none on [0, t_max]."""
import numpy as np

import oracle

DEPTH = 4
WORLD = 4 << DEPTH


def world_and_grid():
    t = oracle.terrain(seed=5, scale=1, caves=True)
    prims = oracle.generate_primitives(DEPTH + 2, 40, 3, sphere_permille=600, r_min=1, r_max=10,
                                       log_uniform=True)
    s = oracle.Sparse(DEPTH, t, prims, shard_levels=1, threads=2)
    g = oracle.Grid(DEPTH).terrain(t).apply_prims(prims)
    solid = np.zeros((WORLD,) * 3, bool)
    lo = (0, 0, 0)
    n = WORLD // 4
    masks = s.leaf_block(lo, (n, n, n))
    for i, m in enumerate(masks):
        lx, ly, lz = i % n, (i // n) % n, i // (n * n)
        for b in range(64):
            if (int(m) >> b) & 1:
                solid[4 * lx + (b & 3), 4 * ly + ((b >> 2) & 3), 4 * lz + (b >> 4)] = True
    # the leaf block is itself checked against the dense grid
    for _ in range(300):
        x, y, z = np.random.default_rng(_).integers(0, WORLD, 3)
        assert solid[x, y, z] == bool(g.get(int(x), int(y), int(z)))
    return s, solid


def random_rays(rng, n):
    r = np.zeros((n, 8), np.float32)
    inside = rng.random(n) < 0.5
    r[:, :3] = np.where(inside[:, None], rng.uniform(0, WORLD, (n, 3)),
                        rng.uniform(-WORLD, 2 * WORLD, (n, 3)))
    d = rng.normal(size=(n, 3))
    d[::7, rng.integers(0, 3)] = 0.0          # axis-parallel components
    d[::11] = np.eye(3)[rng.integers(0, 3)] * rng.choice([-1, 1])
    r[:, 3:6] = d
    r[:, 6] = np.where(rng.random(n) < 0.2, rng.uniform(0, 40, n), 1e9)
    return r


def test_oracle_raycast_meaning():
    s, solid = world_and_grid()
    rng = np.random.default_rng(7)
    rays = random_rays(rng, 3000)
    hits = s.raycast(rays)
    n_hit = 0
    for ray, h in zip(rays, hits):
        o, d, tmax = ray[:3].astype(np.float64), ray[3:6].astype(np.float64), float(ray[6])
        face = int(h[3])
        t_hit = float(np.array([h[4]], np.uint32).view(np.float32)[0])
        # interval of the ray inside the world
        t_in, t_out = 0.0, np.inf
        for a in range(3):
            if d[a] == 0:
                continue
            ta, tb = (0 - o[a]) / d[a], (WORLD - o[a]) / d[a]
            t_in, t_out = max(t_in, min(ta, tb)), min(t_out, max(ta, tb))
        end = min(t_out, tmax) if face == 6 else t_hit
        if face != 6:
            n_hit += 1
            v = h[:3].astype(np.int64)
            assert solid[tuple(v)]
            p = o + t_hit * d
            assert np.all(p >= v - 1e-2) and np.all(p <= v + 1 + 1e-2)
            if t_hit > 0:
                a, neg = face // 2, face % 2
                assert abs(p[a] - (v[a] if neg else v[a] + 1)) < 1e-2
        # samples strictly before `end` (away from voxel boundaries) are empty
        if end > t_in:
            ts = np.linspace(t_in, end, 400)[:-1]
            pts = o[None, :] + ts[:, None] * d[None, :]
            frac = pts - np.floor(pts)
            away = np.all((frac > 2e-3) & (frac < 1 - 2e-3), axis=1)
            inb = np.all((pts >= 0) & (pts < WORLD), axis=1)
            q = np.floor(pts[away & inb]).astype(np.int64)
            assert not solid[q[:, 0], q[:, 1], q[:, 2]].any()
    assert 500 < n_hit < 2900
