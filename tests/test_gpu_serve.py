"""Serving loop: continuous batching over a resident Hash DAG.  The final DAG
must equal sequential application of the requests in arrival order, and every
request's result must be the same whether it runs alone (one request per
launch) or coalesced with others (compared at every root a batch publishes)."""
import numpy as np
import pytest

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu

DEPTH = 6


def stream(n_seconds=0.2, rate=1500.0, seed=3, max_size=48, r_max=12):
    return vx.generate_requests(DEPTH + 2, rate, n_seconds, seed, max_size=max_size,
                                r_max=r_max)


def fresh_dag():
    dag = vx.HashDag(DEPTH, max_nodes=1 << 20, arena_bytes=64 << 20)
    dag.build_terrain(5, 1, True)
    assert dag.status() == 0
    return dag


def run(dag, arr, sizes, prims, **cfg):
    srv = vx.Server(dag, **cfg)
    off = 0
    t0 = srv.now_ns()
    for i, (a, k) in enumerate(zip(arr, sizes)):
        srv.submit(i, prims[off:off + k], t0 + int(a))
        off += k
    srv.drain()
    done = srv.poll(1 << 20)
    stats = srv.stats()
    srv.close()
    return done, stats


def canon(dag, root=0xFFFFFFFF):
    return oracle.DagCanon(*dag.canonical(root))


def test_served_final_state_is_sequential_application(cuda):
    arr, sizes, prims = stream()
    assert len(arr) > 100
    dag = fresh_dag()
    done, stats = run(dag, arr, sizes, prims)
    assert len(done) == len(arr) and (done["status"] == 0).all()
    assert sorted(done["request_id"].tolist()) == list(range(len(arr)))
    # commits follow arrival order
    order = np.argsort(done["request_id"])
    assert (np.diff(done["commit_ns"][order].astype(np.int64)) >= 0).all()
    assert stats.batches < len(arr)  # requests were coalesced
    t = oracle.terrain(5, 1, True)
    expect = oracle.Grid(DEPTH).terrain(t).apply_prims(prims).dag()
    assert canon(dag) == expect


def test_each_result_same_alone_and_in_the_mix(cuda):
    arr, sizes, prims = stream(seed=9)
    alone = fresh_dag()
    d_alone, s_alone = run(alone, arr, sizes, prims, max_batch_requests=1,
                           compact_at_fill=1e9)
    assert s_alone.batches == len(arr)
    mixed = fresh_dag()
    d_mix, s_mix = run(mixed, arr, sizes, prims, compact_at_fill=1e9)
    assert s_mix.batches < len(arr)
    root_alone = dict(zip(d_alone["request_id"].tolist(), d_alone["root"].tolist()))
    # A batch is a run of consecutive requests completed together (same
    # commit time and root); two batches may publish the same root when the
    # later one changes nothing.  The last request of each mixed batch must
    # see the same content as right after it ran alone.
    order = np.argsort(d_mix["request_id"])
    rids = d_mix["request_id"][order].tolist()
    roots = d_mix["root"][order].tolist()
    commits = d_mix["commit_ns"][order].tolist()
    checked = 0
    for i, rid in enumerate(rids):
        if i + 1 < len(rids) and (roots[i + 1], commits[i + 1]) == (roots[i], commits[i]):
            continue
        assert canon(mixed, roots[i]) == canon(alone, root_alone[rid])
        checked += 1
    assert checked == s_mix.batches


def test_serving_with_compaction_between_batches(cuda):
    arr, sizes, prims = stream(seed=17)
    dag = fresh_dag()
    done, stats = run(dag, arr, sizes, prims, compact_at_fill=1e-6, max_batch_prims=200)
    assert (done["status"] == 0).all()
    assert stats.compactions > 0
    t = oracle.terrain(5, 1, True)
    assert canon(dag) == oracle.Grid(DEPTH).terrain(t).apply_prims(prims).dag()


def test_graph_and_direct_launches_agree(cuda):
    """The per-slot CUDA graphs and the kernel-by-kernel launches serve the
    same stream to the same final DAG."""
    arr, sizes, prims = stream(seed=23)
    a = fresh_dag()
    run(a, arr, sizes, prims, graphs=True)
    b = fresh_dag()
    run(b, arr, sizes, prims, graphs=False)
    assert canon(a) == canon(b)


def test_admission_by_need_compacts_before_the_tables_fill(cuda):
    """A small DAG (32 Ki nodes per table) under a stream that creates far
    more nodes than that: admission by each request's estimated need compacts
    before a batch can overflow, so no batch fails and is recovered, and the
    final state is still sequential application."""
    arr, sizes, prims = stream(n_seconds=0.3, seed=29)
    dag = vx.HashDag(DEPTH, max_nodes=1 << 15, arena_bytes=64 << 20)
    dag.build_terrain(5, 1, True)
    assert dag.status() == 0
    done, stats = run(dag, arr, sizes, prims)
    assert (done["status"] == 0).all()
    assert stats.compactions > 0
    assert stats.recoveries == 0
    t = oracle.terrain(5, 1, True)
    assert canon(dag) == oracle.Grid(DEPTH).terrain(t).apply_prims(prims).dag()
