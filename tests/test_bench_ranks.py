"""The benchmark's multi-rank host logic on CPU: two replicas as gloo ranks
(world size 2, loopback rendezvous).  Each rank times a different region;
every rank must see the slowest rank's time, and the whole-job rate counts
every replica's units over that time.  The reference arm runs on rank 0
only; the other ranks return without work."""
import datetime
import os
import socket
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, times: list, out):
    import sys
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup()
        job_ms = bench.max_over_ranks(times[rank], w, "cpu")
        rate = bench.job_rate(1000.0, w, job_ms)
        ref = bench.run_reference(None, w, r) if r != 0 else "rank0"
        out.put((r, local, w, job_ms, rate, ref))
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_as_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    times = [2.5, 4.0]  # rank 1 is the slower replica
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(out.get(timeout=10) for _ in range(2))
    for r, (rank, local, ws, job_ms, rate, ref) in enumerate(res):
        assert (rank, local, ws) == (r, r, 2)
        assert job_ms == pytest.approx(4.0)           # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 1000.0 / 4e-3)  # both replicas' units / slowest time
    assert res[1][5] is None  # the reference arm does no work off rank 0


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.0, 1, "cpu") == 3.0
    assert bench.job_rate(500.0, 1, 2.0) == pytest.approx(250_000.0)
