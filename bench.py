"""Benchmark of the B200 voxel-editing path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline (Hash DAG, batched): a 16384^3 Hash DAG (depth 12 inner levels, 4^3
leaves) built on the GPU from the cave terrain generator at scale 64, then one
batch of 16,384 sphere edits (radius log-uniform in [1, 256], 60 % add) applied
in one stream-ordered submission.  One step restores the terrain snapshot
(device copy, outside the timed events) and applies the batch; the value is
voxels edited (sum of the spheres' clipped voxel counts) per second of device
time.  The plain per-call path (one rasterised voxel list per sphere through
vx_dag_apply_voxels, the reference API shape) is timed on a prefix of the same
spheres for the batched/plain ratio.

Components (the primitives sweep): exclusive scan of 2^28 u32 in [0, 255];
stable radix sort of 2^28 u32 keys and of 2^28 u64 Morton keys (64 Gaussian
blobs, sigma 2^14, 2^20 cube) with u32 payload = index; slab set and cuckoo
map with 2^26 u64 keys at load factor 0.8 and 2^26 lookups at 50 % hits.
Every sweep step has its own input buffers, each larger than the 126 MB L2.

Multi-GPU: every rank runs the same work on its own GPU (independent
replicas, weak scaling); timed regions are bracketed by barriers and the
maximum over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("Hash DAG voxels edited/s batched vs plain (bit-exact); "
          "sort/scan GB/s; p99 ms")
N_SCAN = 1 << 28
N_SORT = 1 << 28
BYTES_SCAN = 8          # read 4 + write 4 per element
BYTES_SORT_U32 = 68     # 4 passes x (read 8 + write 8) + 4 histogram read
BYTES_SORT_U64 = 200    # 8 passes x (read 12 + write 12) + 8 histogram read
# Per-launch algorithmic bytes of the dominant kernel (one u64 partition
# pass: read key 8 + value 4, write key 8 + value 4 per element).
PART_U64_BYTES = N_SORT * 24
# DRAM bytes per sort_partition_u64 launch: an ncu capture of one 2^24-key
# pass (dram__bytes_read 202.8 MB + dram__bytes_write 158.7 MB) scaled by the
# keys of a launch here (2^28).  At 2^24 part of the input stays in L2, so
# this is a lower bound for the full size.
PART_U64_TRAFFIC = round((202.8e6 + 158.7e6) / (1 << 24) * N_SORT)
DAG_DEPTH = 12            # inner levels: world side 4 << 12 = 16384
DAG_SCALE = 64            # terrain generator scale (height 8192 + 2560 v)
DAG_SEED = 7
DAG_EDITS = 16384
DAG_MAX_NODES = 1 << 27
DAG_ARENA = 16 << 30
PLAIN_SAMPLE = 96         # spheres of the plain per-call sample (a prefix)
# DRAM bytes per dag_leafparent work item: an ncu capture of the small case
# (bench.py --case dag --elements 4096: dram__bytes_read 441.5 MB +
# dram__bytes_write 217.2 MB) divided by that launch's 5,280,796 items; the
# roofline's `traffic` scales it by the full launch's items.
LEAFPARENT_TRAFFIC_PER_ITEM = (441.5e6 + 217.2e6) / 5280796
SVO_C3_DEPTH = 10         # 4096^3
SVO_C3_EDITS = 65536
SERVE_DEPTH = 11          # 8192^3
SERVE_RATE = 2000.0       # requests per second (Poisson)
SERVE_SECONDS = 60.0
SERVE_MAX_NODES = 1 << 28   # per level; two such DAGs (served + check) ~ 100 GB
SERVE_ARENA = 16 << 30
C5_REGION_BASE = 5       # served-DAG check regions: cells of 256^3 at level 5
C5_REGIONS = 16
N_HASH = 1 << 26
HASH_LOAD = 0.8
BYTES_HASH_INSERT = 40  # read key 8 + one 32-B sector read-modify-write
BYTES_HASH_LOOKUP = 44  # read key 8 + one 32-B sector + 4-B result


# --------------------------------------------------------------- helpers --

def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.marks = {}
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}",
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.PIPE, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi needs a moment before its first sample.
            deadline = time.time() + 10
            while not self.rows and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.05)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def mark(self, name):
        self.marks[name] = time.time()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append((time.time(), parts))

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        """Median SM clock and active throttle reasons of the samples taken
        between mark('start') and mark('end') (all samples if none fell in
        that window)."""
        t0 = self.marks.get("start", 0.0) - 0.25
        t1 = self.marks.get("end", float("inf")) + 0.25
        rows = [r for t, r in self.rows if t0 <= t <= t1] or [r for _, r in self.rows]
        if not rows:
            err = self.proc.stderr.read() if self.proc is not None else "not started"
            return {"sm_mhz": None, "sm_max_mhz": None,
                    "reasons": ["unsampled"], "error": str(err)[:200]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = set()
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms: float, ws: int, device) -> float:
    """The largest of every rank's `ms` (the job's time for a timed region
    that all replicas run between the same barriers); `ms` itself on one
    rank.  Every rank must call it at the same point."""
    if ws <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ws: int, job_ms: float) -> float:
    """Whole-job throughput of ws replicas that each processed
    units_per_rank in the region the slowest rank timed at job_ms."""
    return ws * units_per_rank / (job_ms / 1e3)


# ------------------------------------------------------------ workloads --

def make_inputs(torch, device, seed_base=0):
    """Device-resident inputs of one step (generated on the GPU)."""
    g = torch.Generator(device=device)
    g.manual_seed(2 + seed_base)
    scan = torch.randint(0, 256, (N_SCAN,), dtype=torch.int32, device=device,
                         generator=g)
    g.manual_seed(3 + seed_base)
    k32 = torch.randint(-2**31, 2**31, (N_SORT,), dtype=torch.int32,
                        device=device, generator=g)
    k64 = morton_keys(torch, device, N_SORT, 4 + seed_base)
    return scan, k32, k64


def morton_keys(torch, device, n, seed):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    centers = torch.randint(0, 1 << 20, (64, 3), dtype=torch.int64,
                            device=device, generator=g)
    key = torch.zeros(n, dtype=torch.int64, device=device)
    chunk = 1 << 25
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        idx = torch.randint(0, 64, (m,), device=device, generator=g)
        pts = centers[idx] + (torch.randn(m, 3, device=device, generator=g)
                              * float(1 << 14)).round().to(torch.int64)
        pts = pts.clamp_(0, (1 << 20) - 1)
        k = torch.zeros(m, dtype=torch.int64, device=device)
        for b in range(20):
            for a in range(3):
                k |= ((pts[:, a] >> b) & 1) << (3 * b + a)
        key[s:s + m] = k
    return key


def run_sweep(args, ws, rank, local, torch, vx, device):
    """The primitives sweep; returns its components, roofline data and e2e."""
    lib = vx.lib()
    steps, warm = args.steps, args.warmup
    base_scan, base_k32, base_k64 = make_inputs(torch, device, seed_base=rank * 10)
    vals = torch.arange(N_SORT, dtype=torch.int32, device=device)
    bufs = []
    for _ in range(steps + warm):
        bufs.append((base_scan.clone(), base_k32.clone(), vals.clone(),
                     base_k64.clone(), vals.clone()))
    gh = torch.Generator(device=device)
    gh.manual_seed(5 + rank * 10)
    hkeys = torch.randint(-2**63, 2**63 - 2, (N_HASH,), dtype=torch.int64,
                          device=device, generator=gh)
    fresh = torch.randint(-2**63, 2**63 - 2, (N_HASH // 2,), dtype=torch.int64,
                          device=device, generator=gh)
    hq = torch.cat([hkeys[torch.randperm(N_HASH, device=device, generator=gh)[:N_HASH // 2]], fresh])
    hq = hq[torch.randperm(N_HASH, device=device, generator=gh)].contiguous()
    del fresh
    slab = vx.SlabHashSet(int(N_HASH / (HASH_LOAD * 15)) + 1, N_HASH // 30)
    cuckoo = vx.CuckooMap(int(N_HASH / HASH_LOAD) + 1, 2000)
    hfound = torch.empty(N_HASH, dtype=torch.int32, device=device)
    ws_scan = torch.empty(lib.vx_scan_workspace_size(N_SCAN), dtype=torch.uint8, device=device)
    ws_sort = torch.empty(lib.vx_sort_workspace_size(N_SORT, 8), dtype=torch.uint8, device=device)
    torch.cuda.synchronize()

    def step(b):
        scan, k32, v32, k64, v64 = b
        vx.exclusive_sum(scan, ws_scan)
        vx.sort_pairs(k32, v32, 32, ws_sort)
        vx.sort_pairs(k64, v64, 60, ws_sort)
        slab.clear()
        slab.insert(hkeys)
        slab.contains(hq, hfound)
        cuckoo.clear()
        cuckoo.insert(hkeys)
        cuckoo.find(hq, hfound)

    for i in range(warm):
        step(bufs[i])
    torch.cuda.synchronize()

    # Per-component times (events around each op) and the whole step.
    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    lib.vx_profile_reset()
    lib.vx_profile_enable(1)
    launches0 = lib.vx_profile_launches()
    stream = torch.cuda.current_stream()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(10)]
          for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        clk.mark("start")
        t0.record(stream)
        for i in range(steps):
            scan, k32, v32, k64, v64 = bufs[warm + i]
            ev[i][0].record(stream)
            vx.exclusive_sum(scan, ws_scan)
            ev[i][1].record(stream)
            vx.sort_pairs(k32, v32, 32, ws_sort)
            ev[i][2].record(stream)
            vx.sort_pairs(k64, v64, 60, ws_sort)
            ev[i][3].record(stream)
            slab.clear()
            ev[i][4].record(stream)
            slab.insert(hkeys)
            ev[i][5].record(stream)
            slab.contains(hq, hfound)
            ev[i][6].record(stream)
            cuckoo.clear()
            ev[i][7].record(stream)
            cuckoo.insert(hkeys)
            ev[i][8].record(stream)
            cuckoo.find(hq, hfound)
            ev[i][9].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
        clk.mark("end")
    barrier()
    launches = lib.vx_profile_launches() - launches0
    lib.vx_profile_enable(0)
    total_ms = t0.elapsed_time(t1)
    scan_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    s32_ms = sum(e[1].elapsed_time(e[2]) for e in ev)
    s64_ms = sum(e[2].elapsed_time(e[3]) for e in ev)
    slab_ins_ms = sum(e[4].elapsed_time(e[5]) for e in ev)
    slab_q_ms = sum(e[5].elapsed_time(e[6]) for e in ev)
    ck_ins_ms = sum(e[7].elapsed_time(e[8]) for e in ev)
    ck_q_ms = sum(e[8].elapsed_time(e[9]) for e in ev)
    hits = int(hfound.ne(-1).sum().item())
    dropped = cuckoo.dropped()
    part_ms = _prof(lib, "sort_partition_u64")

    total_ms = max_over_ranks(total_ms, ws, device)

    # correctness spot check of the timed outputs (cheap, device-side)
    scan, k32, v32, k64, v64 = bufs[warm]
    host_io = None
    if rank == 0:  # inputs and outputs of the first timed step, for the CPU check
        host_io = {"scan_in": base_scan.cpu().numpy().view(np.uint32),
                   "k32_in": base_k32.cpu().numpy().view(np.uint32),
                   "k64_in": base_k64.cpu().numpy().view(np.uint64),
                   "scan_out": scan.cpu().numpy().view(np.uint32),
                   "k32_out": k32.cpu().numpy().view(np.uint32),
                   "v32_out": v32.cpu().numpy().view(np.uint32),
                   "k64_out": k64.cpu().numpy().view(np.uint64),
                   "v64_out": v64.cpu().numpy().view(np.uint32)}
    ok = bool(((k64[1:] >= k64[:-1]) | (k64[1:] < 0) | (k64[:-1] < 0)).all()) and \
        bool((k32[1:].to(torch.int64) & 0xFFFFFFFF >= k32[:-1].to(torch.int64) & 0xFFFFFFFF).all())

    bytes_step = (N_SCAN * BYTES_SCAN + N_SORT * BYTES_SORT_U32 + N_SORT * BYTES_SORT_U64
                  + 2 * N_HASH * (BYTES_HASH_INSERT + BYTES_HASH_LOOKUP))
    value = job_rate(bytes_step * steps, ws, total_ms) / 1e9
    del bufs
    torch.cuda.empty_cache()
    # A library sort beside ours, for context: torch.sort (CUB radix sort),
    # stable, on the same 2^28 32-bit keys (it returns int64 indices, so it
    # writes more than our u32 payload).
    ks = base_k32.clone()
    torch.cuda.synchronize()
    cub_ms = []
    for _ in range(3):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        torch.sort(ks, stable=True)
        b.record()
        torch.cuda.synchronize()
        cub_ms.append(a.elapsed_time(b))
    del ks
    torch.cuda.empty_cache()
    e2e = run_e2e(torch, vx, device, base_scan, base_k32, base_k64, vals,
                  ws_scan, ws_sort, max(1, min(steps, 3)), ws,
                  (slab, cuckoo, hkeys, hq))
    part_n, part_total = part_ms
    achieved = PART_U64_BYTES / (part_total / part_n / 1e3) / 1e9 if part_n else None
    hbm, kind = peaks()
    return {
        "sweep_GBps": round(value, 2),
        "sweep_ms_per_step": round(total_ms / steps, 3),
        "scan_u32_GBps": round(N_SCAN * BYTES_SCAN * steps / scan_ms / 1e6, 1),
        "sort_u32_GBps": round(N_SORT * BYTES_SORT_U32 * steps / s32_ms / 1e6, 1),
        "sort_u64_GBps": round(N_SORT * BYTES_SORT_U64 * steps / s64_ms / 1e6, 1),
        "scan_u32_ms": round(scan_ms / steps, 3),
        "sort_u32_ms": round(s32_ms / steps, 3),
        "sort_u64_ms": round(s64_ms / steps, 3),
        "sort_u32_Gkeys_per_s": round(N_SORT * steps / s32_ms / 1e6, 3),
        "library_sort_u32_ms": round(min(cub_ms), 3),
        "library_sort": "torch.sort (CUB radix sort), stable, 2^28 int32 keys -> values + int64 indices",
        "sort_u64_Gkeys_per_s": round(N_SORT * steps / s64_ms / 1e6, 3),
        "slab_insert_GBps": round(N_HASH * BYTES_HASH_INSERT * steps / slab_ins_ms / 1e6, 1),
        "slab_lookup_GBps": round(N_HASH * BYTES_HASH_LOOKUP * steps / slab_q_ms / 1e6, 1),
        "cuckoo_insert_GBps": round(N_HASH * BYTES_HASH_INSERT * steps / ck_ins_ms / 1e6, 1),
        "cuckoo_lookup_GBps": round(N_HASH * BYTES_HASH_LOOKUP * steps / ck_q_ms / 1e6, 1),
        "slab_insert_Mops": round(N_HASH * steps / slab_ins_ms / 1e3, 1),
        "slab_lookup_Mops": round(N_HASH * steps / slab_q_ms / 1e3, 1),
        "cuckoo_insert_Mops": round(N_HASH * steps / ck_ins_ms / 1e3, 1),
        "cuckoo_lookup_Mops": round(N_HASH * steps / ck_q_ms / 1e3, 1),
        "cuckoo_lookup_hit_fraction": round(hits / N_HASH, 4),
        "cuckoo_dropped": dropped,
        "sort_partition_u64": {
            "achieved_GBps": round(achieved, 1) if achieved else None,
            "frac_of_" + kind + "_hbm": round(achieved / hbm, 3) if achieved else None,
            "launches": part_n,
            "algorithmic_bytes_per_launch": PART_U64_BYTES,
            "dram_bytes_per_launch": PART_U64_TRAFFIC,
        },
        "sweep_e2e_GBps": e2e["value"],
        "sweep_outputs_sorted": ok,
        "sweep_gpu_launches": int(launches),
        "sweep_clocks": clk.summary(),
        "_io": host_io,
    }


def count_voxels(torch, vx, prims, world_exp):
    n = prims.numel() // 8
    counts = torch.zeros(n, dtype=torch.int64, device=prims.device)
    vx.check(vx.lib().vx_rasterize_count(prims.data_ptr(), n, world_exp,
                                         counts.data_ptr(), vx.stream_handle()),
             "vx_rasterize_count")
    return counts


def run_dag(args, ws, rank, local, torch, vx, device):
    """C4: batched Hash DAG edit on the 16384^3 cave terrain, plain sample,
    e2e through host buffers, per-kernel device times."""
    lib = vx.lib()
    steps, warm = args.steps, args.warmup
    world_exp = DAG_DEPTH + 2
    pristine = vx.HashDag(DAG_DEPTH, DAG_MAX_NODES, DAG_ARENA)
    torch.cuda.synchronize()
    t = time.perf_counter()
    tb0 = torch.cuda.Event(enable_timing=True)
    tb1 = torch.cuda.Event(enable_timing=True)
    tb0.record()
    pristine.build_terrain(DAG_SEED, DAG_SCALE, True)
    tb1.record()
    st = pristine.status()
    terrain_ms = tb0.elapsed_time(tb1)
    ts = pristine.stats()
    if st != 0:
        raise RuntimeError(
            f"terrain build failed: status {st}; items/level "
            f"{list(ts.items_per_level)[:DAG_DEPTH]} pairs/level "
            f"{list(ts.pairs_per_level)[:DAG_DEPTH]} nodes/level "
            f"{list(ts.nodes_per_level)[:DAG_DEPTH + 1]}")
    terrain_nodes = [int(ts.nodes_per_level[l]) for l in range(DAG_DEPTH + 1)]

    work = vx.HashDag(DAG_DEPTH, DAG_MAX_NODES, DAG_ARENA)
    prims_np = vx.config_c4_edits(DAG_EDITS, seed=DAG_SEED, world_exp=world_exp)
    prims = vx.prims_to_device(prims_np, device)
    counts = count_voxels(torch, vx, prims, world_exp)
    voxels_batch = int(counts.sum().item())

    for _ in range(warm):
        work.copy_from(pristine)
        work.apply_primitives(prims)
        st = work.status()
        if st != 0:
            raise RuntimeError(f"batched edit failed: status {st}")

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    lib.vx_profile_reset()
    lib.vx_profile_enable(1)
    launches0 = lib.vx_profile_launches()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        clk.mark("start")
        for i in range(steps):
            work.copy_from(pristine)          # restore the terrain (untimed)
            ev[i][0].record(stream)
            work.apply_primitives(prims)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        clk.mark("end")
    barrier()
    launches = lib.vx_profile_launches() - launches0
    kern = {k: _prof(lib, k) for k in ("dag_init", "dag_expand", "dag_expand_big",
                                       "dag_leafparent", "dag_build", "dag_publish")}
    lib.vx_profile_enable(0)
    st = work.status()
    if st != 0:
        raise RuntimeError(f"batched edit failed: status {st}")
    # the edited DAG (terrain + batch) as a canonical dump in host memory,
    # checked against the CPU oracle after the timed legs
    canon = work.canonical() if rank == 0 else None
    rays = run_raycast(torch, vx, device, work)
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), ws, device)
    es = work.stats()
    edited_nodes = [int(es.nodes_per_level[l]) - terrain_nodes[l] for l in range(DAG_DEPTH + 1)]
    items = [int(es.items_per_level[l]) for l in range(DAG_DEPTH)]
    pairs = [int(es.pairs_per_level[l]) for l in range(DAG_DEPTH)]
    batched_vps = voxels_batch * steps / (ms / 1e3)

    # Plain per-call path on a prefix of the same spheres.
    plain = run_plain_sample(torch, vx, device, work, pristine, prims, counts,
                             prims_np, world_exp)

    # e2e through the public call with host buffers: the primitive list comes
    # from pinned host memory each step, the status is read back.
    h_prims = prims.cpu().pin_memory()
    d_prims = torch.empty_like(prims)
    e2e_ms = 0.0
    e_steps = max(1, min(steps, 3))
    for _ in range(e_steps):
        work.copy_from(pristine)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        d_prims.copy_(h_prims, non_blocking=True)
        work.apply_primitives(d_prims)
        st = work.status()          # D2H of the status word + synchronise
        b.record(stream)
        torch.cuda.synchronize()
        if st != 0:
            raise RuntimeError(f"e2e batched edit failed: status {st}")
        e2e_ms += a.elapsed_time(b)
    e2e_ms = max_over_ranks(e2e_ms, ws, device)  # whole job: the slowest replica
    e2e = {"value": round(job_rate(voxels_batch * e_steps, ws, e2e_ms), 1),
           "unit": "voxels/s", "h2d_bytes_per_step": int(prims.numel() * 4),
           "d2h_bytes_per_step": 4, "ms_per_step": round(e2e_ms / e_steps, 3)}
    # The same batch replayed as a CUDA graph (one launch per edit).
    graph = work.graph_primitives(prims)
    g_ms = 0.0
    for i in range(steps + 1):
        work.copy_from(pristine)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        graph.launch()
        b.record(stream)
        torch.cuda.synchronize()
        if i:
            g_ms += a.elapsed_time(b)
    if work.status() != 0:
        raise RuntimeError("graph replay of the batched edit failed")
    graph_kernels = graph.kernels
    graph.close()
    dag_bytes = ts.bytes_reserved
    del work, pristine
    torch.cuda.empty_cache()
    return {
        "batched_vps": batched_vps, "ms": ms, "voxels_batch": voxels_batch,
        "terrain_ms": terrain_ms, "terrain_nodes": terrain_nodes,
        "edited_new_nodes": edited_nodes, "items_per_level": items,
        "pairs_per_level": pairs, "kernels": kern, "plain": plain, "e2e": e2e,
        "launches": int(launches), "clocks": clk.summary(),
        "dag_bytes_reserved": int(dag_bytes),
        "graph_ms": g_ms / steps, "graph_kernels": int(graph_kernels),
        "canon": canon, "prims_np": prims_np, "rays": rays,
    }


RAYS = 1 << 20
RAYS_CHECKED = 20_000


def c4_rays(n, seed=13):
    """Rays over the C4 world: from above the terrain looking down at random
    angles, and from random points in any direction."""
    import voxel_b200 as vx
    rng = np.random.default_rng(seed)
    world = 4 << DAG_DEPTH
    r = np.zeros(n, vx.RAY_DTYPE)
    o = rng.uniform(0, world, (n, 3))
    down = rng.random(n) < 0.5
    o[down, 2] = rng.uniform(10240, 12288, down.sum())
    d = rng.normal(size=(n, 3))
    d[down, 2] = -np.abs(d[down, 2]) - 0.3
    r["origin"], r["dir"], r["t_max"] = o, d, 3.0e38
    return r


def run_raycast(torch, vx, device, dag):
    """Ray casts against the edited C4 DAG: device time of one launch over
    RAYS rays (inputs resident), and the first RAYS_CHECKED hits for the CPU
    check."""
    rays = c4_rays(RAYS)
    d_rays = torch.from_numpy(rays.view(np.uint8)).to(device)
    dag.raycast(d_rays)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    reps = 3
    a.record()
    for _ in range(reps):
        hits = dag.raycast(d_rays)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    h = hits.cpu().numpy().view(np.uint32).reshape(-1, 5)
    return {"ms": ms, "rays": RAYS, "hit_fraction": float((h[:, 3] != 6).mean()),
            "check_rays": rays[:RAYS_CHECKED], "check_hits": h[:RAYS_CHECKED].copy()}


def run_plain_sample(torch, vx, device, work, pristine, prims, counts, prims_np,
                     world_exp):
    """One vx_dag_apply_voxels call per sphere (its rasterised voxel list),
    in order, starting from the terrain; the rasterisation is untimed."""
    n = PLAIN_SAMPLE
    c = counts[:n].cpu().numpy()
    cap = int(c.max())
    vox = torch.empty((max(cap, 1), 3), dtype=torch.int32, device=device)
    ws_plain = torch.empty(vx.lib().vx_dag_voxel_workspace_size(cap),
                           dtype=torch.uint8, device=device)
    zero = torch.zeros(1, dtype=torch.int64, device=device)
    work.copy_from(pristine)
    stream = torch.cuda.current_stream()
    total_ms = 0.0
    for i in range(n):
        p = prims[i:i + 1]
        vx.check(vx.lib().vx_rasterize(p.data_ptr(), 1, world_exp, zero.data_ptr(),
                                       vox.data_ptr(), vx.stream_handle()), "raster")
        op = (int(prims_np[i]["flags"]) >> 8) & 0xFF
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st = work.apply_voxels(vox[:int(c[i])], op, ws_plain)
        b.record(stream)
        if st != 0:
            raise RuntimeError(f"plain edit {i} failed: status {st}")
        torch.cuda.synchronize()
        total_ms += a.elapsed_time(b)
    voxels = int(c.sum())
    # The same prefix through the batched path must give the same voxels:
    # compare point queries of both structures.
    check = vx.HashDag(DAG_DEPTH, DAG_MAX_NODES, 1 << 30)
    check.copy_from(pristine)
    check.apply_primitives(prims[:n].contiguous())
    assert check.status() == 0
    g = torch.Generator(device=device)
    g.manual_seed(99)
    pts = torch.randint(0, 1 << world_exp, (4_000_000, 3), dtype=torch.int32,
                        device=device, generator=g)
    near = prims[:n, :3].repeat_interleave(20000, 0)
    jitter = torch.randint(-256, 257, near.shape, dtype=torch.int32, device=device,
                           generator=g)
    near = (near + jitter).clamp_(0, (1 << world_exp) - 1)
    pts = torch.cat([pts, near]).contiguous()
    mismatches = int((work.query(pts) != check.query(pts)).sum().item())
    del check
    return {"voxels_per_s": voxels / (total_ms / 1e3), "spheres": n,
            "voxels": voxels, "ms": round(total_ms, 2),
            "query_mismatches_vs_batched": mismatches,
            "points_checked": int(pts.shape[0])}


def run_svo(args, ws, rank, local, torch, vx, device):
    """C1 (plain per-call SVO edits on 256^3 with materials) and C3 (one
    batched launch of 65,536 mixed primitives on the 4096^3 cave terrain)."""
    stream = torch.cuda.current_stream()
    out = {}
    # --- C1: 256^3 heightfield, 1,000 spheres, plain path (one call each)
    depth = 6
    prims_np = vx.config_c1_edits(1000, seed=1)
    prims = vx.prims_to_device(prims_np, device)
    vox, off = vx.rasterize(prims, depth + 2)
    off_h = off.cpu().numpy()
    voxels = int(off_h[-1])
    ws_svo = torch.empty(vx.lib().vx_svo_voxel_workspace_size(int(np.diff(off_h).max())),
                         dtype=torch.uint8, device=device)
    ops = [((int(p["flags"]) >> 8) & 0xFF, (int(p["flags"]) >> 16) & 0xFF) for p in prims_np]
    times = []
    # best of four timed passes (each the whole 1,000-call sequence) after
    # the warm-up ones: a per-call path is sensitive to host noise
    for rep in range(max(1, args.warmup // 3) + 4):
        s1 = vx.Svo(depth, 1 << 18, 1 << 18, materials=True, arena_bytes=64 << 20)
        s1.build_terrain(1, 1, False)
        assert s1.status() == 0
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i, (op, mat) in enumerate(ops):
            st = s1.apply_voxels(vox[off_h[i]:off_h[i + 1]], op, mat, ws_svo)
            if st != 0:
                raise RuntimeError(f"C1 plain edit {i} failed: {st}")
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
        del s1
    out["svo_c1_plain_ms"] = round(min(times[1:] or times), 2)
    out["svo_c1_plain_voxels_per_s"] = round(voxels / (out["svo_c1_plain_ms"] / 1e3), 1)
    # the same 1,000 spheres in one batched launch
    times = []
    for rep in range(args.warmup + args.steps):
        s1 = vx.Svo(depth, 1 << 18, 1 << 18, materials=True, arena_bytes=64 << 20)
        s1.build_terrain(1, 1, False)
        assert s1.status() == 0
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s1.apply_primitives(prims)
        b.record(stream)
        assert s1.status() == 0
        times.append(a.elapsed_time(b))
        del s1
    t_b = sum(times[args.warmup:]) / args.steps
    out["svo_c1_voxels"] = voxels
    out["svo_c1_batched_ms"] = round(t_b, 3)
    out["svo_c1_batched_voxels_per_s"] = round(voxels / (t_b / 1e3), 1)
    del vox
    # --- C3: 4096^3 cave terrain (scale 16), 65,536 mixed primitives batched
    depth = SVO_C3_DEPTH
    c3_np = vx.config_c3_edits(SVO_C3_EDITS, seed=6, world_exp=depth + 2)
    out["_c3_prims"] = c3_np
    prims = vx.prims_to_device(c3_np, device)
    c3_vox = int(count_voxels(torch, vx, prims, depth + 2).sum().item())
    s3 = vx.Svo(depth, 1 << 25, 1 << 27, materials=True, arena_bytes=8 << 30)
    times = []
    build_ms = None
    for rep in range(args.warmup + args.steps):
        a0 = torch.cuda.Event(enable_timing=True)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        s3.build_terrain(6, 16, True)      # restore the terrain (untimed)
        a.record(stream)
        s3.apply_primitives(prims)
        b.record(stream)
        st = s3.status()
        if st != 0:
            c = s3.counters()
            raise RuntimeError(f"C3 batched edit failed: {st} (nodes {c.node_count}, "
                               f"leaves {c.leaf_count})")
        build_ms = a0.elapsed_time(a)
        times.append(a.elapsed_time(b))
    t3 = sum(times[args.warmup:]) / args.steps
    c = s3.counters()
    out["_c3_canon"] = s3.canonical() if rank == 0 else None
    out["svo_c3_terrain_build_ms"] = round(build_ms, 2)
    out["svo_c3_voxels"] = c3_vox
    out["svo_c3_batched_ms"] = round(t3, 3)
    out["svo_c3_batched_voxels_per_s"] = round(c3_vox / (t3 / 1e3), 1)
    out["svo_c3_nodes_leaves_live"] = [c.node_count - c.free_node_count,
                                       c.leaf_count - c.free_leaf_count]
    del s3
    torch.cuda.empty_cache()
    return out


def run_serve(args, ws, rank, local, torch, vx, device):
    """C5: resident 8192^3 cave-terrain DAG, Poisson arrivals submitted in
    real time, continuous batching; p50 / p99 edit-to-commit latency."""
    import threading
    world_exp = SERVE_DEPTH + 2
    arr, sizes, prims = vx.generate_requests(world_exp, SERVE_RATE, args.serve_seconds, 8)
    offs = np.zeros(len(sizes) + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    dprims = vx.prims_to_device(prims, device)
    voxels = int(count_voxels(torch, vx, dprims, world_exp).sum().item())
    dag = vx.HashDag(SERVE_DEPTH, SERVE_MAX_NODES, SERVE_ARENA)
    dag.build_terrain(8, 32, True)
    assert dag.status() == 0
    srv = vx.Server(dag, max_batch_prims=1 << 16, compact_at_fill=0.9)
    t0 = srv.now_ns() + 200_000_000  # first arrival 0.2 s from now

    def submitter():
        for i in range(len(arr)):
            due = t0 + int(arr[i])
            while True:
                now = srv.now_ns()
                if now >= due:
                    break
                time.sleep(min(0.002, (due - now) / 1e9))
            srv.submit(i, prims[offs[i]:offs[i + 1]], due)

    th = threading.Thread(target=submitter)
    with ClockSampler(local) as clk:
        clk.mark("start")
        th.start()
        th.join()
        srv.drain()
        clk.mark("end")
    done = srv.poll(len(arr) + 16)
    st = srv.stats()
    srv.close()
    ok = done["status"] == 0
    # leaf blocks of sample regions of the final DAG, checked on the CPU later
    regions = c5_regions()
    n_leaf = 1 << (SERVE_DEPTH - C5_REGION_BASE)
    blocks = [dag.read_leaves([v // 4 for v in r], (n_leaf,) * 3).cpu().numpy().view(np.uint64)
              for r in regions] if rank == 0 else None
    committed = np.zeros(len(arr), bool)
    committed[done["request_id"][ok].astype(np.int64)] = True
    lat_ms = (done["commit_ns"][ok].astype(np.int64) - done["arrival_ns"][ok].astype(np.int64)) / 1e6
    span_s = (int(done["commit_ns"].max()) - t0) / 1e9
    # Spot check: the same primitives applied with the batched call in
    # sequential chunks on a fresh terrain must give the same voxels.
    check = vx.HashDag(SERVE_DEPTH, SERVE_MAX_NODES, SERVE_ARENA)
    check.build_terrain(8, 32, True)
    chunk = 1 << 16
    for a in range(0, dprims.shape[0], chunk):
        part = dprims[a:a + chunk].contiguous()
        check.apply_primitives(part)
        if check.status() != 0:      # tables full: compact and apply again
            check.compact()
            check.apply_primitives(part)
            if check.status() != 0:
                raise RuntimeError("sequential check could not apply a chunk")
        if (a // chunk) % 16 == 15:
            check.compact()
    g = torch.Generator(device=device)
    g.manual_seed(5)
    pts = torch.randint(0, 1 << world_exp, (8_000_000, 3), dtype=torch.int32,
                        device=device, generator=g)
    mism = int((dag.query(pts) != check.query(pts)).sum().item())
    del check, dag, dprims
    torch.cuda.empty_cache()
    return {
        "serve_requests": int(len(arr)),
        "serve_prims": int(len(prims)),
        "serve_voxels": voxels,
        "serve_committed": int(ok.sum()),
        "serve_p50_ms": round(float(np.percentile(lat_ms, 50)), 3),
        "serve_p99_ms": round(float(np.percentile(lat_ms, 99)), 3),
        "serve_max_ms": round(float(lat_ms.max()), 3),
        "serve_voxels_per_s": round(voxels / span_s, 1),
        "serve_wall_s": round(span_s, 2),
        "serve_batches": int(st.batches),
        "serve_compactions": int(st.compactions),
        "serve_compact_ms_total": round(st.compact_ms, 1),
        "serve_compact_share": round(st.compact_ms / 1e3 / span_s, 4),
        "serve_p999_ms": round(float(np.percentile(lat_ms, 99.9)), 3),
        "serve_query_mismatches_vs_sequential": mism,
        "_c5": {"regions": regions, "blocks": blocks, "prims": prims, "offs": offs,
                "committed": committed},
        "serve_clocks": clk.summary(),
        "serve_config": f"8192^3 cave terrain (scale 32), Poisson {SERVE_RATE:g} req/s for "
                        f"{args.serve_seconds:g} s, Zipf(1.2) sizes in [1, 4096], "
                        "r log-uniform [1, 128], 50/50 add/remove, spheres/boxes",
    }


def c5_regions():
    """Seeded 256^3 cells of the served world: half in the band of the
    terrain surface (height 4096 + 1280 v), half anywhere."""
    rng = np.random.default_rng(51)
    side = 4 << (SERVE_DEPTH - C5_REGION_BASE)
    world = 4 << SERVE_DEPTH
    out = []
    for i in range(C5_REGIONS):
        x, y = (int(v) for v in rng.integers(0, world, 2))
        z = int(rng.integers(0, world) if i % 2 else rng.integers(2816, 5376))
        out.append((x // side * side, y // side * side, z // side * side))
    return out


def prims_reaching(prims, lo, hi):
    """The primitives whose bounding box meets the box [lo, hi), in order."""
    c = prims["c"].astype(np.int64)
    r = prims["r"].astype(np.int64)
    sphere = (prims["flags"] & 0xFF) == 0
    r = np.where(sphere[:, None], r[:, :1], r)
    return prims[np.all((c + r >= np.asarray(lo)) & (c - r < np.asarray(hi)), axis=1)]


def run_parity(dag, svo, serve, sweep):
    """Every configuration's GPU result against the CPU oracle on the host
    cores (after the timed legs): C4 and C3 as full canonical dumps, the
    served C5 DAG on seeded regions (leaf masks of each 256^3 cell after all
    committed requests in arrival order; the whole 24.8 M-primitive stream is
    beyond a CPU replay), the 2^28 sorts (keys and the index payload, so
    stability too) and the scan bit for bit."""
    import oracle
    out = {}
    secs = {}
    t = time.perf_counter()
    want = oracle.Sparse(DAG_DEPTH, oracle.terrain(DAG_SEED, DAG_SCALE, True), dag["prims_np"])
    out["c4_full_dag"] = want.dag() == oracle.DagCanon(*dag["canon"])
    rc = dag["rays"]
    out["c4_raycast"] = bool(np.array_equal(want.raycast(rc["check_rays"]), rc["check_hits"]))
    del want
    secs["c4"] = time.perf_counter() - t
    t = time.perf_counter()
    want = oracle.Sparse(SVO_C3_DEPTH, oracle.terrain(6, 16, True), svo["_c3_prims"],
                         materials=True).svo()
    got = oracle.SvoCanon(*svo["_c3_canon"])
    out["c3_full_svo_with_materials"] = bool(want == got and np.array_equal(want.mats, got.mats))
    del want, got
    secs["c3"] = time.perf_counter() - t
    if serve:
        t = time.perf_counter()
        c5 = serve["_c5"]
        keep = np.repeat(c5["committed"], np.diff(c5["offs"]))
        prims = c5["prims"][keep]
        side = 4 << (SERVE_DEPTH - C5_REGION_BASE)
        n_leaf = side // 4
        tt = oracle.terrain(8, 32, True)
        good = 0
        for r, block in zip(c5["regions"], c5["blocks"]):
            part = prims_reaching(prims, r, [v + side for v in r])
            cpu = oracle.Sparse(SERVE_DEPTH, tt, part, base=C5_REGION_BASE, cell=r,
                                shard_levels=1).leaf_block([v // 4 for v in r], (n_leaf,) * 3)
            good += int(np.array_equal(cpu, block))
        out["c5_regions_equal"] = f"{good}/{len(c5['regions'])}"
        out["c5_all_regions"] = good == len(c5["regions"])
        secs["c5"] = time.perf_counter() - t
    io = sweep["_io"]
    t = time.perf_counter()
    threads = os.cpu_count() or 1
    L = oracle.lib()
    exp = np.empty_like(io["scan_in"])
    L.orc_exclusive_scan_u32_mt(io["scan_in"].ctypes.data, exp.ctypes.data, exp.size, threads)
    out["scan_2p28"] = bool(np.array_equal(exp, io["scan_out"]))
    for bits, kin, kout, vout, name in ((32, "k32_in", "k32_out", "v32_out", "sort_u32_2p28"),
                                        (60, "k64_in", "k64_out", "v64_out", "sort_u64_2p28")):
        k = io[kin].copy()
        v = np.arange(k.size, dtype=np.uint32)
        fn = L.orc_radix_sort_pairs_u32_mt if bits == 32 else L.orc_radix_sort_pairs_u64_mt
        fn(k.ctypes.data, v.ctypes.data, k.size, bits, threads)
        out[name] = bool(np.array_equal(k, io[kout]) and np.array_equal(v, io[vout]))
        del k, v
    secs["primitives"] = time.perf_counter() - t
    out["all"] = all(v for k, v in out.items() if isinstance(v, bool))
    out["cpu_seconds"] = {k: round(v, 1) for k, v in secs.items()}
    out["oracle"] = (f"oracle/oracle_sparse.cpp (sequential application on a sparse "
                     f"hash-consed DAG, {threads} host threads) and oracle_prims.cpp")
    return out


def run_ours(args, ws, rank, local):
    import torch
    import voxel_b200 as vx

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dag = run_dag(args, ws, rank, local, torch, vx, device)
    svo = run_svo(args, ws, rank, local, torch, vx, device)
    serve = run_serve(args, ws, rank, local, torch, vx, device) if args.serve_seconds > 0 else {}
    sweep = run_sweep(args, ws, rank, local, torch, vx, device)
    hbm, kind = peaks()
    k = dag["kernels"]
    top = max(("dag_expand", "dag_expand_big", "dag_leafparent", "dag_build"),
              key=lambda n: k[n][1])
    total_k = sum(v[1] for v in k.values())
    # Algorithmic bytes of one leaf-parent launch (the last level of the
    # expansion): per item its 32-B record, 4-B result, the old parent item
    # (~24 B) and the new item's hash-cons (8-B index slot + ~24-B item), and
    # per leaf child the old leaf (8 B) and its hash-cons slot (read + CAS,
    # 16 B); per (item, primitive) pair the 4-B index and 32-B primitive.
    lp_items = dag["items_per_level"][DAG_DEPTH - 1]
    lp_pairs = dag["pairs_per_level"][DAG_DEPTH - 1]
    lp_bytes = lp_items * (32 + 4 + 24 + 32 + 8 * (8 + 16)) + lp_pairs * 36
    lp_n, lp_ms = k["dag_leafparent"]
    lp_achieved = lp_bytes / (lp_ms / lp_n / 1e3) / 1e9 if lp_n else None
    plain = dag["plain"]
    result = {
        "metric": METRIC,
        "value": round(ws * dag["batched_vps"], 1),
        "unit": "voxels/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dag["ms"] / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32/u64",
        "data": "synthetic (seeded cave terrain and edit streams)",
        "config": {
            "workload": "batched Hash DAG edit: 16384^3 DAG (reference depth 12, "
                        "4^3 u64 leaves, one table per level) from the cave "
                        "terrain at scale 64, one batch of 16,384 spheres "
                        "(r log-uniform [1,256], 60% add, seed 7); plus the "
                        "primitives sweep (scan/sort 2^28, slab/cuckoo 2^26)",
            "voxels_per_batch": dag["voxels_batch"],
            "l2_policy": "DAG tables and edit arenas of tens of GB (>> L2); "
                         "sweep inputs are fresh 1-3 GB buffers per step",
            "step": "restore terrain snapshot (device copy, untimed) + batched edit",
            "parallelism": f"replicas x{ws}",
        },
        "components": {
            "batched_voxels_per_s": round(dag["batched_vps"], 1),
            "plain_voxels_per_s": round(plain["voxels_per_s"], 1),
            "batched_over_plain": round(dag["batched_vps"] / plain["voxels_per_s"], 2),
            "plain_sample": {k2: v for k2, v in plain.items() if k2 != "voxels_per_s"},
            "terrain_build_ms": round(dag["terrain_ms"], 2),
            "terrain_nodes_per_level": dag["terrain_nodes"],
            "new_nodes_per_batch": dag["edited_new_nodes"],
            "work_items_per_level": dag["items_per_level"],
            "pairs_per_level": dag["pairs_per_level"],
            "dag_kernel_ms": {n: round(v[1], 3) for n, v in k.items()},
            "dag_kernel_share": {n: round(v[1] / total_k, 3) for n, v in k.items()} if total_k else {},
            "dag_bytes_reserved": dag["dag_bytes_reserved"],
            "batched_graph_ms_per_batch": round(dag["graph_ms"], 3),
            "batched_graph_voxels_per_s": round(dag["voxels_batch"] / (dag["graph_ms"] / 1e3), 1),
            "batched_graph_kernels": dag["graph_kernels"],
            "raycast_Mrays_per_s": round(dag["rays"]["rays"] / dag["rays"]["ms"] / 1e3, 1),
            "raycast_ms": round(dag["rays"]["ms"], 3),
            "raycast_hit_fraction": round(dag["rays"]["hit_fraction"], 3),
            "tuning": vx.tuning(),
            **{k2: v for k2, v in svo.items() if not k2.startswith("_")},
            **{k2: v for k2, v in serve.items() if not k2.startswith("_")},
            **{k2: v for k2, v in sweep.items() if not k2.startswith("_")},
        },
        "roofline": {
            "kernel": "dag_leafparent",
            "dominant_kernel_measured": top,
            "bound": "hbm",
            "achieved": round(lp_achieved, 1) if lp_achieved else None,
            "peak": hbm,
            "peak_kind": kind,
            "unit": "GB/s",
            "frac": round(lp_achieved / hbm, 4) if lp_achieved else None,
            "traffic": (round(LEAFPARENT_TRAFFIC_PER_ITEM * lp_items)
                        if LEAFPARENT_TRAFFIC_PER_ITEM else None),
            # the DRAM bytes ncu counted per item, over the measured launch time
            "dram_frac": (round(LEAFPARENT_TRAFFIC_PER_ITEM * lp_items / (lp_ms / lp_n / 1e3)
                                / 1e9 / hbm, 4)
                          if LEAFPARENT_TRAFFIC_PER_ITEM and lp_n else None),
            "algorithmic_bytes_per_launch": lp_bytes,
            "launches": lp_n,
            "avg_launch_ms": round(lp_ms / lp_n, 3) if lp_n else None,
        },
        "e2e": dag["e2e"],
        "gpu_launches": dag["launches"],
        "clocks": dag["clocks"],
    }
    parity = run_parity(dag, svo, serve, sweep) if rank == 0 else None
    del dag, svo, serve, sweep
    if rank == 0:
        result["cpu_baseline"] = dag_cpu_baseline()
        # the headline ratios and the CPU parity verdicts, last on the line
        result["parity"] = parity
        result["summary"] = {
            "batched_voxels_per_s": result["value"],
            "batched_over_plain": result["components"]["batched_over_plain"],
            "over_reference_cpu": (round(result["value"] / result["cpu_baseline"]["value"], 1)
                                   if result["cpu_baseline"]["value"] else None),
            "parity_all": parity["all"],
        }
        # the same verdicts right after the headline keys too, for readers that
        # keep only the start of the line
        head = ("metric", "value", "unit")
        result = {**{k: result[k] for k in head}, "headline": result["summary"],
                  **{k: v for k, v in result.items() if k not in head}}
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return result


# The reference CPU sample: the reference HashDAG(12) holding the cave terrain
# of one 2048^3 cell of the C4 world (the cell at level 3 that contains voxel
# REF_CELL; the rest of its world is empty), edited with the first
# REF_SPHERES spheres of the C4 list that reach the cell, clipped to it.  The
# whole 16384^3 terrain does not fit the reference's HashDAG: its levels above
# 10 have 2^10 buckets of 2^11 words (2 M words), and the terrain needs about
# 3 M words at level 8 and 11 M at level 9.
REF_BASE = 3
REF_CELL = (8192, 8192, 8192)
REF_SPHERES = 11


def reference_sample():
    """(dag, spheres, lo, hi, terrain_dump): a reference HashDAG(12) loaded
    with the terrain of the sample cell, and the sample's spheres."""
    import oracle
    t = oracle.terrain(seed=DAG_SEED, scale=DAG_SCALE, caves=True)
    side = 4 << (DAG_DEPTH - REF_BASE)
    lo = np.array([c // side * side for c in REF_CELL], np.int64)
    hi = lo + side
    prims = oracle.config_c4_edits(DAG_EDITS, seed=DAG_SEED, world_exp=DAG_DEPTH + 2)
    c = prims["c"].astype(np.int64)
    r = prims["r"][:, 0].astype(np.int64)
    reach = np.all((c + r[:, None] >= lo) & (c - r[:, None] < hi), axis=1)
    spheres = prims[reach][:REF_SPHERES]
    dump = oracle.Sparse(DAG_DEPTH, t, None, base=REF_BASE, cell=REF_CELL,
                         shard_levels=2).dag()
    return spheres, lo, hi, dump


def reference_run(spheres, lo, hi, dump, check: bool = False):
    """Time the sample on a fresh reference HashDAG(12) (terrain import
    untimed); with check, also compare the edited cell with the sparse
    oracle's sequential application (canonical dumps)."""
    import oracle
    d = oracle.RefDag(DAG_DEPTH)
    d.import_region(REF_BASE, REF_CELL, dump)
    f = oracle.ref().ref_dag_apply_prim_clipped
    lo_c, hi_c = np.ascontiguousarray(lo), np.ascontiguousarray(hi)
    voxels = 0
    t0 = time.perf_counter()
    for p in spheres:
        fl = int(p["flags"])
        v = f(d._h, fl & 0xFF, *map(int, p["c"]), *map(int, p["r"]),
              int(((fl >> 8) & 0xFF) == 1), lo_c.ctypes.data, hi_c.ctypes.data)
        if v < 0:
            raise RuntimeError("reference HashDAG edit failed")
        voxels += v
    secs = time.perf_counter() - t0
    same = None
    if check:
        t = oracle.terrain(seed=DAG_SEED, scale=DAG_SCALE, caves=True)
        want = oracle.Sparse(DAG_DEPTH, t, spheres, base=REF_BASE, cell=REF_CELL,
                             shard_levels=2).dag()
        got = d.canon()
        skip = int(sum(got.counts[:REF_BASE])) * 10
        same = (got.counts[REF_BASE:] == want.counts and got.root == 2
                and np.array_equal(got.nodes[skip:], want.nodes)
                and np.array_equal(got.leaves, want.leaves))
    return voxels, secs, same


def reference_sample_text(voxels, secs):
    return (f"reference HashDAG(12) holding the cave terrain of the 2048^3 cell at "
            f"{tuple(c // 2048 * 2048 for c in REF_CELL)} of the C4 world, edited with the "
            f"first {REF_SPHERES} of the 16,384 C4 spheres that reach it (x-run "
            f"fill_box/clear_box clipped to the cell): {voxels} voxels in {secs:.2f} s, "
            f"1 thread (the reference is single-threaded; host has {os.cpu_count()} "
            "threads); the full terrain exceeds the reference's fixed bucket capacity")


def dag_cpu_baseline():
    """The reference's own CPU HashDAG (oracle/_ref, compiled from its
    headers) on the fixed C4 sample, 1 thread; also checks the sample's
    result against the sparse oracle."""
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": "voxels/s", "cores": 1, "kind": "reference",
                "sample": "reference shim not built"}
    spheres, lo, hi, dump = reference_sample()
    voxels, secs, same = reference_run(spheres, lo, hi, dump, check=True)
    return {"value": round(voxels / secs, 1), "unit": "voxels/s", "cores": 1,
            "kind": "reference", "sample": reference_sample_text(voxels, secs),
            "sample_matches_oracle": same}


def _prof(lib, name):
    import ctypes as C
    ms = C.c_double(0)
    n = C.c_uint64(0)
    lib.vx_profile_query(name.encode(), C.byref(ms), C.byref(n))
    return n.value, ms.value


def run_e2e(torch, vx, device, base_scan, base_k32, base_k64, vals, ws_scan,
            ws_sort, steps, world, hash_parts):
    """Same sweep through the public API with host inputs: every step copies
    its inputs from pinned host memory and reads every result back."""
    slab, cuckoo, hkeys, hq = hash_parts
    srcs = [t.cpu().pin_memory() for t in (base_scan, base_k32, vals, base_k64,
                                            vals, hkeys, hq)]
    d = [torch.empty_like(t, device=device) for t in srcs]
    found = torch.empty(N_HASH, dtype=torch.int32, device=device)
    outs = [torch.empty_like(t).pin_memory() for t in srcs[:5]]
    h_found = [torch.empty(N_HASH, dtype=torch.int32).pin_memory() for _ in range(2)]
    stream = torch.cuda.current_stream()
    h2d = sum(t.numel() * t.element_size() for t in srcs)
    d2h = sum(t.numel() * t.element_size() for t in outs) + 2 * N_HASH * 4

    def one():
        for dst, src in zip(d, srcs):
            dst.copy_(src, non_blocking=True)
        vx.exclusive_sum(d[0], ws_scan)
        vx.sort_pairs(d[1], d[2], 32, ws_sort)
        vx.sort_pairs(d[3], d[4], 60, ws_sort)
        for o, s in zip(outs, d):
            o.copy_(s, non_blocking=True)
        slab.clear()
        slab.insert(d[5])
        slab.contains(d[6], found)
        h_found[0].copy_(found, non_blocking=True)
        cuckoo.clear()
        cuckoo.insert(d[5])
        cuckoo.find(d[6], found)
        h_found[1].copy_(found, non_blocking=True)

    one()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        one()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    bytes_step = (N_SCAN * BYTES_SCAN + N_SORT * BYTES_SORT_U32 + N_SORT * BYTES_SORT_U64
                  + 2 * N_HASH * (BYTES_HASH_INSERT + BYTES_HASH_LOOKUP))
    return {"value": round(world * bytes_step * steps / (ms / 1e3) / 1e9, 2),
            "unit": "GB/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(ms / steps, 2)}


def cpu_baseline(sample_log2=24):
    """Oracle port on all host threads over a 2^24-element sample of each
    component, reported in the same algorithmic GB/s."""
    import oracle
    threads = os.cpu_count() or 1
    n = 1 << sample_log2
    rng = np.random.default_rng(2)
    x = rng.integers(0, 256, n, dtype=np.uint32)
    out = np.empty_like(x)
    k32 = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    k64 = rng.integers(0, 2**60, n, dtype=np.uint64)
    v = np.arange(n, dtype=np.uint32)
    L = oracle.lib()
    t = time.perf_counter()
    L.orc_exclusive_scan_u32_mt(x.ctypes.data, out.ctypes.data, n, threads)
    t_scan = time.perf_counter() - t
    kk, vv = k32.copy(), v.copy()
    t = time.perf_counter()
    L.orc_radix_sort_pairs_u32_mt(kk.ctypes.data, vv.ctypes.data, n, 32, threads)
    t_s32 = time.perf_counter() - t
    kk, vv = k64.copy(), v.copy()
    t = time.perf_counter()
    L.orc_radix_sort_pairs_u64_mt(kk.ctypes.data, vv.ctypes.data, n, 60, threads)
    t_s64 = time.perf_counter() - t
    nh = n >> 2
    hk = rng.integers(0, 2**64 - 2, nh, dtype=np.uint64)
    hq = np.concatenate([hk[: nh // 2], rng.integers(0, 2**64 - 2, nh // 2, dtype=np.uint64)])
    t = time.perf_counter()
    oracle.hash_set(hk, hq)
    t_hash = time.perf_counter() - t
    total_b = (n * (BYTES_SCAN + BYTES_SORT_U32 + BYTES_SORT_U64)
               + 2 * nh * (BYTES_HASH_INSERT + BYTES_HASH_LOOKUP))
    # std::unordered_set is single-threaded: one set stands for both tables.
    secs = t_scan + t_s32 + t_s64 + 2 * t_hash
    return {"value": round(total_b / secs / 1e9, 3),
            "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"2^{sample_log2} elements per scan/sort component on "
                      f"{threads} host threads; 2^{sample_log2 - 2} u64 keys "
                      "inserted + looked up in std::unordered_set (1 thread), "
                      "counted for both hash tables",
            "seconds": round(secs, 3)}


def run_reference(args, ws, rank):
    """The reference's own CPU implementation of the headline path: its
    HashDAG (oracle/_ref, compiled from the reference headers) on the fixed
    C4 sample (reference_sample), 1 thread (the reference is
    single-threaded).  Each step re-imports the terrain (untimed) and applies
    the sample; rank 0 only.  Loads nothing of this repository's library."""
    if rank != 0:
        return None
    import oracle
    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "reference shim not built"}
    spheres, lo, hi, dump = reference_sample()
    for _ in range(args.warmup):
        reference_run(spheres, lo, hi, dump)
    runs = [reference_run(spheres, lo, hi, dump) for _ in range(args.steps)]
    voxels = runs[0][0]
    secs = statistics.median(r[1] for r in runs)
    v = round(voxels / secs, 1)
    return {"metric": METRIC, "value": v, "unit": "voxels/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(secs * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/u64", "data": "synthetic (seeded cave terrain and edit stream)",
            "impl": "reference",
            "config": {"workload": "batched Hash DAG edit: the C4 cave terrain (scale 64) "
                                   "and sphere list (r log-uniform [1,256], 60% add, "
                                   "seed 7), sampled on one 2048^3 cell",
                       "parallelism": "1 host thread"},
            "cpu_baseline": {"value": v, "unit": "voxels/s", "cores": 1,
                             "kind": "reference",
                             "sample": reference_sample_text(voxels, secs)},
            "e2e": {"value": v, "unit": "voxels/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_case_dag_full(args, torch, vx, dev):
    """The C4 batch alone (16384^3 terrain, 16,384 spheres): device time per
    batch and per kernel over --steps batches, each from the restored
    terrain; for measuring and profiling the headline edit."""
    lib = vx.lib()
    world_exp = DAG_DEPTH + 2
    pristine = vx.HashDag(DAG_DEPTH, DAG_MAX_NODES, DAG_ARENA)
    pristine.build_terrain(DAG_SEED, DAG_SCALE, True)
    assert pristine.status() == 0
    work = vx.HashDag(DAG_DEPTH, DAG_MAX_NODES, DAG_ARENA)
    prims = vx.prims_to_device(vx.config_c4_edits(DAG_EDITS, seed=DAG_SEED, world_exp=world_exp),
                               dev)
    stream = torch.cuda.current_stream()
    ms = []
    lib.vx_profile_reset()
    for i in range(args.steps + 1):
        work.copy_from(pristine)
        lib.vx_profile_enable(1 if i else 0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        work.apply_primitives(prims)
        b.record(stream)
        torch.cuda.synchronize()
        lib.vx_profile_enable(0)
        assert work.status() == 0
        if i:
            ms.append(a.elapsed_time(b))
    kern = {k: round(_prof(lib, k)[1] / args.steps, 3)
            for k in ("dag_expand", "dag_expand_big", "dag_leafparent", "dag_build")}
    print(json.dumps({"case": "dag_full", "ms": [round(x, 3) for x in ms],
                      "kernel_ms_per_batch": kern, "tuning": vx.tuning()}))


def run_case_hash(args, torch, vx, dev):
    """--case slab|cuckoo --elements N: N u64 keys inserted at load factor
    0.8, then N lookups at 50 % hits, --steps times; device time per insert
    and per lookup launch (for profiling the hash tables alone)."""
    n = args.elements
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    keys = torch.randint(-2**63, 2**63 - 2, (n,), dtype=torch.int64, device=dev, generator=g)
    fresh = torch.randint(-2**63, 2**63 - 2, (n // 2,), dtype=torch.int64, device=dev, generator=g)
    q = torch.cat([keys[torch.randperm(n, device=dev, generator=g)[:n // 2]], fresh])
    q = q[torch.randperm(n, device=dev, generator=g)].contiguous()
    out = torch.empty(n, dtype=torch.int32, device=dev)
    if args.case == "slab":
        t = vx.SlabHashSet(int(n / (HASH_LOAD * 15)) + 1, n // 30)
        ins, look = (lambda: t.insert(keys)), (lambda: t.contains(q, out))
    else:
        t = vx.CuckooMap(int(n / HASH_LOAD) + 1, 2000)
        ins, look = (lambda: t.insert(keys)), (lambda: t.find(q, out))
    res = {"insert_ms": [], "lookup_ms": []}
    for _ in range(args.steps):
        t.clear()
        for name, fn in (("insert_ms", ins), ("lookup_ms", look)):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            res[name].append(round(a.elapsed_time(b), 3))
    print(json.dumps({"case": args.case, "elements": n, **res}))


def run_case_gather(args, torch, dev):
    """--case gather --elements N: N random 8-byte reads from a 2 GiB table
    (torch.take, a library gather), each touching one 32-byte sector: the rate
    of random sectors the hash tables' lookups are bound by."""
    n = args.elements
    table = torch.zeros(1 << 28, dtype=torch.int64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(9)
    idx = torch.randint(0, 1 << 28, (n,), dtype=torch.int64, device=dev, generator=g)
    torch.take(table, idx)
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        torch.take(table, idx)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    best = min(ms)
    print(json.dumps({"case": "gather", "elements": n, "ms": [round(x, 3) for x in ms],
                      "G_sectors_per_s": round(n / best / 1e6, 2)}))


def run_case(args):
    """One operation alone, for profiler captures: --case scan|sort_u32|sort_u64
    --elements N (runs --steps launches); --case dag --elements E (E spheres
    on a 4096^3 terrain); --case dag_full (the headline C4 batch, --steps
    batches, device time per batch and per kernel); --case slab|cuckoo
    --elements N (insert and look up N u64 keys)."""
    import torch
    import voxel_b200 as vx
    dev = torch.device("cuda:0")
    for setting in args.tuning:  # NAME=VALUE launch-shape knobs for this case
        name, _, value = setting.partition("=")
        vx.set_tuning(name, int(value))
    n = args.elements
    ms = []
    if args.case == "dag_full":
        return run_case_dag_full(args, torch, vx, dev)
    if args.case in ("slab", "cuckoo"):
        return run_case_hash(args, torch, vx, dev)
    if args.case == "gather":
        return run_case_gather(args, torch, dev)
    for _ in range(args.steps):
        if args.case == "scan":
            x = torch.randint(0, 256, (n,), dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            t = time.perf_counter()
            vx.exclusive_sum(x)
        elif args.case == "sort_u32":
            k = torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device=dev)
            v = torch.arange(n, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            t = time.perf_counter()
            vx.sort_pairs(k, v, 32)
        elif args.case == "sort_u64":
            k = morton_keys(torch, dev, n, 4)
            v = torch.arange(n, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            t = time.perf_counter()
            vx.sort_pairs(k, v, 60)
        else:
            # dag: 4096^3 cave terrain (scale 16) + n spheres of the C4 mix
            depth = 10
            dag = vx.HashDag(depth, 1 << 23, 1 << 30)
            dag.build_terrain(7, 16, True)
            st = dag.status()
            ts = dag.stats()
            print(json.dumps({"terrain_status": st,
                              "items": list(ts.items_per_level)[:depth],
                              "nodes": list(ts.nodes_per_level)[:depth + 1]}))
            assert st == 0
            prims = vx.prims_to_device(vx.config_c4_edits(n, seed=7, world_exp=depth + 2), dev)
            torch.cuda.synchronize()
            t = time.perf_counter()
            dag.apply_primitives(prims)
            assert dag.status() == 0
            es = dag.stats()
            print(json.dumps({"edit_items": list(es.items_per_level)[:depth],
                              "edit_pairs": list(es.pairs_per_level)[:depth]}))
        torch.cuda.synchronize()
        ms.append((time.perf_counter() - t) * 1e3)
    print(json.dumps({"case": args.case, "elements": n, "ms": ms}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--case", choices=["scan", "sort_u32", "sort_u64", "dag", "dag_full",
                                       "slab", "cuckoo", "gather"],
                    default=None)
    ap.add_argument("--elements", type=int, default=1 << 24)
    ap.add_argument("--tuning", action="append", default=[], metavar="NAME=VALUE",
                    help="set a launch-shape knob for a --case run (repeatable)")
    ap.add_argument("--serve-seconds", type=float, default=SERVE_SECONDS,
                    help="length of the served arrival stream (0 skips serving)")
    args = ap.parse_args()
    if args.case is not None:
        run_case(args)
        return
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        res = run_reference(args, ws, rank)
    else:
        if args.warmup < 3:
            args.warmup = 3
        res = run_ours(args, ws, rank, local)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
