"""Autotuner for the library's launch-shape knobs (vx_tuning_*).

    python -m voxel_b200.autotune [--quick] [--out PATH]

Times every allowed value of each knob on a representative workload on the
current GPU and writes the fastest settings to voxel_b200/tuning/<device>.json,
which the library applies when it is first loaded on that kind of device:

  * sort.items_u32 / sort.items_u64 / sort.early_counts / sort.rank_ballots /
    sort.radix_bits: radix-sort partition tile size (items per thread, hence
    blocks per SM), whether a tile publishes its digit counts before or after
    ranking, whether keys are ranked with per-bit ballots or a shared-memory
    atomic OR per digit, and the digit width (6, 7 or 8 bits: 6, 5 or 4
    passes over 32-bit keys); timed on 2^26
    u32 and 2^25 60-bit u64 key/value pairs;
  * scan.tile_kb: the prefix sum's tile (32, 16 or 8 KB, with 6, 12 or 24
    resident blocks per SM); timed on 2^28 u32;
  * edit.big_item / edit.blocks_per_sm / edit.leafparent_blocks /
    edit.leafparent_lanes / edit.leafparent_prefetch: the primitive-list
    length above which a work item is expanded by a whole block, the grid of
    the edit pipelines' item kernels, and the resident blocks, threads per
    item and next-node prefetch of the DAG leaf-parent kernel; timed on the
    batched Hash
    DAG edit of the benchmark (16384^3 cave terrain at scale 64, 16,384
    spheres of radius log-uniform in [1, 256], 60 % add).

Every setting's output is compared with the default setting's (the sorted
arrays bit for bit, the edited DAG by 2^20 point queries) before its time
counts, so a setting that computed something else is reported, not chosen.
"""
from __future__ import annotations

import argparse
import itertools
import json
import time

import numpy as np
import torch

from . import lib
from . import api as vx
from . import tuning_file


def _time(fn, reps: int, before=None) -> float:
    """Median device time of fn() in ms (before() runs untimed each rep)."""
    ts = []
    for i in range(reps + 1):
        if before is not None:
            before()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        if i:  # the first run warms up
            ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def tune_sort(n32: int, n64: int, reps: int, log) -> tuple[dict, dict]:
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    cases = {
        "u32": (torch.randint(-(1 << 31), (1 << 31) - 1, (n32,), dtype=torch.int32,
                              device="cuda", generator=g), 32, "sort.items_u32"),
        "u64": (torch.randint(0, 1 << 60, (n64,), dtype=torch.int64, device="cuda",
                              generator=g), 60, "sort.items_u64"),
    }
    times: dict = {}
    for label, (keys0, bits, knob) in cases.items():
        n = keys0.numel()
        vals0 = torch.arange(n, dtype=torch.int32, device="cuda")
        ws = torch.empty(lib().vx_sort_workspace_size(n, keys0.element_size()),
                         dtype=torch.uint8, device="cuda")
        k, v = keys0.clone(), vals0.clone()

        def restore():
            k.copy_(keys0)
            v.copy_(vals0)

        vx.reset_tuning()
        restore()
        vx.sort_pairs(k, v, bits, ws)
        ref_k, ref_v = k.clone(), v.clone()
        for items, early, ballots, radix in itertools.product(
                vx.tuning_options(knob), vx.tuning_options("sort.early_counts"),
                vx.tuning_options("sort.rank_ballots"), vx.tuning_options("sort.radix_bits")):
            vx.set_tuning(knob, items)
            vx.set_tuning("sort.early_counts", early)
            vx.set_tuning("sort.rank_ballots", ballots)
            vx.set_tuning("sort.radix_bits", radix)
            restore()
            vx.sort_pairs(k, v, bits, ws)
            same = bool(torch.equal(k, ref_k) and torch.equal(v, ref_v))
            ms = _time(lambda: vx.sort_pairs(k, v, bits, ws), reps, restore) if same else None
            times[(label, items, early, ballots, radix)] = ms
            log(f"  sort {label} items={items} early={early} ballots={ballots} radix={radix}: "
                + (f"{ms:.3f} ms" if same else "DIFFERENT OUTPUT (not used)"))
    vx.reset_tuning()
    # early / ballots / digit width are shared by both key widths: pick the
    # triple with the least total time (each width at its best items); then
    # items per width.
    best: dict = {}
    score = {}
    for early, ballots, radix in itertools.product(vx.tuning_options("sort.early_counts"),
                                                   vx.tuning_options("sort.rank_ballots"),
                                                   vx.tuning_options("sort.radix_bits")):
        tot = 0.0
        for label, (_, _, knob) in cases.items():
            cand = [times[(label, i, early, ballots, radix)] for i in vx.tuning_options(knob)]
            cand = [c for c in cand if c is not None]
            tot = tot + min(cand) if cand else float("inf")
        score[(early, ballots, radix)] = tot
    early, ballots, radix = min(score, key=score.get)
    best["sort.early_counts"], best["sort.rank_ballots"] = early, ballots
    best["sort.radix_bits"] = radix
    for label, (_, _, knob) in cases.items():
        opts = {i: times[(label, i, early, ballots, radix)] for i in vx.tuning_options(knob)}
        opts = {i: t for i, t in opts.items() if t is not None}
        best[knob] = min(opts, key=opts.get)
    return best, {f"{l} items={i} early={e} ballots={b} radix={r}": t
                  for (l, i, e, b, r), t in times.items()}


def tune_scan(n: int, reps: int, log) -> tuple[dict, dict]:
    """scan.tile_kb: exclusive sum of n u32 (inputs larger than L2), each
    tile shape's output compared with the default shape's."""
    g = torch.Generator(device="cuda")
    g.manual_seed(13)
    data0 = torch.randint(0, 1 << 20, (n,), dtype=torch.int32, device="cuda", generator=g)
    ws = torch.empty(lib().vx_scan_workspace_size(n), dtype=torch.uint8, device="cuda")
    d = data0.clone()
    vx.reset_tuning()
    vx.exclusive_sum(d, ws)
    ref = d.clone()
    times: dict = {}
    for kb in vx.tuning_options("scan.tile_kb"):
        vx.set_tuning("scan.tile_kb", kb)
        d.copy_(data0)
        vx.exclusive_sum(d, ws)
        same = bool(torch.equal(d, ref))
        ms = _time(lambda: vx.exclusive_sum(d, ws), reps, lambda: d.copy_(data0)) if same else None
        times[f"tile_kb={kb}"] = ms
        log(f"  scan u32 tile_kb={kb}: " + (f"{ms:.3f} ms" if same else "DIFFERENT OUTPUT (not used)"))
    vx.reset_tuning()
    valid = {int(k.split("=")[1]): t for k, t in times.items() if t is not None}
    return {"scan.tile_kb": min(valid, key=valid.get)}, times


def tune_edit(depth: int, scale: int, count: int, reps: int, log, max_nodes: int,
              arena: int) -> tuple[dict, dict]:
    prims = vx.prims_to_device(vx.config_c4_edits(count, seed=7, world_exp=depth + 2), "cuda")
    pristine = vx.HashDag(depth, max_nodes, arena)
    pristine.build_terrain(7, scale, True)
    if pristine.status() != 0:
        raise RuntimeError("terrain build failed")
    work = vx.HashDag(depth, max_nodes, arena)
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    pts = torch.randint(0, 4 << depth, (1 << 20, 3), dtype=torch.int32, device="cuda",
                        generator=g)
    vx.reset_tuning()
    work.copy_from(pristine)
    work.apply_primitives(prims)
    if work.status() != 0:
        raise RuntimeError("reference edit failed")
    ref = work.query(pts)
    times: dict = {}

    def measure(big, bps, lpb, lanes, pf=0):
        vx.set_tuning("edit.big_item", big)
        vx.set_tuning("edit.blocks_per_sm", bps)
        vx.set_tuning("edit.leafparent_blocks", lpb)
        vx.set_tuning("edit.leafparent_lanes", lanes)
        vx.set_tuning("edit.leafparent_prefetch", pf)
        work.copy_from(pristine)
        work.apply_primitives(prims)
        ok = work.status() == 0 and bool(torch.equal(work.query(pts), ref))
        ms = _time(lambda: work.apply_primitives(prims), reps,
                   lambda: work.copy_from(pristine)) if ok else None
        if ok and work.status() != 0:
            ms = None
        key = (f"big_item={big} blocks_per_sm={bps} leafparent_blocks={lpb} "
               f"leafparent_lanes={lanes}" + (" leafparent_prefetch=1" if pf else ""))
        times[key] = ms
        log(f"  edit {key}: "
            + (f"{ms:.3f} ms" if ms is not None else "FAILED OR DIFFERENT (not used)"))
        return ms

    # Stage 1: long-list threshold and grid.  Among settings within 2 % of
    # the fastest, take the smallest grid: on a large batch more blocks gain
    # little, while on small batches (the serving loop's) every extra block
    # is launch overhead.
    lpb0 = vx.tuning()["edit.leafparent_blocks"]
    lanes0 = vx.tuning()["edit.leafparent_lanes"]
    stage1 = {}
    for big, bps in itertools.product(vx.tuning_options("edit.big_item"),
                                      vx.tuning_options("edit.blocks_per_sm")):
        ms = measure(big, bps, lpb0, lanes0)
        if ms is not None:
            stage1[(big, bps)] = ms
    fastest = min(stage1.values())
    near = [k for k, t in stage1.items() if t <= 1.02 * fastest]
    big, bps = min(near, key=lambda k: (k[1], stage1[k]))
    # Stage 2: threads per item, resident blocks and next-node prefetch of
    # the leaf-parent kernel at that setting (the prefetch form exists for 4
    # threads per item).
    stage2 = {}
    for lpb, lanes, pf in itertools.product(vx.tuning_options("edit.leafparent_blocks"),
                                            vx.tuning_options("edit.leafparent_lanes"),
                                            vx.tuning_options("edit.leafparent_prefetch")):
        if pf and lanes != 4:
            continue
        ms = measure(big, bps, lpb, lanes, pf)
        if ms is not None:
            stage2[(lpb, lanes, pf)] = ms
    lpb, lanes, pf = min(stage2, key=stage2.get)
    vx.reset_tuning()
    return {"edit.big_item": big, "edit.blocks_per_sm": bps,
            "edit.leafparent_blocks": lpb, "edit.leafparent_lanes": lanes,
            "edit.leafparent_prefetch": pf}, times


def tune_serve(depth: int, scale: int, batch: int, reps: int, log, max_nodes: int,
               arena: int) -> tuple[dict, dict]:
    """serve.blocks_per_sm: latency of one small batch (the serving loop's
    typical size) replayed as a graph with a device-side count, on the served
    terrain; the same pipeline the serving loop captures."""
    prims = vx.generate_primitives(depth + 2, batch, 8, sphere_permille=500, add_permille=500,
                                   r_min=1, r_max=128, log_uniform=True)
    buf = vx.prims_to_device(prims, "cuda")
    cnt = torch.tensor([batch], dtype=torch.int32, device="cuda")
    pristine = vx.HashDag(depth, max_nodes, arena)
    pristine.build_terrain(8, scale, True)
    if pristine.status() != 0:
        raise RuntimeError("terrain build failed")
    work = vx.HashDag(depth, max_nodes, arena)
    times: dict = {}
    for bps in vx.tuning_options("serve.blocks_per_sm"):
        vx.set_tuning("edit.blocks_per_sm", bps)  # the serving graphs' grid
        graph = work.graph_primitives(buf, cnt, batch)
        work.copy_from(pristine)
        graph.launch()
        ok = work.status() == 0
        ms = _time(graph.launch, reps, lambda: work.copy_from(pristine)) if ok else None
        graph.close()
        times[f"blocks_per_sm={bps}"] = ms
        log(f"  serve batch of {batch} blocks_per_sm={bps}: "
            + (f"{ms:.3f} ms" if ms is not None else "FAILED (not used)"))
    vx.reset_tuning()
    valid = {int(k.split("=")[1]): t for k, t in times.items() if t is not None}
    return {"serve.blocks_per_sm": min(valid, key=valid.get)}, times


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--quick", action="store_true", help="small sizes (a test run)")
    ap.add_argument("--out", default=None, help="output JSON (default: the device's file)")
    ap.add_argument("--quiet", action="store_true")
    args = ap.parse_args(argv)
    log = (lambda m: None) if args.quiet else (lambda m: print(m, flush=True))
    if not torch.cuda.is_available():
        raise SystemExit("autotune needs a CUDA device")
    dev = torch.cuda.get_device_name()
    t0 = time.time()
    if args.quick:
        sort_best, sort_t = tune_sort(1 << 20, 1 << 19, 2, log)
        scan_best, scan_t = tune_scan(1 << 20, 2, log)
        edit_best, edit_t = tune_edit(6, 1, 256, 2, log, 1 << 18, 64 << 20)
        serve_best, serve_t = tune_serve(6, 1, 64, 2, log, 1 << 18, 64 << 20)
    else:
        sort_best, sort_t = tune_sort(1 << 26, 1 << 25, 5, log)
        scan_best, scan_t = tune_scan(1 << 28, 5, log)
        edit_best, edit_t = tune_edit(12, 64, 16384, 5, log, 1 << 27, 16 << 30)
        serve_best, serve_t = tune_serve(11, 32, 400, 9, log, 1 << 27, 8 << 30)
    vx.reset_tuning()
    untuned = vx.tuning()  # knobs no sweep here times keep their defaults
    result = {
        "device": dev,
        "quick": bool(args.quick),
        "seconds": round(time.time() - t0, 1),
        "knobs": {**untuned, **sort_best, **scan_best, **edit_best, **serve_best},
        "timings_ms": {"sort": sort_t, "scan": scan_t, "edit": edit_t, "serve": serve_t},
    }
    out = args.out or str(tuning_file(dev))
    from pathlib import Path
    Path(out).parent.mkdir(parents=True, exist_ok=True)
    Path(out).write_text(json.dumps(result, indent=1) + "\n")
    log(f"best {result['knobs']} -> {out}")
    return result


if __name__ == "__main__":
    main()
