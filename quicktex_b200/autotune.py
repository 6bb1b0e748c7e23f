"""Autotuner for the batched persistent path.

For every (op, format, level) class it runs a batch of that class alone
through ``qt_batch_run`` with each candidate tile size (blocks per queue entry;
a warp takes one entry at a time) and keeps the fastest; the measured time per
block becomes the class's cost, which orders the queue heaviest-first. Levels
not measured take the cost and tile of the nearest measured level. Finally it
picks the persistent grid on a mixed batch: threads per CTA (32, 64, 128)
jointly with CTAs per SM. The result is the JSON table ``Batch`` and the
serving loop load by default (``data/batch_tuning.json``).

The kernel maps one 4x4 block to one thread, so two knobs of a sub-warp
mapping have no counterpart here: each thread stages exactly its own block's
16 texels in shared memory (a staging depth of one block per thread, fixed by
the mapping), and each thread reads the cluster-fit ordering table row it
needs straight from L1/L2 (there is no cooperative chunk of the table to size).

    python -m quicktex_b200.autotune [--out PATH] [--quick]
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from .batch import Arena, Batch, Job, TUNING_PATH

# The tuner runs in the source tree: its inputs are the seeded workload textures of
# workloads.py at the repository root (the generator the benchmark uses too).
_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)
import workloads as synth  # noqa: E402

TILES = (32, 64, 128, 256, 512, 1024, 2048, 4096)
THREADS = (32, 64, 128)  # threads per CTA of the persistent kernel
LEVELS = (0, 5, 10, 18)


def _time(batch: Batch, arena: Arena, reps: int = 3) -> float:
    import torch

    s = torch.cuda.current_stream()
    items = arena.items()
    batch.run(items, s.cuda_stream)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        batch.run(items, s.cuda_stream)
        b.record(s)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _class_jobs(op: int, fmt: str, level: int, budget_blocks: int, rng) -> list[Job]:
    """Textures of mixed sizes (log-uniform 16..1024 sides) of one class, about budget_blocks in total."""
    pool = synth.alpha_mix(1024, 1024, workload=6, stream=1) if fmt == "bc3" else synth.block_mix(1024, 1024, workload=6, stream=2)
    jobs, blocks = [], 0
    while blocks < budget_blocks:
        w = int(np.exp(rng.uniform(np.log(16), np.log(1024))))
        h = int(np.exp(rng.uniform(np.log(16), np.log(1024))))
        img = np.ascontiguousarray(pool[:h, :w])
        if op == 0:
            j = Job.encode(fmt, img, w, h, level=level, channel=0, chan0=0, chan1=1)
        else:
            nb = ((w + 3) // 4) * ((h + 3) // 4) * (16 if fmt in ("bc3", "bc5") else 8)
            j = Job.decode(fmt, rng.integers(0, 256, nb, dtype=np.uint8), w, h, channel=0, chan0=0, chan1=1)
        jobs.append(j)
        blocks += j.nblocks
    return jobs


def tune(device: int = 0, quick: bool = False) -> dict:
    import torch

    torch.cuda.set_device(device)
    rng = np.random.default_rng(0xB200)
    tiles = TILES[1:6] if quick else TILES
    measured = []
    classes = [(0, f, L) for f in ("bc1", "bc3") for L in LEVELS] + [(0, f, -1) for f in ("bc4", "bc5")] + \
              [(1, f, -1) for f in ("bc1", "bc3", "bc4", "bc5")]
    fmt_id = {"bc1": 1, "bc3": 3, "bc4": 4, "bc5": 5}
    batch = Batch(device, use_default_tuning=False)
    for op, fmt, level in classes:
        budget = 60_000 if level == 18 else 250_000 if level == 10 else 1_000_000
        if quick:
            budget //= 4
        arena = Arena(_class_jobs(op, fmt, max(level, 0), budget, rng), device)
        arena.upload()
        nblocks = sum(j.nblocks for j in arena.jobs)
        best = None
        for t in tiles:
            batch.set_rules([{"op": op, "format": fmt_id[fmt], "level": level, "tile_blocks": t, "cost_per_block": 1.0}])
            ms = _time(batch, arena)
            if best is None or ms < best[1]:
                best = (t, ms)
        measured.append({"op": op, "format": fmt_id[fmt], "level": level, "tile_blocks": best[0],
                         "us_per_kblock": best[1] * 1e3 / (nblocks / 1e3)})
        del arena
    # costs relative to the cheapest class
    base = min(m["us_per_kblock"] for m in measured)
    rules = []
    for m in measured:
        if m["level"] < 0:
            rules.append({"op": m["op"], "format": m["format"], "level": -1, "tile_blocks": m["tile_blocks"],
                          "cost_per_block": m["us_per_kblock"] / base})
    for fmt in (1, 3):
        ms = {m["level"]: m for m in measured if m["format"] == fmt and m["op"] == 0 and m["level"] >= 0}
        for L in range(20):
            near = min(ms, key=lambda x: (abs(x - L), -x))
            rules.append({"op": 0, "format": fmt, "level": L, "tile_blocks": ms[near]["tile_blocks"],
                          "cost_per_block": ms[near]["us_per_kblock"] / base})
    # persistent grid on a mixed batch: threads per CTA x resident warps per SM (4 to 16; the
    # kernel's registers allow 16)
    items = synth.mixed_batch(300 if quick else 1500, workload=7)
    pools = synth.MixedBatchPools(workload=7, side=2048)
    mixed = Arena([Job.encode(i.fmt, pools.texture(i), i.width, i.height, level=i.level, channel=0) for i in items], device)
    mixed.upload()
    batch.set_rules(rules)
    grid = {}
    for threads in THREADS:
        batch.set_threads(threads)
        for warps in (4, 8, 12, 16):
            k = warps * 32 // threads
            batch.set_grid(k)
            grid[f"{threads}x{k}"] = _time(batch, mixed)
    best = min(grid, key=grid.get)
    best_threads, best_k = (int(x) for x in best.split("x"))
    batch.close()
    return {"device": torch.cuda.get_device_name(device), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "threads_per_cta": best_threads, "ctas_per_sm": best_k, "grid_ms": grid, "measured": measured,
            "rules": rules}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TUNING_PATH)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    t = tune(args.device, args.quick)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(t, f, indent=1)
    print(json.dumps({k: t[k] for k in ("device", "threads_per_cta", "ctas_per_sm", "grid_ms")}))
    for m in t["measured"]:
        print(m)


if __name__ == "__main__":
    main()
