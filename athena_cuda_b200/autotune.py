"""Autotuner for the batched ensemble.

Tunable, all without changing a single result bit:

* the predictor's y-sweep march segment length `ly` (rows a thread walks up
  a column), per size class (the column length Nx2).  Short segments expose
  more parallelism but recompute one PLM cell per segment; long segments do
  less work with fewer threads;
* the threads per work unit of the phased launches (64, 128 or 256: the
  block size of every phase, which also sets the predictor's role-X rows per
  block, its role-Y columns per block and the register budget per thread).
  It is one value for the whole batch, chosen jointly with the `ly` table.

In a batch the GPU is saturated by many instances, so the right choice is
the one that maximises throughput when the GPU is full -- which is what this
tuner measures: for each size class and thread count, a batch of identical
blast instances holding ~4M cells is timed for a few launches with each `ly`
candidate (CUDA events on the batch's stream).  The thread count that
minimises the estimated time of the actual batch (each instance's cells
times its class's best time per cell) wins, with its classes' best `ly`.
Results are cached in JSON.
"""
from __future__ import annotations

import json
from pathlib import Path

LY_CANDIDATES = (2, 4, 8, 16, 32, 64)
NT_CANDIDATES = (64, 128, 256)
TARGET_CELLS = 4_000_000


def size_class(nx1: int, nx2: int, mode: int = 0, nt: int = 128) -> str:
    return f"{nx2}" if mode == 0 else f"{nx2}/phased/{nt}"


def tune_class(nx2: int, nx1: int = 256, launches: int = 3, candidates=LY_CANDIDATES,
               mode: int = 0, nt: int = 128) -> tuple[int, dict]:
    """Fastest segment length for columns of nx2 cells in a saturated batch
    run in execution mode `mode` (Batch.PERSISTENT or Batch.PHASED) with nt
    threads per unit; returns (ly, {ly: ms per launch})."""
    return _tune(nx2, nx1, launches, candidates, mode, nt)[:2]


def _tune(nx2, nx1, launches, candidates, mode, nt):
    import torch

    from . import Batch, Params, configs, problem_state

    blocks = configs.blast(nx1, nx2, tlim=10.0)
    p = Params.from_blocks(blocks)
    cfg = p.config()
    planes = problem_state("blast", p)
    k = max(1, TARGET_CELLS // (nx1 * nx2))
    b = Batch([cfg] * k)
    b.mode = mode
    if mode == Batch.PHASED:
        b.threads = nt
    for i in range(k):
        b.upload(i, planes)
    b.prepare()
    stream = torch.cuda.ExternalStream(b.stream)
    times = {}
    b.run_async(1)  # warm-up (graph instantiation)
    for ly in candidates:
        if ly > nx2 + 3:
            continue
        for i in range(k):
            b.set_ly(i, ly)
        b.commit()
        b.run_async(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run_async(launches)
        e1.record(stream)
        e1.synchronize()
        times[ly] = e0.elapsed_time(e1) / launches
    b.synchronize()
    b.close()
    best = min(times, key=times.get)
    return best, times, times[best] / (k * nx1 * nx2)


def tune_batch(batch, cfg_sizes: list[tuple[int, int]], cache: Path | None = None) -> dict:
    """Set every instance's segment length from its class's tuned value and,
    in the phased mode, the batch's threads per unit (tuning classes not in
    the cache); return the table ({class: ly}, and "threads")."""
    from . import Batch

    table = {}
    if cache and Path(cache).exists():
        table = json.loads(Path(cache).read_text())
    mode = batch.mode
    classes = sorted(set(nx2 for _, nx2 in cfg_sizes))
    nts = NT_CANDIDATES if mode == Batch.PHASED else (128,)
    cost = {}
    for nt in nts:
        total = 0.0
        for nx2 in classes:
            key = size_class(0, nx2, mode, nt)
            entry = table.get(key)
            if not (isinstance(entry, list) and len(entry) == 2):
                ly, _, per_cell = _tune(nx2, 256, 3, LY_CANDIDATES, mode, nt)
                table[key] = entry = [ly, per_cell]
            cells = sum(a * b for a, b in cfg_sizes if b == nx2)
            total += cells * entry[1]
        cost[nt] = total
    nt = min(cost, key=cost.get)
    if mode == Batch.PHASED:
        batch.threads = nt
    for k, (nx1, nx2) in enumerate(cfg_sizes):
        batch.set_ly(k, int(table[size_class(nx1, nx2, mode, nt)][0]))
    batch.commit()
    if cache:
        Path(cache).write_text(json.dumps(table, indent=1, sort_keys=True))
    out = {size_class(0, nx2, mode, nt): table[size_class(0, nx2, mode, nt)][0] for nx2 in classes}
    out["threads"] = nt
    out["estimated_ms_per_launch_by_threads"] = {str(t): c for t, c in cost.items()}
    return out
