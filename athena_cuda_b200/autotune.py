"""Autotuner for the batched ensemble.

Tunable: the predictor's y-sweep march segment length `ly` (rows a thread
walks up a column).  Short segments expose more parallelism but recompute one
PLM cell per segment; long segments do less work but fewer threads.  In a
batch the GPU is saturated by many instances, so the right choice is the one
that maximises throughput when the GPU is full -- which is what this tuner
measures: for each column-length class (Nx2), a batch of identical blast
instances holding ~4M cells is timed for a few persistent launches with each
candidate, CUDA events on the batch's stream.  All candidates give
bit-identical results; only speed differs.  Results are cached in JSON.
"""
from __future__ import annotations

import json
from pathlib import Path

LY_CANDIDATES = (2, 4, 8, 16, 32, 64)
TARGET_CELLS = 4_000_000


def size_class(nx1: int, nx2: int, mode: int = 0) -> str:
    return f"{nx2}" if mode == 0 else f"{nx2}/phased"


def tune_class(nx2: int, nx1: int = 256, launches: int = 3, candidates=LY_CANDIDATES,
               mode: int = 0) -> tuple[int, dict]:
    """Fastest segment length for columns of nx2 cells in a saturated batch
    run in execution mode `mode` (Batch.PERSISTENT or Batch.PHASED)."""
    import torch

    from . import Batch, Params, configs, problem_state

    blocks = configs.blast(nx1, nx2, tlim=10.0)
    p = Params.from_blocks(blocks)
    cfg = p.config()
    planes = problem_state("blast", p)
    k = max(1, TARGET_CELLS // (nx1 * nx2))
    b = Batch([cfg] * k)
    b.mode = mode
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
    return min(times, key=times.get), times


def tune_batch(batch, cfg_sizes: list[tuple[int, int]], cache: Path | None = None) -> dict:
    """Set every instance's segment length from its class's tuned value
    (tuning classes not in the cache) and return the table."""
    table = {}
    if cache and Path(cache).exists():
        table = json.loads(Path(cache).read_text())
    mode = batch.mode
    for nx1, nx2 in sorted(set(cfg_sizes)):
        key = size_class(nx1, nx2, mode)
        if key not in table:
            table[key] = tune_class(nx2, mode=mode)[0]
    for k, (nx1, nx2) in enumerate(cfg_sizes):
        batch.set_ly(k, int(table[size_class(nx1, nx2, mode)]))
    batch.commit()
    if cache:
        Path(cache).write_text(json.dumps(table, indent=1, sort_keys=True))
    return table
