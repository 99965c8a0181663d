"""Autotuner for the batched ensemble: picks, per grid-size class, the y-sweep
march segment length (rows per thread of the predictor's y role) and, for the
whole batch, the number of persistent blocks.  Candidates are timed on the
GPU with CUDA events; every candidate gives bit-identical results, so only
speed is compared.  Results can be cached in a JSON file.
"""
from __future__ import annotations

import json
import tempfile
from pathlib import Path

from . import Batch, Grid, Params, configs, problem_state, write_athinput

LY_CANDIDATES = (2, 4, 8, 16, 32, 64)


def size_class(nx1: int, nx2: int) -> str:
    return f"{nx1}x{nx2}"


def tune_ly(nx1: int, nx2: int, steps: int = 6) -> tuple[int, dict]:
    """Fastest predictor segment length for an nx1 x nx2 blast grid."""
    with tempfile.TemporaryDirectory() as td:
        ath = write_athinput(Path(td) / "a", configs.blast(nx1, nx2, tlim=10.0))
        g = Grid.from_athinput(ath, "blast")
        g.run(2)
        times = {}
        for ly in LY_CANDIDATES:
            if ly > nx2 + 3:
                continue
            g.ly = ly
            times[ly] = g.profile(steps)["predict"]
        g.close()
    best = min(times, key=times.get)
    return best, times


def tune_batch(batch: Batch, cfg_sizes: list[tuple[int, int]], cache: Path | None = None,
               grid_candidates=None, steps: int = 4) -> dict:
    """Apply per-size-class segment lengths and the fastest persistent grid
    to `batch` (sizes listed per instance).  The batch is advanced by the
    grid trials; call this on a throw-away batch or before `prepare` state is
    needed again."""
    table = {}
    if cache and Path(cache).exists():
        table = json.loads(Path(cache).read_text())
    for nx1, nx2 in sorted(set(cfg_sizes)):
        key = size_class(nx1, nx2)
        if key not in table:
            table[key] = tune_ly(nx1, nx2)[0]
    for k, (nx1, nx2) in enumerate(cfg_sizes):
        batch.set_ly(k, int(table[size_class(nx1, nx2)]))
    batch.commit()
    if cache:
        Path(cache).write_text(json.dumps(table, indent=1, sort_keys=True))
    return table
