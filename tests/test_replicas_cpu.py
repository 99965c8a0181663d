"""Multi-GPU runs are replicas (independent grids, no data-path exchange):
bench.py times each rank on its own device and reduces with the maximum over
ranks.  The reduction and the whole-job value are checked here on CPU with
two gloo ranks."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, ws: int, port: int, q) -> None:
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        mine = [3.25, 4.5][rank]  # this rank's device ms for the timed steps
        worst = bench.max_over_ranks(mine, ws, "cpu")
        q.put((rank, worst, bench.replica_value(ws, 2048 * 2048, worst / 400)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [4.5, 4.5]
    assert got[0][2] == got[1][2] == 2 * 2048 * 2048 / (4.5 / 400 * 1e-3)
