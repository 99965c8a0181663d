"""A grid split over processes as x2 slabs (athena_cuda_b200/decomp.py) gives
the single grid's state bit for bit: 2 and 3 ranks, periodic, outflow and
reflecting x2 boundaries.  The ranks share this one GPU and exchange rows
through host memory (transport "host", gloo) or through device buffers
(transport "ipc": rows packed on the GPU and copied with cudaMemcpyAsync into
the neighbours' CUDA-IPC-mapped receive buffers, the 1/dt maximum over device
words); host barriers order the copies, so no kernel waits on another rank.
The exchange time per iteration is printed."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
CASES = {
    "loop_periodic_2": ("field_loop", dict(nx1=48, nx2=36), 2, 20),
    "blast_outflow_reflect_3": ("blast", dict(nx1=40, nx2=60, bc=(2, 2, 1, 2)), 3, 25),
    "blast_periodic_3": ("blast", dict(nx1=30, nx2=45), 3, 25),
}


def _blocks(problem, kw):
    sys.path.insert(0, str(ROOT))
    from athena_cuda_b200 import configs

    return configs.field_loop(**kw) if problem == "field_loop" else configs.blast(**kw)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ranks, port, name, transport, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from athena_cuda_b200.decomp import SlabGrid

    problem, kw, _, steps = CASES[name]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ranks, timeout=datetime.timedelta(seconds=120))
    try:
        s = SlabGrid(_blocks(problem, kw), problem, rank, ranks, transport=transport)
        s.run(steps)
        per_iter_ms = 1e3 * s.exchange_s / max(1, s.iterations)
        full = s.gather()
        st = s.status()
        s.close()
        if rank == 0:
            q.put((full, st["dt"], st["time"], st["nstep"], per_iter_ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("transport", ["host", "ipc"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_slabs_equal_single_grid(name, transport):
    from athena_cuda_b200 import Grid, Params

    problem, kw, ranks, steps = CASES[name]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ranks, port, name, transport, q)) for r in range(ranks)]
    for p in procs:
        p.start()
    full, dt, t, n, per_iter_ms = q.get(timeout=300)
    print(f"{name} {transport}: exchange + maximum {per_iter_ms:.3f} ms per iteration")
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    blocks = _blocks(problem, kw)
    p = Params.from_blocks(blocks)
    from athena_cuda_b200 import problem_state

    g = Grid.create(p.config())
    g.upload(problem_state(problem, p))
    g.set_bvals()
    g.new_dt()
    g.run(steps)
    planes, dt1, t1, n1 = g.download()
    g.close()
    want = planes[:, 4:-4, 4:-4]
    assert np.array_equal(full, want), f"{int(np.sum(full != want))} values differ"
    assert (dt, t, n) == (dt1, t1, n1)
