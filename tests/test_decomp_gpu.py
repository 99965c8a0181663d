"""A grid split over processes as x2 slabs or px x py blocks
(athena_cuda_b200/decomp.py) gives the single grid's state bit for bit: 2, 3,
4 and 6 ranks, periodic, outflow, reflecting and mixed boundaries.  The ranks share this one GPU and exchange rows
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
CASES = {   # name: (problem, grid, px, py, steps)
    "loop_periodic_2": ("field_loop", dict(nx1=48, nx2=36), 1, 2, 20),
    "blast_outflow_reflect_3": ("blast", dict(nx1=40, nx2=60, bc=(2, 2, 1, 2)), 1, 3, 25),
    "blast_periodic_3": ("blast", dict(nx1=30, nx2=45), 1, 3, 25),
}
# 2D blocks (ipc transport): periodic both ways, mixed physical boundaries,
# uneven splits, a 2 x 1 row of blocks
BLOCK_CASES = {
    "loop_periodic_2x2": ("field_loop", dict(nx1=40, nx2=36), 2, 2, 20),
    "blast_mixed_3x2": ("blast", dict(nx1=45, nx2=34, bc=(1, 2, 2, 1)), 3, 2, 25),
    "blast_periodic_2x1": ("blast", dict(nx1=38, nx2=30), 2, 1, 25),
    "blast_reflect_1x2_ipc": ("blast", dict(nx1=30, nx2=41, bc=(1, 1, 1, 1)), 1, 2, 25),
    "blast_hlle_2x2": ("blast", dict(nx1=64, nx2=48, bc=(2, 2, 4, 4), flux="hlle"), 2, 2, 30),
    "loop_128x96_2x2": ("field_loop", dict(nx1=128, nx2=96), 2, 2, 40),
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
    return _run_rank(rank, ranks, port, {**CASES, **BLOCK_CASES, **NCCL_CASES}[name], transport, q)


def _run_rank(rank, ranks, port, case, transport, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from athena_cuda_b200.decomp import BlockGrid, SlabGrid

    problem, kw, px, py, steps = case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    if transport == "nccl":
        import torch

        torch.cuda.set_device(0)
    dist.init_process_group("nccl" if transport == "nccl" else "gloo", rank=rank, world_size=ranks,
                            timeout=datetime.timedelta(seconds=120))
    try:
        if px == 1 and transport == "host":
            s = SlabGrid(_blocks(problem, kw), problem, rank, ranks, transport=transport)
        else:
            s = BlockGrid(_blocks(problem, kw), problem, rank, px, py, transport=transport)
        s.run(steps)
        per_iter_ms = 1e3 * s.exchange_s / max(1, s.iterations)
        full = s.gather()
        st = s.status()
        s.close()
        if rank == 0:
            q.put((full, st["dt"], st["time"], st["nstep"], per_iter_ms))
    finally:
        dist.destroy_process_group()


# the NCCL transport needs one GPU per rank; on one GPU it runs as one rank,
# which exercises its device maximum (a device word all-reduced by NCCL on the
# grid's stream) but no exchange
NCCL_CASES = {"loop_nccl_1": ("field_loop", dict(nx1=40, nx2=36), 1, 1, 15)}


@pytest.mark.parametrize("name,transport", [(n, t) for n in sorted(CASES) for t in ("host", "ipc")]
                         + [(n, "ipc") for n in sorted(BLOCK_CASES)] + [(n, "nccl") for n in NCCL_CASES])
def test_slabs_equal_single_grid(name, transport):
    from athena_cuda_b200 import Grid, Params

    problem, kw, px, py, steps = {**CASES, **BLOCK_CASES, **NCCL_CASES}[name]
    ranks = px * py
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
