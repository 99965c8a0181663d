"""One grid split over several processes (one GPU each) as slabs along x2.

Each rank holds rows [j0, j0 + ny) of the global Nx1 x Nx2 interior with the
global cell sizes, and runs every main-loop iteration (src/main.c:229-307) as

1. the step of its interior (``athb_integrate_local``);
2. a max over the ranks of the CFL rate 1/dt (``athb_max_dti_bits``; the
   bits of positive doubles order like the doubles, so an integer max is
   exact), then the dt rule and the time advance (``athb_finish_step``) --
   every rank gets the dt of the single grid;
3. the x1 ghost columns on its own rows (``athb_ghost_fill`` mode 1);
4. the exchange of 4 full rows of all 11 planes with the neighbours below and
   above (x1 ghosts included, as the reference's x2 boundaries copy whole
   rows after the x1 boundaries, src/set_bvals.c:114-145), ring-wise for a
   periodic x2 boundary;
5. the physical x2 boundaries at the global ends (mode 2, one side).

So every rank's state equals the matching rows of the single grid bit for
bit.  The rows travel through host memory over ``torch.distributed`` (gloo,
or any backend that takes CPU tensors), one exchange per iteration; the
reference itself has no multi-process grid (``MPI_SERIAL``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import PLANES, Config, Grid, Params, _check, lib, problem_state

NG = 4  # ghost rows exchanged per side (nghost)


def slab_rows(nx2: int, ranks: int) -> list[tuple[int, int]]:
    """(first interior row, rows) of each rank: as even as possible, the
    first nx2 % ranks ranks one row more."""
    if ranks < 1 or nx2 < ranks * NG:
        raise ValueError(f"{nx2} rows cannot be split into {ranks} slabs of at least {NG} rows")
    base, extra = divmod(nx2, ranks)
    out, j0 = [], 0
    for r in range(ranks):
        n = base + (1 if r < extra else 0)
        out.append((j0, n))
        j0 += n
    return out


def neighbours(rank: int, ranks: int, periodic: bool) -> tuple[int | None, int | None]:
    """Ranks holding the rows below and above (None at a non-periodic end)."""
    below = rank - 1 if rank > 0 else (ranks - 1 if periodic and ranks > 1 else None)
    above = rank + 1 if rank < ranks - 1 else (0 if periodic and ranks > 1 else None)
    return below, above


def x2_sides(rank: int, ranks: int, periodic: bool) -> int:
    """Sides (bit 0 inner, bit 1 outer) whose x2 ghosts this rank fills from
    its own rows with the physical boundary condition."""
    if periodic and ranks > 1:
        return 0
    return (1 if rank == 0 else 0) | (2 if rank == ranks - 1 else 0)


_sigs_done = False


def _sigs():
    global _sigs_done
    if _sigs_done:
        return
    L, P, I, D = lib(), C.c_void_p, C.c_int, C.c_double
    u64p, dp = C.POINTER(C.c_ulonglong), C.POINTER(C.c_double)
    for name, res, args in [
        ("athb_set_geometry", I, [P, D, D, D, D]),
        ("athb_integrate_local", I, [P]),
        ("athb_cfl_local", I, [P]),
        ("athb_max_dti_bits", I, [P, u64p]),
        ("athb_finish_step", I, [P, C.c_ulonglong, I]),
        ("athb_ghost_fill", I, [P, I, I]),
        ("athb_rows_get", I, [P, I, I, dp]),
        ("athb_rows_put", I, [P, I, I, dp]),
    ]:
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _sigs_done = True


class SlabGrid:
    """This rank's slab of a grid given by athinput blocks; the process group
    must be initialised (any backend that reduces and sends CPU tensors)."""

    def __init__(self, blocks: dict, problem: str, rank: int, ranks: int, group=None):
        import torch.distributed as dist

        _sigs()
        self.dist, self.group, self.rank, self.ranks = dist, group, rank, ranks
        params = Params.from_blocks(blocks)
        gcfg = params.config()
        self.nx1, self.nx2 = gcfg.nx1, gcfg.nx2
        self.slabs = slab_rows(gcfg.nx2, ranks)
        self.j0, self.ny = self.slabs[rank]
        self.periodic = gcfg.bc_ix2 == 4 and gcfg.bc_ox2 == 4
        self.below, self.above = neighbours(rank, ranks, self.periodic)
        self.sides2 = x2_sides(rank, ranks, self.periodic)
        dx1 = (gcfg.x1max - gcfg.x1min) / gcfg.nx1  # src/init_grid.c
        dx2 = (gcfg.x2max - gcfg.x2min) / gcfg.nx2
        cfg = Config.from_buffer_copy(gcfg)
        cfg.nx2 = self.ny
        cfg.x2min = gcfg.x2min + self.j0 * dx2
        cfg.x2max = gcfg.x2min + (self.j0 + self.ny) * dx2
        self.grid = Grid.create(cfg)
        _check(lib().athb_set_geometry(self.grid._h, dx1, dx2, gcfg.x1min, cfg.x2min))
        self.sx = self.nx1 + 2 * NG
        # initial state: the global generator, this rank's rows (ghost rows
        # are refilled below)
        full = problem_state(problem, params)
        self.grid.upload(np.ascontiguousarray(full[:, self.j0:self.j0 + self.ny + 2 * NG, :]))
        self._ghosts()
        _check(lib().athb_cfl_local(self.grid._h))
        _check(lib().athb_finish_step(self.grid._h, self._global_max(), 0))

    # -- pieces ------------------------------------------------------------
    def _global_max(self) -> int:
        import torch

        bits = C.c_ulonglong()
        _check(lib().athb_max_dti_bits(self.grid._h, C.byref(bits)))
        t = torch.tensor([np.int64(np.uint64(bits.value).view(np.int64))], dtype=torch.int64)
        if self.ranks > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return int(np.int64(t.item()).view(np.uint64))

    def _rows(self, j0: int) -> np.ndarray:
        buf = np.empty((len(PLANES), NG, self.sx))
        _check(lib().athb_rows_get(self.grid._h, j0, NG, buf.ctypes.data_as(C.POINTER(C.c_double))))
        return buf

    def _put(self, j0: int, buf: np.ndarray) -> None:
        buf = np.ascontiguousarray(buf)
        _check(lib().athb_rows_put(self.grid._h, j0, NG, buf.ctypes.data_as(C.POINTER(C.c_double))))

    def _exchange(self) -> None:
        import torch

        if self.ranks == 1:
            return
        js, je = NG, NG + self.ny - 1
        up, down = 0, 1  # tags: rows travelling to the rank above / below
        sends, recvs = [], []
        if self.below is not None:  # my lowest rows become the ghosts above the rank below
            sends.append((self.below, down, torch.from_numpy(self._rows(js))))
            recvs.append((self.below, up, js - NG, torch.empty((len(PLANES), NG, self.sx), dtype=torch.float64)))
        if self.above is not None:  # my highest rows become the ghosts below the rank above
            sends.append((self.above, up, torch.from_numpy(self._rows(je - NG + 1))))
            recvs.append((self.above, down, je + 1, torch.empty((len(PLANES), NG, self.sx), dtype=torch.float64)))
        ops = [self.dist.P2POp(self.dist.isend, t, peer, group=self.group, tag=tag) for peer, tag, t in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer, group=self.group, tag=tag) for peer, tag, _, t in recvs]
        for w in self.dist.batch_isend_irecv(ops):
            w.wait()
        for _, _, j0, t in recvs:
            self._put(j0, t.numpy())

    def _ghosts(self) -> None:
        _check(lib().athb_ghost_fill(self.grid._h, 1, 3))
        self._exchange()
        if self.sides2:
            _check(lib().athb_ghost_fill(self.grid._h, 2, self.sides2))

    # -- public ------------------------------------------------------------
    def step(self) -> None:
        """One iteration of the main loop on every rank (collective)."""
        _check(lib().athb_integrate_local(self.grid._h))
        _check(lib().athb_finish_step(self.grid._h, self._global_max(), 1))
        self._ghosts()

    def status(self) -> dict:
        return self.grid.status()

    def run(self, max_steps: int) -> int:
        """Iterations until tlim / nlim or max_steps (collective)."""
        n = 0
        while n < max_steps and not self.grid.status()["done"]:
            self.step()
            n += 1
        return n

    def gather(self) -> np.ndarray | None:
        """The global interior state (planes x Nx2 x Nx1) on rank 0."""
        import torch

        planes = self.grid.download()[0][:, NG:NG + self.ny, NG:NG + self.nx1]
        mine = torch.from_numpy(np.ascontiguousarray(planes))
        if self.ranks == 1:
            return mine.numpy()
        if self.rank == 0:
            parts = [mine]
            for r in range(1, self.ranks):
                t = torch.empty((len(PLANES), self.slabs[r][1], self.nx1), dtype=torch.float64)
                self.dist.recv(t, src=r, group=self.group)
                parts.append(t)
            return torch.cat(parts, dim=1).numpy()
        self.dist.send(mine, dst=0, group=self.group)
        return None

    def close(self) -> None:
        self.grid.close()
