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
bit.  Three transports carry the rows and the maximum (the reference itself
has no multi-process grid, ``MPI_SERIAL``):

* ``host``: rows through host memory over ``torch.distributed`` (gloo, or any
  backend that takes CPU tensors), the maximum as a CPU all-reduce;
* ``nccl``: ranks on distinct GPUs; the rows packed on the GPU into device
  buffers (``athb_rows_pack``), sent and received by NCCL on the grid's
  stream and unpacked on the GPU, the maximum all-reduced by NCCL on a device
  word (``athb_max_dti_bits_device`` / ``athb_finish_step_device``): no host
  copy and no host synchronisation per iteration;
* ``ipc``: ranks sharing a GPU (or peers): every rank's receive buffers and
  maximum words live in one device allocation mapped by the other ranks
  through CUDA IPC; a rank packs its rows and copies them with
  ``cudaMemcpyAsync`` into its neighbours' receive buffers, writes its
  maximum into rank 0's words, and two host barriers per iteration order the
  copies (the buffers alternate between two parities, so a copy never lands
  in a buffer its owner is still unpacking).
"""
from __future__ import annotations

import ctypes as C
import time

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
        ("athb_rows_pack", I, [P, I, I, P]),
        ("athb_rows_unpack", I, [P, I, I, P]),
        ("athb_max_dti_bits_device", I, [P, P]),
        ("athb_finish_step_device", I, [P, P, I, I]),
        ("athb_device_alloc", P, [P, C.c_ulonglong]),
        ("athb_device_free", None, [P, P]),
        ("athb_ipc_handle", I, [P, P, C.c_char_p]),
        ("athb_ipc_open", I, [P, C.c_char_p, C.POINTER(C.c_void_p)]),
        ("athb_ipc_close", I, [P, P]),
        ("athb_copy_async", I, [P, P, P, C.c_ulonglong]),
    ]:
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _sigs_done = True


MAX_RANKS = 64          # words of the ipc maximum board per parity
BOARD_BYTES = 2 * MAX_RANKS * 8


class SlabGrid:
    """This rank's slab of a grid given by athinput blocks; the process group
    must be initialised: for transport "host" any backend that reduces and
    sends CPU tensors, for "nccl" an NCCL group (one GPU per rank), for "ipc"
    a group that gathers objects and has a barrier (gloo)."""

    TRANSPORTS = ("host", "nccl", "ipc")

    def __init__(self, blocks: dict, problem: str, rank: int, ranks: int, group=None, transport: str = "host"):
        import torch.distributed as dist

        _sigs()
        if transport not in self.TRANSPORTS:
            raise ValueError(f"transport must be one of {self.TRANSPORTS}")
        if transport == "ipc" and ranks > MAX_RANKS:
            raise ValueError(f"ipc transport: at most {MAX_RANKS} ranks")
        self.transport = transport
        self.exchange_s = 0.0    # host time spent in the exchange and the maximum
        self.iterations = 0
        self.parity = 0          # ipc receive buffers in use (alternate per exchange)
        self.bpar = 0            # ipc maximum board in use (alternate per step finish)
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
        self.row_doubles = len(PLANES) * NG * self.sx
        if transport == "nccl":
            self._nccl_setup(gcfg.device)
        elif transport == "ipc":
            self._ipc_setup()
        self._ghosts()
        _check(lib().athb_cfl_local(self.grid._h))
        self._finish(0)

    # -- transports ----------------------------------------------------------
    def _nccl_setup(self, device: int) -> None:
        import torch

        dev = torch.device("cuda", device)
        self.tdev = dev
        self.stream = torch.cuda.ExternalStream(self.grid.stream, device=dev)
        self.dti = torch.zeros(1, dtype=torch.int64, device=dev)
        self.sendbuf = {s: torch.empty(self.row_doubles, dtype=torch.float64, device=dev) for s in ("lo", "hi")}
        self.recvbuf = {s: torch.empty(self.row_doubles, dtype=torch.float64, device=dev) for s in ("lo", "hi")}

    def _ipc_setup(self) -> None:
        L, h = lib(), self.grid._h
        rb = self.row_doubles * 8
        # one allocation per rank: the maximum board, then receive buffers
        # [parity][side] (side 0: rows from the rank below -> my lower
        # ghosts; side 1: rows from the rank above -> my upper ghosts)
        self.own = L.athb_device_alloc(h, BOARD_BYTES + 4 * rb)
        self.send = L.athb_device_alloc(h, 2 * rb)
        if not self.own or not self.send:
            raise RuntimeError("athb_device_alloc failed")
        handle = C.create_string_buffer(64)
        _check(L.athb_ipc_handle(h, C.c_void_p(self.own), handle))
        handles = [None] * self.ranks
        self.dist.all_gather_object(handles, bytes(handle.raw), group=self.group)
        self.peer = {self.rank: self.own}
        for r in {self.below, self.above, 0} - {None, self.rank}:
            ptr = C.c_void_p()
            _check(L.athb_ipc_open(h, handles[r], C.byref(ptr)))
            self.peer[r] = ptr.value
        self.rb = rb

    def _recv_addr(self, r: int, parity: int, side: int) -> int:
        return self.peer[r] + BOARD_BYTES + (2 * parity + side) * self.rb

    def _barrier(self) -> None:
        self.dist.barrier(group=self.group)

    def _finish(self, after_step: int) -> None:
        """The maximum of 1/dt over the ranks, then the dt rule (and the
        time advance after a step) on every rank."""
        t0 = time.perf_counter()
        L, h = lib(), self.grid._h
        if self.transport == "host":
            _check(L.athb_finish_step(h, self._global_max(), after_step))
        elif self.transport == "nccl":
            import torch

            _check(L.athb_max_dti_bits_device(h, C.c_void_p(self.dti.data_ptr())))
            with torch.cuda.stream(self.stream):
                if self.ranks > 1:
                    self.dist.all_reduce(self.dti, op=self.dist.ReduceOp.MAX, group=self.group)
                _check(L.athb_finish_step_device(h, C.c_void_p(self.dti.data_ptr()), 1, after_step))
        else:
            # the board alternates between two parities per call: a rank
            # writes parity q only after every rank has passed the barrier of
            # the previous call, which each enters after its read of parity q
            # two calls back has completed
            board = self.peer[0] + self.bpar * MAX_RANKS * 8
            self.bpar ^= 1
            _check(L.athb_max_dti_bits_device(h, C.c_void_p(board + 8 * self.rank)))
            self.grid.synchronize()
            self._barrier()   # every rank's word is on rank 0's board
            _check(L.athb_finish_step_device(h, C.c_void_p(board), self.ranks, after_step))
        self.exchange_s += time.perf_counter() - t0

    def _exchange_device(self) -> None:
        L, h = lib(), self.grid._h
        js, je = NG, NG + self.ny - 1
        if self.transport == "nccl":
            import torch

            if self.below is not None:
                _check(L.athb_rows_pack(h, js, NG, C.c_void_p(self.sendbuf["lo"].data_ptr())))
            if self.above is not None:
                _check(L.athb_rows_pack(h, je - NG + 1, NG, C.c_void_p(self.sendbuf["hi"].data_ptr())))
            with torch.cuda.stream(self.stream):
                ops = []
                if self.below is not None:
                    ops.append(self.dist.P2POp(self.dist.isend, self.sendbuf["lo"], self.below, group=self.group))
                    ops.append(self.dist.P2POp(self.dist.irecv, self.recvbuf["lo"], self.below, group=self.group))
                if self.above is not None:
                    ops.append(self.dist.P2POp(self.dist.isend, self.sendbuf["hi"], self.above, group=self.group))
                    ops.append(self.dist.P2POp(self.dist.irecv, self.recvbuf["hi"], self.above, group=self.group))
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()   # the grid's stream waits for the transfers
            if self.below is not None:
                _check(L.athb_rows_unpack(h, js - NG, NG, C.c_void_p(self.recvbuf["lo"].data_ptr())))
            if self.above is not None:
                _check(L.athb_rows_unpack(h, je + 1, NG, C.c_void_p(self.recvbuf["hi"].data_ptr())))
            return
        # ipc: my lowest rows become the upper ghosts of the rank below (its
        # side 1), my highest rows the lower ghosts of the rank above (its
        # side 0)
        q = self.parity
        if self.below is not None:
            _check(L.athb_rows_pack(h, js, NG, C.c_void_p(self.send)))
            _check(L.athb_copy_async(h, C.c_void_p(self._recv_addr(self.below, q, 1)), C.c_void_p(self.send),
                                     self.rb))
        if self.above is not None:
            _check(L.athb_rows_pack(h, je - NG + 1, NG, C.c_void_p(self.send + self.rb)))
            _check(L.athb_copy_async(h, C.c_void_p(self._recv_addr(self.above, q, 0)), C.c_void_p(self.send + self.rb),
                                     self.rb))
        self.grid.synchronize()
        self._barrier()   # every copy into my receive buffers has landed
        if self.below is not None:
            _check(L.athb_rows_unpack(h, js - NG, NG, C.c_void_p(self._recv_addr(self.rank, q, 0))))
        if self.above is not None:
            _check(L.athb_rows_unpack(h, je + 1, NG, C.c_void_p(self._recv_addr(self.rank, q, 1))))

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
        t0 = time.perf_counter()
        if self.ranks > 1:
            if self.transport == "host":
                self._exchange()
            else:
                self._exchange_device()
        self.exchange_s += time.perf_counter() - t0
        if self.sides2:
            _check(lib().athb_ghost_fill(self.grid._h, 2, self.sides2))
        self.parity ^= 1   # the next exchange lands in the other buffers

    # -- public ------------------------------------------------------------
    def step(self) -> None:
        """One iteration of the main loop on every rank (collective)."""
        _check(lib().athb_integrate_local(self.grid._h))
        self._finish(1)
        self._ghosts()
        self.iterations += 1

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
        """Release the transport's buffers (collective for "ipc": no rank
        frees a buffer another may still write), then the grid."""
        if self.transport == "ipc" and getattr(self, "own", None):
            L, h = lib(), self.grid._h
            self.grid.synchronize()
            self._barrier()
            for r, ptr in self.peer.items():
                if r != self.rank:
                    _check(L.athb_ipc_close(h, C.c_void_p(ptr)))
            self._barrier()
            L.athb_device_free(h, C.c_void_p(self.own))
            L.athb_device_free(h, C.c_void_p(self.send))
            self.own = None
        self.grid.close()
