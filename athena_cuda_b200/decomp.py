"""One grid split over several processes (one GPU each) as px x py blocks.

Rank r holds columns [i0, i0 + nx) x rows [j0, j0 + ny) of the global
Nx1 x Nx2 interior (block (r % px, r // px)) with the global cell sizes, and
runs every main-loop iteration (src/main.c:229-307) as

1. the step of its interior (``athb_integrate_local``);
2. a max over the ranks of the CFL rate 1/dt (the bits of positive doubles
   order like the doubles, so an integer max is exact), then the dt rule and
   the time advance -- every rank gets the dt of the single grid;
3. the x1 ghosts, in the reference's order (src/set_bvals.c:114-145): the
   physical x1 boundary where the block touches the global x1 ends
   (``athb_ghost_fill`` mode 1), and the exchange of 4 columns of all 11
   planes with the blocks left and right, on the block's interior rows plus
   row je+1 (the last interior row of B2i);
4. the x2 ghosts: the exchange of 4 full-width rows (x1 ghosts included, as
   the reference's x2 boundaries copy whole rows after the x1 boundaries)
   with the blocks below and above, then the physical x2 boundary at the
   global x2 ends (mode 2).

Exchanges are ring-wise along a periodic direction.  Faces on a block edge
(B1i at column ie+1, B2i at row je+1) are computed by both neighbours from
the same inputs, so the copy that crosses them carries equal values.  Every
rank's state equals the matching block of the single grid bit for bit.
Three transports carry the ghosts and the maximum (the reference itself has
no multi-process grid, ``MPI_SERIAL``):

* ``host`` (px = 1 only): rows through host memory over
  ``torch.distributed`` (gloo, or any backend that takes CPU tensors), the
  maximum as a CPU all-reduce;
* ``nccl``: ranks on distinct GPUs; the columns or rows packed on the GPU
  into device buffers (``athb_rect_pack``), sent and received by NCCL on the
  grid's stream and unpacked on the GPU, the maximum all-reduced by NCCL on
  a device word (``athb_max_dti_bits_device`` / ``athb_finish_step_device``):
  no host copy and no host synchronisation per iteration;
* ``ipc``: ranks sharing a GPU (or peers): every rank's receive buffers and
  maximum words live in one device allocation mapped by the other ranks
  through CUDA IPC; a rank packs its edges and copies them with
  ``cudaMemcpyAsync`` into its neighbours' receive buffers, writes its
  maximum into rank 0's words, and host barriers order the copies (buffers
  and words alternate between two parities, so a copy never lands in a
  buffer its owner is still reading).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import PLANES, Config, Grid, Params, _check, lib, problem_state

NG = 4  # ghost cells exchanged per side (nghost)


def slab_rows(nx2: int, ranks: int) -> list[tuple[int, int]]:
    """(first interior cell, cells) of each of `ranks` pieces of nx2 cells: as
    even as possible, the first nx2 % ranks pieces one cell more."""
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
    """Pieces before and after along one direction (None at a non-periodic
    end)."""
    below = rank - 1 if rank > 0 else (ranks - 1 if periodic and ranks > 1 else None)
    above = rank + 1 if rank < ranks - 1 else (0 if periodic and ranks > 1 else None)
    return below, above


def x2_sides(rank: int, ranks: int, periodic: bool) -> int:
    """Sides (bit 0 inner, bit 1 outer) whose ghosts along one direction this
    piece fills from its own cells with the physical boundary condition."""
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
        ("athb_rect_pack", I, [P, I, I, I, I, P]),
        ("athb_rect_unpack", I, [P, I, I, I, I, P]),
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


def block_neighbours(rank: int, px: int, py: int, periodic1: bool, periodic2: bool) -> dict:
    """Neighbours of block rank = rx + px * ry: {0: (left, right), 1: (below,
    above)} (None at a non-periodic end), and the sides of each direction it
    fills with the physical boundary condition {"sides1": .., "sides2": ..}."""
    rx, ry = rank % px, rank // px
    lx, hx = neighbours(rx, px, periodic1)
    ly, hy = neighbours(ry, py, periodic2)
    return {0: (None if lx is None else ry * px + lx, None if hx is None else ry * px + hx),
            1: (None if ly is None else ly * px + rx, None if hy is None else hy * px + rx),
            "sides1": x2_sides(rx, px, periodic1), "sides2": x2_sides(ry, py, periodic2)}


MAX_RANKS = 64          # words of the ipc maximum board per parity
BOARD_BYTES = 2 * MAX_RANKS * 8
X1, X2 = 0, 1           # exchange directions


class BlockGrid:
    """This rank's block of a grid given by athinput blocks, split into
    px x py blocks (ranks = px * py).  The process group must be
    initialised: for transport "host" any backend that reduces and sends CPU
    tensors, for "nccl" an NCCL group (one GPU per rank), for "ipc" a group
    that gathers objects and has a barrier (gloo)."""

    TRANSPORTS = ("host", "nccl", "ipc")

    def __init__(self, blocks: dict, problem: str, rank: int, px: int, py: int, group=None,
                 transport: str = "ipc"):
        import torch.distributed as dist

        _sigs()
        ranks = px * py
        if transport not in self.TRANSPORTS:
            raise ValueError(f"transport must be one of {self.TRANSPORTS}")
        if transport == "ipc" and ranks > MAX_RANKS:
            raise ValueError(f"ipc transport: at most {MAX_RANKS} ranks")
        if transport == "host" and px > 1:
            raise ValueError("the host transport exchanges rows only (px = 1)")
        if not 0 <= rank < ranks:
            raise ValueError("rank outside px * py")
        self.transport = transport
        self.exchange_s = 0.0    # host time spent in the exchanges and the maximum
        self.iterations = 0
        self.parity = 0          # ipc receive buffers in use (alternate per exchange)
        self.bpar = 0            # ipc maximum board in use (alternate per step finish)
        self.dist, self.group, self.rank, self.ranks = dist, group, rank, ranks
        self.px, self.py = px, py
        self.rx, self.ry = rank % px, rank // px
        params = Params.from_blocks(blocks)
        gcfg = params.config()
        self.gnx1, self.gnx2 = gcfg.nx1, gcfg.nx2
        self.cols = slab_rows(gcfg.nx1, px)
        self.rows = slab_rows(gcfg.nx2, py)
        self.i0, self.nx = self.cols[self.rx]
        self.j0, self.ny = self.rows[self.ry]
        per1 = gcfg.bc_ix1 == 4 and gcfg.bc_ox1 == 4
        per2 = gcfg.bc_ix2 == 4 and gcfg.bc_ox2 == 4
        # a periodic side needs the far end's cells: only both sides periodic
        # (a ring) or neither can be split
        for n, a, b in ((px, gcfg.bc_ix1, gcfg.bc_ox1), (py, gcfg.bc_ix2, gcfg.bc_ox2)):
            if n > 1 and (a == 4) != (b == 4):
                raise ValueError("a direction split over several ranks is periodic on both sides or on neither")
        nb = block_neighbours(rank, px, py, per1, per2)
        self.nbr = {X1: nb[X1], X2: nb[X2]}   # per direction: (low side, high side) ranks
        self.sides1, self.sides2 = nb["sides1"], nb["sides2"]
        dx1 = (gcfg.x1max - gcfg.x1min) / gcfg.nx1  # src/init_grid.c
        dx2 = (gcfg.x2max - gcfg.x2min) / gcfg.nx2
        cfg = Config.from_buffer_copy(gcfg)
        cfg.nx1, cfg.nx2 = self.nx, self.ny
        cfg.x1min = gcfg.x1min + self.i0 * dx1
        cfg.x1max = gcfg.x1min + (self.i0 + self.nx) * dx1
        cfg.x2min = gcfg.x2min + self.j0 * dx2
        cfg.x2max = gcfg.x2min + (self.j0 + self.ny) * dx2
        self.grid = Grid.create(cfg)
        _check(lib().athb_set_geometry(self.grid._h, dx1, dx2, cfg.x1min, cfg.x2min))
        self.sx = self.nx + 2 * NG
        # initial state: the global generator, this rank's block (ghosts are
        # refilled below)
        full = problem_state(problem, params)
        self.grid.upload(np.ascontiguousarray(full[:, self.j0:self.j0 + self.ny + 2 * NG,
                                                   self.i0:self.i0 + self.nx + 2 * NG]))
        # exchange buffer sizes, the same on every rank (the largest block)
        maxnx = max(n for _, n in self.cols)
        maxny = max(n for _, n in self.rows)
        self.count = {X1: len(PLANES) * NG * (self.ny + 1), X2: len(PLANES) * NG * self.sx}
        self.slot = ((len(PLANES) * NG * max(maxny + 1, maxnx + 2 * NG) * 8 + 255) // 256) * 256
        if transport == "nccl":
            self._nccl_setup(gcfg.device)
        elif transport == "ipc":
            self._ipc_setup()
        self._ghosts()
        _check(lib().athb_cfl_local(self.grid._h))
        self._finish(0)

    # -- geometry of the exchanges ------------------------------------------
    def _edge(self, d: int, high: bool, ghost: bool) -> tuple[int, int, int, int]:
        """(i0, ni, j0, nj) in array indices of the cells this block sends
        (ghost False) or receives (ghost True) on side `high` along d."""
        is_, ie = NG, NG + self.nx - 1
        js, je = NG, NG + self.ny - 1
        if d == X1:
            if ghost:
                i0 = ie + 1 if high else is_ - NG
            else:
                i0 = ie - NG + 1 if high else is_
            return i0, NG, js, self.ny + 1
        if ghost:
            j0 = je + 1 if high else js - NG
        else:
            j0 = je - NG + 1 if high else js
        return 0, self.sx, j0, NG

    # -- transports ----------------------------------------------------------
    def _nccl_setup(self, device: int) -> None:
        import torch

        dev = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.grid.stream, device=dev)
        self.dti = torch.zeros(1, dtype=torch.int64, device=dev)
        self.sendbuf = {(d, s): torch.empty(self.count[d], dtype=torch.float64, device=dev)
                        for d in (X1, X2) for s in (0, 1)}
        self.recvbuf = {(d, s): torch.empty(self.count[d], dtype=torch.float64, device=dev)
                        for d in (X1, X2) for s in (0, 1)}

    def _ipc_setup(self) -> None:
        L, h = lib(), self.grid._h
        # one allocation per rank: the maximum board, then receive slots
        # [parity][direction][side] (side 0: from the low neighbour into my
        # low ghosts; side 1: from the high neighbour into my high ghosts)
        self.own = L.athb_device_alloc(h, BOARD_BYTES + 8 * self.slot)
        self.send = L.athb_device_alloc(h, 2 * self.slot)
        if not self.own or not self.send:
            raise RuntimeError("athb_device_alloc failed")
        handle = C.create_string_buffer(64)
        _check(L.athb_ipc_handle(h, C.c_void_p(self.own), handle))
        handles = [None] * self.ranks
        self.dist.all_gather_object(handles, bytes(handle.raw), group=self.group)
        self.peer = {self.rank: self.own}
        wanted = {0} | {r for d in (X1, X2) for r in self.nbr[d] if r is not None}
        for r in sorted(wanted - {self.rank}):
            ptr = C.c_void_p()
            _check(L.athb_ipc_open(h, handles[r], C.byref(ptr)))
            self.peer[r] = ptr.value

    def _recv_addr(self, r: int, parity: int, d: int, side: int) -> int:
        return self.peer[r] + BOARD_BYTES + ((parity * 2 + d) * 2 + side) * self.slot

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

    def _exchange_device(self, d: int) -> None:
        """Ghosts along direction d from the neighbours' edges (collective)."""
        L, h = lib(), self.grid._h
        low, high = self.nbr[d]
        if self.transport == "nccl":
            import torch

            for s, peer in ((0, low), (1, high)):
                if peer is not None:
                    _check(L.athb_rect_pack(h, *self._edge(d, s == 1, False),
                                            C.c_void_p(self.sendbuf[(d, s)].data_ptr())))
            with torch.cuda.stream(self.stream):
                # sends in the order (low edge, high edge), receives in the
                # order (high ghosts, low ghosts): where one peer is both
                # neighbours (2 pieces, periodic), messages between a pair
                # match in order, and my low edge is its high ghosts
                ops = []
                if low is not None:
                    ops.append(self.dist.P2POp(self.dist.isend, self.sendbuf[(d, 0)], low, group=self.group))
                if high is not None:
                    ops.append(self.dist.P2POp(self.dist.isend, self.sendbuf[(d, 1)], high, group=self.group))
                if high is not None:
                    ops.append(self.dist.P2POp(self.dist.irecv, self.recvbuf[(d, 1)], high, group=self.group))
                if low is not None:
                    ops.append(self.dist.P2POp(self.dist.irecv, self.recvbuf[(d, 0)], low, group=self.group))
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()   # the grid's stream waits for the transfers
            for s, peer in ((0, low), (1, high)):
                if peer is not None:
                    _check(L.athb_rect_unpack(h, *self._edge(d, s == 1, True),
                                              C.c_void_p(self.recvbuf[(d, s)].data_ptr())))
            return
        # ipc: my low edge becomes the high ghosts of the low neighbour (its
        # side 1), my high edge the low ghosts of the high neighbour (side 0)
        q = self.parity
        nbytes = self.count[d] * 8
        for s, peer in ((0, low), (1, high)):
            if peer is None:
                continue
            src = self.send + s * self.slot
            _check(L.athb_rect_pack(h, *self._edge(d, s == 1, False), C.c_void_p(src)))
            _check(L.athb_copy_async(h, C.c_void_p(self._recv_addr(peer, q, d, 1 - s)), C.c_void_p(src), nbytes))
        self.grid.synchronize()
        self._barrier()   # every copy into my receive buffers has landed
        for s, peer in ((0, low), (1, high)):
            if peer is not None:
                _check(L.athb_rect_unpack(h, *self._edge(d, s == 1, True),
                                          C.c_void_p(self._recv_addr(self.rank, q, d, s))))
        self.parity ^= 1   # the next exchange lands in the other buffers

    # -- host transport (px = 1) --------------------------------------------
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

    def _exchange_host(self) -> None:
        import torch

        below, above = self.nbr[X2]
        js, je = NG, NG + self.ny - 1
        up, down = 0, 1  # tags: rows travelling to the rank above / below
        sends, recvs = [], []
        if below is not None:  # my lowest rows become the ghosts above the rank below
            sends.append((below, down, torch.from_numpy(self._rows(js))))
            recvs.append((below, up, js - NG, torch.empty((len(PLANES), NG, self.sx), dtype=torch.float64)))
        if above is not None:  # my highest rows become the ghosts below the rank above
            sends.append((above, up, torch.from_numpy(self._rows(je - NG + 1))))
            recvs.append((above, down, je + 1, torch.empty((len(PLANES), NG, self.sx), dtype=torch.float64)))
        ops = [self.dist.P2POp(self.dist.isend, t, peer, group=self.group, tag=tag) for peer, tag, t in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer, group=self.group, tag=tag) for peer, tag, _, t in recvs]
        for w in self.dist.batch_isend_irecv(ops):
            w.wait()
        for _, _, j0, t in recvs:
            self._put(j0, t.numpy())

    # -- the ghost zones -----------------------------------------------------
    def _ghosts(self) -> None:
        L, h = lib(), self.grid._h
        if self.sides1:
            _check(L.athb_ghost_fill(h, 1, self.sides1))
        t0 = time.perf_counter()
        if self.px > 1:
            self._exchange_device(X1)
        if self.py > 1:
            if self.transport == "host":
                self._exchange_host()
            else:
                self._exchange_device(X2)
        self.exchange_s += time.perf_counter() - t0
        if self.sides2:
            _check(L.athb_ghost_fill(h, 2, self.sides2))

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
        """The global interior state (planes x Nx2 x Nx1) on rank 0
        (collective; the process group must carry CPU tensors)."""
        import torch

        planes = self.grid.download()[0][:, NG:NG + self.ny, NG:NG + self.nx]
        mine = torch.from_numpy(np.ascontiguousarray(planes))
        if self.ranks == 1:
            return mine.numpy()
        if self.rank == 0:
            out = np.empty((len(PLANES), self.gnx2, self.gnx1))
            for r in range(self.ranks):
                (i0, nx), (j0, ny) = self.cols[r % self.px], self.rows[r // self.px]
                if r == 0:
                    t = mine
                else:
                    t = torch.empty((len(PLANES), ny, nx), dtype=torch.float64)
                    self.dist.recv(t, src=r, group=self.group)
                out[:, j0:j0 + ny, i0:i0 + nx] = t.numpy()
            return out
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


class SlabGrid(BlockGrid):
    """The 1D case: `ranks` slabs along x2 (px = 1), any transport."""

    def __init__(self, blocks: dict, problem: str, rank: int, ranks: int, group=None, transport: str = "host"):
        if transport not in self.TRANSPORTS:
            raise ValueError(f"transport must be one of {self.TRANSPORTS}")
        if transport == "ipc" and ranks > MAX_RANKS:
            raise ValueError(f"ipc transport: at most {MAX_RANKS} ranks")
        super().__init__(blocks, problem, rank, 1, ranks, group, transport)
        self.slabs = self.rows
        self.nx1, self.nx2 = self.gnx1, self.gnx2
