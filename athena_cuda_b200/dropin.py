"""The reference's main loop (src/main.c:221-318) driven through the drop-in
entry points (integrate_2d / new_dt / set_bvals) of libathena_b200.so on a
host Grid in the reference's own layout (src/athena.h:43-120).

This is the path a program written against the reference takes: every call
works on host buffers, so host<->device copies happen inside every step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import NGHOST, NPLANES, lib


class Gas(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("d", "M1", "M2", "M3", "E", "B1c", "B2c", "B3c")]


class GridStruct(C.Structure):
    _fields_ = [
        ("U", C.POINTER(C.POINTER(Gas))),
        ("B1i", C.POINTER(C.POINTER(C.c_double))),
        ("B2i", C.POINTER(C.POINTER(C.c_double))),
        ("B3i", C.POINTER(C.POINTER(C.c_double))),
        ("x1_0", C.c_double), ("x2_0", C.c_double), ("dx1", C.c_double), ("dx2", C.c_double),
        ("dt", C.c_double), ("time", C.c_double),
        ("nstep", C.c_int), ("Nx1", C.c_int), ("Nx2", C.c_int),
        ("is_", C.c_int), ("ie", C.c_int), ("js", C.c_int), ("je", C.c_int),
        ("idisp", C.c_int), ("jdisp", C.c_int), ("outfilename", C.c_char_p),
    ]


def _setup_signatures():
    L = lib()
    gp = C.POINTER(GridStruct)
    for name, args in {
        "integrate_init_2d": [C.c_int, C.c_int], "integrate_destruct_2d": [],
        "integrate_2d": [gp], "lr_states_init": [C.c_int, C.c_int], "lr_states_destruct": [],
        "set_bvals_init": [gp], "set_bvals": [gp, C.c_int], "new_dt": [gp],
        "athb_dropin_set_bc": [C.c_int] * 4, "athb_dropin_set_flux": [C.c_int],
        "athb_dropin_set_device": [C.c_int], "athb_dropin_set_host_unchanged": [C.c_int],
        "athb_dropin_bytes": [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)],
    }.items():
        f = getattr(L, name)
        f.restype, f.argtypes = None, args
    return L


class HostGrid:
    """A reference-layout Grid whose arrays live in pinned host memory."""

    def __init__(self, planes: np.ndarray, dx1: float, dx2: float, x1_0: float, x2_0: float):
        L = lib()
        _, sy, sx = planes.shape
        self.sx, self.sy = sx, sy
        self._bufs = []

        def alloc(nbytes):
            p = L.athb_host_alloc(nbytes)
            if not p:
                raise MemoryError("athb_host_alloc failed")
            self._bufs.append(p)
            return p

        ucells = sy * sx
        up = alloc(ucells * C.sizeof(Gas))
        self.U = np.ctypeslib.as_array((C.c_double * (ucells * 8)).from_address(up)).reshape(sy, sx, 8)
        self.B = []
        bptrs = []
        for _ in range(3):
            bp = alloc(ucells * 8)
            bptrs.append(bp)
            self.B.append(np.ctypeslib.as_array((C.c_double * ucells).from_address(bp)).reshape(sy, sx))
        self._urows = (C.POINTER(Gas) * sy)(*[C.cast(up + j * sx * C.sizeof(Gas), C.POINTER(Gas)) for j in range(sy)])
        self._brows = [(C.POINTER(C.c_double) * sy)(*[C.cast(bp + j * sx * 8, C.POINTER(C.c_double))
                                                       for j in range(sy)]) for bp in bptrs]
        g = GridStruct()
        g.U = C.cast(self._urows, C.POINTER(C.POINTER(Gas)))
        g.B1i, g.B2i, g.B3i = (C.cast(r, C.POINTER(C.POINTER(C.c_double))) for r in self._brows)
        g.x1_0, g.x2_0, g.dx1, g.dx2 = x1_0, x2_0, dx1, dx2
        g.Nx1, g.Nx2 = sx - 2 * NGHOST, sy - 2 * NGHOST
        g.is_, g.js = NGHOST, NGHOST
        g.ie, g.je = g.Nx1 + NGHOST - 1, g.Nx2 + NGHOST - 1
        g.idisp, g.jdisp = -NGHOST, -NGHOST
        self.grid = g
        self.set_planes(planes)

    def set_planes(self, planes: np.ndarray) -> None:
        self.U[...] = np.moveaxis(planes[:8], 0, -1)
        for k in range(3):
            self.B[k][...] = planes[8 + k]

    def planes(self) -> np.ndarray:
        out = np.empty((NPLANES, self.sy, self.sx))
        out[:8] = np.moveaxis(self.U, -1, 0)
        for k in range(3):
            out[8 + k] = self.B[k]
        return out

    def close(self) -> None:
        L = lib()
        for p in self._bufs:
            L.athb_host_free(p)
        self._bufs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DropInLoop:
    """The reference main loop on a HostGrid through the drop-in ABI."""

    def __init__(self, hg: HostGrid, gamma: float, cour_no: float, bc=(4, 4, 4, 4), flux: int = 0,
                 device: int = 0, host_unchanged: bool = False):
        self.L = _setup_signatures()
        self.L.athb_dropin_set_device(device)
        # the loop below never writes the Grid between the drop-in calls
        self.L.athb_dropin_set_host_unchanged(int(host_unchanged))
        self.hg = hg
        C.c_double.in_dll(self.L, "Gamma").value = gamma
        C.c_double.in_dll(self.L, "Gamma_1").value = gamma - 1.0
        C.c_double.in_dll(self.L, "Gamma_2").value = gamma - 2.0
        C.c_double.in_dll(self.L, "CourNo").value = cour_no
        self.L.athb_dropin_set_bc(*bc)
        self.L.athb_dropin_set_flux(flux)
        g = C.byref(hg.grid)
        hg.grid.time, hg.grid.nstep = 0.0, 0
        # src/main.c:130-197
        self.L.set_bvals_init(g)
        self.L.set_bvals(g, 0)
        self.L.new_dt(g)
        self.L.lr_states_init(hg.grid.Nx1, hg.grid.Nx2)
        self.L.integrate_init_2d(hg.grid.Nx1, hg.grid.Nx2)

    def steps(self, n: int, tlim: float = float("inf")) -> int:
        """Up to n iterations of src/main.c:221-318; returns the number run."""
        G, L = self.hg.grid, self.L
        g = C.byref(G)
        done = 0
        while done < n and G.time < tlim:
            if (tlim - G.time) < G.dt:
                G.dt = tlim - G.time
            L.integrate_2d(g)
            G.nstep += 1
            G.time += G.dt
            L.new_dt(g)
            L.set_bvals(g, 0)
            done += 1
        return done

    def bytes_moved(self) -> tuple[int, int]:
        h, d = C.c_ulonglong(), C.c_ulonglong()
        self.L.athb_dropin_bytes(C.byref(h), C.byref(d))
        return h.value, d.value

    def close(self) -> None:
        self.L.integrate_destruct_2d()
        self.L.lr_states_destruct()
