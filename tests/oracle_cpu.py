"""ctypes access to the oracle restatement (oracle/mhd_oracle.cpp) -- used only
as the checker in tests."""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
_lib = None

STAGES = ("predict", "emf_half", "correct", "emf_full", "update", "new_dt")
KINDS = ("add", "mul", "div", "sqrt", "neg")


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        sys.path.insert(0, str(ROOT / "oracle"))
        import build_oracle

        path = build_oracle.build()
        L = C.CDLL(str(path))
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.oracle_run.restype = C.c_int
        L.oracle_run.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, ip, C.c_double, C.c_double,
                                 C.c_double, C.c_int, C.c_int, C.c_int, dp, dp, dp, ip]
        L.oracle_opcount.restype = C.c_int
        L.oracle_opcount.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, ip, C.c_double, C.c_double,
                                     C.c_double, C.c_int, C.c_int, C.c_int, dp, dp]
        _lib = L
    return _lib


def run(planes: np.ndarray, dx1, dx2, bc, gamma, cour_no, tlim, nlim=-1, flux=0, max_steps=-1):
    """Reference main loop from an initial state; returns (planes, dt, time, nstep)."""
    P = np.ascontiguousarray(planes, dtype=np.float64).copy()
    _, sy, sx = P.shape
    b = (C.c_int * 4)(*bc)
    dt, t, n = C.c_double(), C.c_double(), C.c_int()
    lib().oracle_run(sx - 8, sy - 8, dx1, dx2, b, gamma, cour_no, tlim, nlim, flux, max_steps,
                     P.ctypes.data_as(C.POINTER(C.c_double)), C.byref(dt), C.byref(t), C.byref(n))
    return P, dt.value, t.value, n.value


def opcount(planes: np.ndarray, dx1, dx2, bc, gamma, cour_no, tlim, nlim=-1, flux=0, max_steps=-1):
    """Operation counts per stage summed over the steps run: {stage: {kind: n}}, nsteps."""
    P = np.ascontiguousarray(planes, dtype=np.float64)
    _, sy, sx = P.shape
    b = (C.c_int * 4)(*bc)
    out = np.zeros(len(STAGES) * len(KINDS))
    n = lib().oracle_opcount(sx - 8, sy - 8, dx1, dx2, b, gamma, cour_no, tlim, nlim, flux, max_steps,
                             P.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)))
    counts = {s: {k: int(out[i * 5 + j]) for j, k in enumerate(KINDS)} for i, s in enumerate(STAGES)}
    return counts, n
