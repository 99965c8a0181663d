"""ctypes access to the host-CPU build of the tangent-linear model and the
adjoint (tests/hostcheck/adjoint_host.cpp) -- TEST INFRASTRUCTURE: it runs the
library's own generic step / TLM / adjoint code on the CPU."""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
_lib = None


def paths() -> dict:
    sys.path.insert(0, str(ROOT / "tests" / "hostcheck"))
    import build as hostcheck_build

    return hostcheck_build.build()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        from athena_cuda_b200 import Config

        L = C.CDLL(str(paths()["lib"]))
        dp = C.POINTER(C.c_double)
        L.hc_forward.argtypes = [C.POINTER(Config), dp, C.c_int, dp, dp, dp]
        L.hc_tlm.argtypes = [C.POINTER(Config), dp, dp, C.c_int, dp, dp, dp, dp]
        L.hc_adjoint.argtypes = [C.POINTER(Config), dp, C.c_int, C.c_int, dp, dp, C.POINTER(C.c_longlong)]
        L.hc_adjoint_seed.argtypes = [C.POINTER(Config), dp, dp, C.c_int, C.c_int, dp, dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def forward(cfg, S0: np.ndarray, n: int):
    S = np.ascontiguousarray(S0, dtype=np.float64)
    out = np.zeros_like(S)
    dt, t = C.c_double(), C.c_double()
    steps = lib().hc_forward(C.byref(cfg), _p(S), n, _p(out), C.byref(dt), C.byref(t))
    return out, dt.value, t.value, steps


def tlm(cfg, S0: np.ndarray, dS0: np.ndarray, n: int):
    S = np.ascontiguousarray(S0, dtype=np.float64)
    dS = np.ascontiguousarray(dS0, dtype=np.float64)
    SN, dSN = np.zeros_like(S), np.zeros_like(S)
    J, dJ = C.c_double(), C.c_double()
    lib().hc_tlm(C.byref(cfg), _p(S), _p(dS), n, C.byref(J), C.byref(dJ), _p(SN), _p(dSN))
    return J.value, dJ.value, SN, dSN


def adjoint(cfg, S0: np.ndarray, n: int, slots: int):
    S = np.ascontiguousarray(S0, dtype=np.float64)
    g = np.zeros_like(S)
    J, adv = C.c_double(), C.c_longlong()
    steps = lib().hc_adjoint(C.byref(cfg), _p(S), n, slots, C.byref(J), _p(g), C.byref(adv))
    return J.value, g, steps, adv.value


def adjoint_seed(cfg, S0: np.ndarray, seed: np.ndarray, n: int, slots: int):
    """Adjoint seeded with a cotangent of the final state: (<seed, S^N>,
    (dS^N/dS^0)^T seed, steps)."""
    S = np.ascontiguousarray(S0, dtype=np.float64)
    sd = np.ascontiguousarray(seed, dtype=np.float64)
    g = np.zeros_like(S)
    J = C.c_double()
    steps = lib().hc_adjoint_seed(C.byref(cfg), _p(S), _p(sd), n, slots, C.byref(J), _p(g))
    return J.value, g, steps


def interior_direction(rng, cfg, planes=range(11)) -> np.ndarray:
    """A random direction on the cells a step writes (interior, B1i column
    ie+1, B2i row je+1) of the chosen planes; zero in the ghost zones."""
    sx, sy = cfg.nx1 + 8, cfg.nx2 + 8
    d = np.zeros((11, sy, sx))
    for p in planes:
        d[p, 4:4 + cfg.nx2, 4:4 + cfg.nx1] = rng.standard_normal((cfg.nx2, cfg.nx1))
    if 8 in planes:
        d[8, 4:4 + cfg.nx2, 4 + cfg.nx1] = rng.standard_normal(cfg.nx2)
    if 9 in planes:
        d[9, 4 + cfg.nx2, 4:4 + cfg.nx1] = rng.standard_normal(cfg.nx1)
    return d


def objective(S: np.ndarray, cfg) -> float:
    """J = sum over interior cells of (B1c^2 + B2c^2)/2 (the adjoint's objective)."""
    b1 = S[5, 4:4 + cfg.nx2, 4:4 + cfg.nx1]
    b2 = S[6, 4:4 + cfg.nx2, 4:4 + cfg.nx1]
    return float(np.sum(0.5 * (b1 * b1 + b2 * b2)))
