"""The adjoint workload: the gradient of the field loop's final magnetic
energy with respect to its initial density.

Initial state: the field-loop problem (src/field_loop.c:40-137; rho = 1,
v = (2, 1), P = 1, face B from the curl of A_z) with the density replaced by
rho_0(x) at fixed velocity and pressure, so M = rho_0 v and
E = P/(gamma-1) + |B|^2/2 + rho_0 |v|^2/2.  rho_0 = 1 + amp * N(0,1) smoothed
by a periodic Gaussian of `width` cells (seeded).  Objective: J = sum over the
interior cells of (B1c^2 + B2c^2)/2 after N main-loop iterations.

The device computes dJ/d(state) (Grid.adjoint_gradient); the chain rule to
rho_0 is linear and done here: dJ/drho = g_d + v . g_M + |v|^2/2 g_E.
"""
from __future__ import annotations

import numpy as np

NG = 4  # ghost cells


def smoothed_density(nx1: int, nx2: int, seed: int, amp: float = 0.01, width: float = 4.0) -> np.ndarray:
    """1 + amp * (white noise convolved with a periodic Gaussian of standard
    deviation `width` cells, rescaled to unit standard deviation)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((nx2, nx1))
    ky = np.fft.fftfreq(nx2)[:, None]
    kx = np.fft.fftfreq(nx1)[None, :]
    kernel = np.exp(-2.0 * (np.pi * width) ** 2 * (kx * kx + ky * ky))
    s = np.real(np.fft.ifft2(np.fft.fft2(noise) * kernel))
    s /= np.std(s)
    return 1.0 + amp * s


def _velocity(base: np.ndarray):
    d = base[0, NG:-NG, NG:-NG]
    return base[1, NG:-NG, NG:-NG] / d, base[2, NG:-NG, NG:-NG] / d, base[3, NG:-NG, NG:-NG] / d


def density_state(base: np.ndarray, rho: np.ndarray) -> np.ndarray:
    """The base state with density rho at the base's velocity and pressure."""
    S = np.array(base, dtype=np.float64, copy=True)
    v1, v2, v3 = _velocity(base)
    d0 = base[0, NG:-NG, NG:-NG]
    S[0, NG:-NG, NG:-NG] = rho
    S[1, NG:-NG, NG:-NG] = rho * v1
    S[2, NG:-NG, NG:-NG] = rho * v2
    S[3, NG:-NG, NG:-NG] = rho * v3
    S[4, NG:-NG, NG:-NG] = base[4, NG:-NG, NG:-NG] + 0.5 * (rho - d0) * (v1 * v1 + v2 * v2 + v3 * v3)
    return S


def density_direction(base: np.ndarray, drho: np.ndarray) -> np.ndarray:
    """The state direction of a density direction drho (the linear map of
    density_state)."""
    D = np.zeros_like(base, dtype=np.float64)
    v1, v2, v3 = _velocity(base)
    D[0, NG:-NG, NG:-NG] = drho
    D[1, NG:-NG, NG:-NG] = drho * v1
    D[2, NG:-NG, NG:-NG] = drho * v2
    D[3, NG:-NG, NG:-NG] = drho * v3
    D[4, NG:-NG, NG:-NG] = 0.5 * drho * (v1 * v1 + v2 * v2 + v3 * v3)
    return D


def density_gradient(base: np.ndarray, grad: np.ndarray) -> np.ndarray:
    """dJ/drho from dJ/d(state) (the transpose of density_direction)."""
    v1, v2, v3 = _velocity(base)
    g = lambda p: grad[p, NG:-NG, NG:-NG]
    return g(0) + v1 * g(1) + v2 * g(2) + v3 * g(3) + 0.5 * (v1 * v1 + v2 * v2 + v3 * v3) * g(4)


def objective(S: np.ndarray) -> float:
    """J = sum over the interior cells of (B1c^2 + B2c^2)/2."""
    b1, b2 = S[5, NG:-NG, NG:-NG], S[6, NG:-NG, NG:-NG]
    return float(np.sum(0.5 * (b1 * b1 + b2 * b2)))
