"""The batched blast ensemble: independent MHD blast problems (src/blast.c)
of uneven sizes, each with its own dt and end time, seeded per instance.

Per instance: Nx1, Nx2 drawn independently from {64, 96, 128, 192, 256, 384,
512}, domain [-0.5, 0.5] x [-0.5 Nx2/Nx1, 0.5 Nx2/Nx1] (aspect Nx1:Nx2),
periodic, pressure ratio log-uniform in [10, 1000], blast radius uniform in
[0.05, 0.15], |B| uniform in [0.1, 2] at an angle uniform in [0, 180) degrees,
gamma 5/3, CFL 0.8, Roe fluxes, run to its own t = 0.1.
"""
from __future__ import annotations

import math

import numpy as np

from . import configs

SIZES = (64, 96, 128, 192, 256, 384, 512)


def instances(n: int = 512, seed: int = 2024, sizes=SIZES, tlim: float = 0.1,
              flux: str = "roe") -> list[tuple[str, dict]]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx1 = int(rng.choice(sizes))
        nx2 = int(rng.choice(sizes))
        prat = float(math.exp(rng.uniform(math.log(10.0), math.log(1000.0))))
        radius = float(rng.uniform(0.05, 0.15))
        b0 = float(rng.uniform(0.1, 2.0))
        angle = float(rng.uniform(0.0, 180.0))
        out.append(("blast", configs.blast(nx1, nx2, tlim=tlim, prat=prat, radius=radius, b0=b0,
                                           angle=angle, flux=flux)))
    return out


def work_estimate(blocks: dict) -> float:
    """Relative cost of one instance run to its end time: cells times steps,
    the steps taken as proportional to the cells across the smaller cell
    width (the CFL step shrinks with the cell size)."""
    g = blocks["grid"]
    dx = min((g["x1max"] - g["x1min"]) / g["Nx1"], (g["x2max"] - g["x2min"]) / g["Nx2"])
    return g["Nx1"] * g["Nx2"] * blocks["time"]["tlim"] / dx


def partition(items: list[tuple[str, dict]], ranks: int) -> list[list[int]]:
    """Instance indices per rank (one GPU each), balanced by work_estimate:
    largest first, each to the least-loaded rank.  The instances are
    independent, so a partitioned ensemble needs no communication."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    order = sorted(range(len(items)), key=lambda k: (-work_estimate(items[k][1]), k))
    load = [0.0] * ranks
    parts: list[list[int]] = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += work_estimate(items[k][1])
    return [sorted(p) for p in parts]
