"""Ensemble bookkeeping: the seeded instances and their partition over GPUs."""
from __future__ import annotations

from athena_cuda_b200 import ensemble


def test_instances_are_seeded_and_in_range():
    a, b = ensemble.instances(32, seed=5), ensemble.instances(32, seed=5)
    assert a == b and a != ensemble.instances(32, seed=6)
    for name, blocks in a:
        g, p = blocks["grid"], blocks["problem"]
        assert name == "blast" and g["Nx1"] in ensemble.SIZES and g["Nx2"] in ensemble.SIZES
        assert 10.0 <= p["prat"] <= 1000.0 and 0.05 <= p["radius"] <= 0.15 and 0.1 <= p["b0"] <= 2.0
        assert abs((g["x2max"] - g["x2min"]) / (g["x1max"] - g["x1min"]) - g["Nx2"] / g["Nx1"]) < 1e-12


def test_partition_covers_every_instance_once_and_balances():
    items = ensemble.instances(512)
    for ranks in (1, 2, 3, 8):
        parts = ensemble.partition(items, ranks)
        assert sorted(k for p in parts for k in p) == list(range(len(items)))
        loads = [sum(ensemble.work_estimate(items[k][1]) for k in p) for p in parts]
        biggest = max(ensemble.work_estimate(b) for _, b in items)
        assert max(loads) - min(loads) <= biggest
