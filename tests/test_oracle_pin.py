"""Pin the oracle restatement (oracle/mhd_oracle.cpp) to the reference itself:
starting from the reference's own initial state, the restatement must give
bit-identical states, dt, time and nstep to the reference's compiled CPU path
(oracle/_ref) on every configuration the GPU tests use.  Runs on CPU."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_cpu
import refutil
from athena_cuda_b200 import PLANES, configs, write_athinput

CASES = {
    "field_loop_64x32": ("field_loop", "roe", configs.field_loop(64, 32), 20),
    "field_loop_64x32_hlle": ("field_loop", "hlle", configs.field_loop(64, 32, flux="hlle"), 20),
    "blast_40x60": ("blast", "roe", configs.blast(40, 60), 30),
    "blast_40x60_outflow": ("blast", "roe", configs.blast(40, 60, bc=(2, 2, 2, 2)), 30),
    "blast_40x60_reflect": ("blast", "roe", configs.blast(40, 60, bc=(1, 1, 1, 1)), 30),
    "blast_48x40_mixed": ("blast", "roe", configs.blast(48, 40, bc=(1, 2, 4, 4)), 25),
    "blast_40x60_hlle": ("blast", "hlle", configs.blast(40, 60, flux="hlle"), 30),
    "cpaw2d_32x16_period": ("cpaw2d", "roe", configs.cpaw2d(32, 16), None),
    "cpaw2d_32x16_hlle_period": ("cpaw2d", "hlle", configs.cpaw2d(32, 16, flux="hlle"), None),
    "ragged_5x7": ("blast", "roe", configs.blast(5, 7, bc=(2, 4, 1, 2)), 12),
    "minimum_4x4": ("field_loop", "roe", configs.field_loop(4, 4), 8),
}


def _bc(blocks):
    g = blocks["grid"]
    return (g["ibc_x1"], g["obc_x1"], g["ibc_x2"], g["obc_x2"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(name, tmp_path):
    problem, flux, blocks, steps = CASES[name]
    if not refutil.have_ref(problem, flux):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    ath = write_athinput(tmp_path / "athinput", blocks)
    init = refutil.run_ref(problem, flux, ath, tmp_path, steps=0)
    ref = refutil.run_ref(problem, flux, ath, tmp_path, steps=steps)
    t = blocks["time"]
    planes, dt, time, n = oracle_cpu.run(
        init["planes"], init["dx1"], init["dx2"], _bc(blocks), configs.GAMMA, t["cour_no"], t["tlim"],
        t.get("nlim", -1), 1 if flux == "hlle" else 0, -1 if steps is None else steps)
    rep = refutil.mismatch_report(ref["planes"], planes, PLANES)
    assert rep == "", rep
    assert (n, time, dt) == (ref["nstep"], ref["time"], ref["dt"])
