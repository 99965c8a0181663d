"""Bit-exact parity of the sm_100a step against the reference CPU path.

Every case builds the same athinput for both sides, runs the reference's own
CPU sources (oracle/_ref, compiled by oracle/build_ref.py) and the CUDA library
for the same number of main-loop iterations, and requires every value of every
plane (ghost zones included), dt, time and nstep to be identical.  FP64
arithmetic is IEEE-754 on both sides and the CUDA build does not fuse
multiply-adds, so the tolerance is zero.
"""
from __future__ import annotations

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Grid, write_athinput
from athena_cuda_b200 import configs

pytestmark = pytest.mark.gpu

CASES = {
    # name: (problem, flux, blocks, steps)
    "field_loop_64x32": ("field_loop", "roe", configs.field_loop(64, 32), 20),
    "field_loop_64x32_hlle": ("field_loop", "hlle", configs.field_loop(64, 32, flux="hlle"), 20),
    "blast_40x60": ("blast", "roe", configs.blast(40, 60), 30),
    "blast_40x60_outflow": ("blast", "roe", configs.blast(40, 60, bc=(2, 2, 2, 2)), 30),
    "blast_40x60_reflect": ("blast", "roe", configs.blast(40, 60, bc=(1, 1, 1, 1)), 30),
    "blast_48x40_mixed": ("blast", "roe", configs.blast(48, 40, bc=(1, 2, 4, 4)), 25),
    "blast_40x60_hlle": ("blast", "hlle", configs.blast(40, 60, flux="hlle"), 30),
    "blast_strong_b": ("blast", "roe", configs.blast(32, 32, b0=4.0, prat=1000.0, angle=30.0), 25),
    "cpaw2d_32x16_period": ("cpaw2d", "roe", configs.cpaw2d(32, 16), None),
    "cpaw2d_32x16_hlle_period": ("cpaw2d", "hlle", configs.cpaw2d(32, 16, flux="hlle"), None),
    "ragged_5x7": ("blast", "roe", configs.blast(5, 7, bc=(2, 4, 1, 2)), 12),
    "minimum_4x4": ("field_loop", "roe", configs.field_loop(4, 4), 8),
    "ragged_37x11": ("field_loop", "roe", configs.field_loop(37, 11), 15),
    "nlim_stop": ("blast", "roe", configs.blast(24, 24, nlim=7), None),
}


def _compare(ref: dict, planes: np.ndarray, dt: float, t: float, n: int) -> None:
    rep = refutil.mismatch_report(ref["planes"], planes, PLANES)
    assert rep == "", "state differs from the reference:\n" + rep
    assert n == ref["nstep"]
    assert t == ref["time"], (t, ref["time"])
    assert dt == ref["dt"], (dt, ref["dt"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_step_bit_exact(name, tmp_path):
    problem, flux, blocks, steps = CASES[name]
    if not refutil.have_ref(problem, flux):
        pytest.skip("oracle/_ref not built (python oracle/build_ref.py)")
    ath = write_athinput(tmp_path / "athinput", blocks)
    ref = refutil.run_ref(problem, flux, ath, tmp_path, steps=steps)
    g = Grid.from_athinput(ath, problem)
    g.run(steps if steps is not None else 1_000_000)
    planes, dt, t, n = g.download()
    g.close()
    _compare(ref, planes, dt, t, n)


@pytest.mark.parametrize("smooth", [True, False])
@pytest.mark.parametrize("flux", ["roe", "hlle"])
def test_random_states_bit_exact(smooth, flux, tmp_path):
    """Random (smooth and white-noise) states exercise every branch: limiter
    cases, supersonic faces, negative intermediate states (HLLE fallback)."""
    if not refutil.have_ref("file", flux):
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(1234 + smooth)
    nx1, nx2 = 40, 28
    P = refutil.random_state(rng, nx1, nx2, smooth)
    blocks = configs.field_loop(nx1, nx2, flux=flux)
    blocks["time"]["nlim"] = 6
    ath = write_athinput(tmp_path / "athinput", blocks)
    init = refutil.write_raw(tmp_path / "init.bin", P)
    ref = refutil.run_ref("file", flux, ath, tmp_path, init=init)
    cfg_grid = Grid.from_athinput(ath, "field_loop")  # geometry and parameters
    cfg_grid.upload(P)
    cfg_grid.set_bvals()
    cfg_grid.new_dt()
    cfg_grid.run(100)
    planes, dt, t, n = cfg_grid.download()
    cfg_grid.close()
    _compare(ref, planes, dt, t, n)


@pytest.mark.slow
def test_blast_200x300_to_t02_bit_exact(tmp_path):
    """The full blast configuration (200x300, t = 0.2, ~190 steps)."""
    if not refutil.have_ref("blast", "roe"):
        pytest.skip("oracle/_ref not built")
    ath = write_athinput(tmp_path / "athinput", configs.blast(200, 300, tlim=0.2))
    ref = refutil.run_ref("blast", "roe", ath, tmp_path)
    g = Grid.from_athinput(ath, "blast")
    g.run(1_000_000)
    planes, dt, t, n = g.download()
    g.close()
    _compare(ref, planes, dt, t, n)
