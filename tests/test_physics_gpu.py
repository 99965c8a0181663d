"""Size-independent properties of the GPU step and the reference's own
physics checks: constrained transport keeps div B at
round-off on every step; periodic runs conserve mass and energy to
round-off; the circularly polarised Alfven wave converges at second order
and its L1 errors equal the reference's Userwork_after_loop output
(src/cpaw2d.c:222-302)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import Grid, Params, configs, problem_state, write_athinput

pytestmark = pytest.mark.gpu


def _grid(tmp_path, problem, blocks):
    return Grid.from_athinput(write_athinput(tmp_path / "athinput", blocks), problem)


@pytest.mark.parametrize("problem,blocks", [
    ("field_loop", configs.field_loop(256, 128)),
    ("blast", configs.blast(120, 180, b0=2.0)),
    ("cpaw2d", configs.cpaw2d(64, 32)),
])
def test_divb_roundoff_and_conservation_every_step(problem, blocks, tmp_path):
    g = _grid(tmp_path, problem, blocks)
    d0 = g.diagnostics()
    bscale = max(1e-300, math.sqrt(2.0 * d0["emag"] / d0["mass"]))  # rms |B| (density ~ 1)
    dx = (blocks["grid"]["x1max"] - blocks["grid"]["x1min"]) / blocks["grid"]["Nx1"]
    for _ in range(40):
        g.run(1)
        d = g.diagnostics()
        # |div B| * dx / |B| is the relative round-off of the face differences
        assert d["max_divb"] * dx / bscale < 1e-13, d
        assert abs(d["mass"] - d0["mass"]) <= 1e-12 * abs(d0["mass"])
        assert abs(d["energy"] - d0["energy"]) <= 1e-12 * abs(d0["energy"])
    g.close()


def test_field_loop_magnetic_energy_decays_slowly(tmp_path):
    """Field-loop advection (Gardiner & Stone 2005): the loop's magnetic
    energy decays monotonically and slowly under numerical dissipation."""
    g = _grid(tmp_path, "field_loop", configs.field_loop(128, 64, tlim=0.5))
    e = [g.diagnostics()["bp2"]]
    while not g.status()["done"]:
        g.run(20)
        e.append(g.diagnostics()["bp2"])
    g.close()
    assert all(b <= a for a, b in zip(e, e[1:]))
    assert 0.5 < e[-1] / e[0] < 1.0


CPAW_SWEEP = [(32, 16), (64, 32), (128, 64)]


def test_cpaw2d_second_order_and_reference_errors(tmp_path):
    errs = []
    for nx1, nx2 in CPAW_SWEEP:
        blocks = configs.cpaw2d(nx1, nx2)
        d = tmp_path / f"{nx1}"
        d.mkdir()
        ath = write_athinput(d / "athinput", blocks)
        g = Grid.from_athinput(ath, "cpaw2d")
        g.run(1_000_000)
        e = g.cpaw2d_errors()
        # the device sums are the reference's serial row-major sums, bit for
        # bit (np.cumsum adds left to right)
        U = g.download()[0]
        S0 = problem_state("cpaw2d", Params(ath))
        n = nx1 * nx2
        sums = [float(np.cumsum(np.abs(U[k, 4:-4, 4:-4] - S0[k, 4:-4, 4:-4]).ravel())[-1]) for k in range(8)]
        rms = sums[0] ** 2 + sums[1] ** 2 + sums[2] ** 2 + sums[3] ** 2
        rms += sums[5] ** 2 + sums[6] ** 2 + sums[7] ** 2
        rms += sums[4] ** 2
        assert [e[0]] + list(e[1:]) == [math.sqrt(rms) / n] + [x / n for x in sums]
        g.close()
        assert g is not None and e[0] > 0
        errs.append(e[0])
        if refutil.have_ref("cpaw2d"):
            refutil.run_ref("cpaw2d", "roe", ath, d, extra=["--l1"])
            row = [l for l in (d / "cpaw2d-errors.dat").read_text().splitlines() if not l.startswith("#")][-1]
            ref = [float(x) for x in row.split()[2:]]  # RMS d M1 M2 M3 E B1c B2c B3c (6 digits)
            for mine, theirs in zip(e, ref):
                assert float(f"{mine:e}") == theirs, (mine, theirs)
    order = [math.log2(a / b) for a, b in zip(errs, errs[1:])]
    assert all(o > 1.8 for o in order), order
