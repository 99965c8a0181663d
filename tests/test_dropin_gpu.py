"""The drop-in boundary: programs written against the reference's entry points
(integrate_2d, set_bvals, new_dt, ...) run on the GPU through
libathena_b200.so with bit-identical results.

* oracle/_ref/athdrop_<problem>: the reference's own init_grid.c, par.c and
  problem generator plus the main-loop driver of oracle/ref_harness.c, linked
  against libathena_b200.so instead of the reference's integrator, boundary
  and dt sources (built by oracle/build_ref.py);
* the same loop driven from Python through athena_cuda_b200.dropin on a host
  Grid in the reference layout.
"""
from __future__ import annotations

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Params, configs, problem_state, write_athinput
from athena_cuda_b200.dropin import DropInLoop, HostGrid

pytestmark = pytest.mark.gpu

CASES = {
    "blast_40x60": ("blast", configs.blast(40, 60), 20),
    "blast_outflow": ("blast", configs.blast(36, 30, bc=(2, 2, 2, 2)), 15),
    "blast_reflect_mixed": ("blast", configs.blast(30, 36, bc=(1, 4, 2, 1)), 15),
    "field_loop_64x32": ("field_loop", configs.field_loop(64, 32), 20),
    "cpaw2d_32x16_period": ("cpaw2d", configs.cpaw2d(32, 16), None),
    # a user boundary condition registered by the problem file through
    # set_bvals_fun (oracle/userbc_problem.c): inflow on the left x1 side
    "userbc_inflow_40x30": ("userbc", configs.blast(40, 30, bc=(2, 2, 2, 2)), None),
    "userbc_inflow_periodic_x2": ("userbc", configs.blast(36, 24, bc=(2, 2, 4, 4)), None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_linked_dropin_binary_bit_exact(name, tmp_path):
    problem, blocks, steps = CASES[name]
    drop = refutil.REF_DIR / f"athdrop_{problem}"
    if not (drop.exists() and refutil.have_ref(problem)):
        pytest.skip("oracle/_ref drop-in builds missing (python oracle/build_ref.py)")
    ath = write_athinput(tmp_path / "athinput", blocks)
    ref = refutil.run_ref(problem, "roe", ath, tmp_path, steps=steps)
    got = refutil.run_ref(problem, "roe", ath, tmp_path, steps=steps, exe=drop)
    rep = refutil.mismatch_report(ref["planes"], got["planes"], PLANES)
    assert rep == "", rep
    assert (got["nstep"], got["time"], got["dt"]) == (ref["nstep"], ref["time"], ref["dt"])


@pytest.mark.parametrize("name", ["blast_40x60", "blast_reflect_mixed", "field_loop_64x32", "cpaw2d_32x16_period",
                                  "userbc_inflow_40x30"])
def test_linked_dropin_binary_host_unchanged_mode(name, tmp_path, monkeypatch):
    """The reference's own driver, relinked, with the opt-in host-unchanged
    mode (ATHB_DROPIN_HOST_UNCHANGED=1): same output bit for bit; user
    boundary functions fall back to the full path."""
    problem, blocks, steps = CASES[name]
    drop = refutil.REF_DIR / f"athdrop_{problem}"
    if not (drop.exists() and refutil.have_ref(problem)):
        pytest.skip("oracle/_ref drop-in builds missing (python oracle/build_ref.py)")
    ath = write_athinput(tmp_path / "athinput", blocks)
    ref = refutil.run_ref(problem, "roe", ath, tmp_path, steps=steps)
    monkeypatch.setenv("ATHB_DROPIN_HOST_UNCHANGED", "1")
    got = refutil.run_ref(problem, "roe", ath, tmp_path, steps=steps, exe=drop)
    rep = refutil.mismatch_report(ref["planes"], got["planes"], PLANES)
    assert rep == "", rep
    assert (got["nstep"], got["time"], got["dt"]) == (ref["nstep"], ref["time"], ref["dt"])


@pytest.mark.parametrize("host_unchanged", [False, True])
@pytest.mark.parametrize("name", ["blast_40x60", "blast_reflect_mixed", "field_loop_64x32"])
def test_python_dropin_loop_bit_exact(name, host_unchanged, tmp_path):
    problem, blocks, steps = CASES[name]
    if not refutil.have_ref(problem):
        pytest.skip("oracle/_ref not built")
    ath = write_athinput(tmp_path / "athinput", blocks)
    ref = refutil.run_ref(problem, "roe", ath, tmp_path, steps=steps)
    p = Params(ath)
    cfg = p.config()
    hg = HostGrid(problem_state(problem, p), (cfg.x1max - cfg.x1min) / cfg.nx1,
                  (cfg.x2max - cfg.x2min) / cfg.nx2, cfg.x1min, cfg.x2min)
    loop = DropInLoop(hg, configs.GAMMA, cfg.cour_no, bc=(cfg.bc_ix1, cfg.bc_ox1, cfg.bc_ix2, cfg.bc_ox2),
                      host_unchanged=host_unchanged)
    h_entry, _ = loop.bytes_moved()   # the counters run for the whole process
    loop.steps(steps, tlim=cfg.tlim)
    h2d = loop.bytes_moved()[0] - h_entry
    got = hg.planes()
    G = hg.grid
    loop.close()
    rep = refutil.mismatch_report(ref["planes"], got, PLANES)
    assert rep == "", rep
    assert (G.nstep, G.time, G.dt) == (ref["nstep"], ref["time"], ref["dt"])
    if host_unchanged:   # one full upload by the first step, none after it
        state = 8 * 11 * hg.sx * hg.sy
        assert h2d <= state, (h2d, state)
    hg.close()
