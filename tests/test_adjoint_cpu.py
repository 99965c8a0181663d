"""The tangent-linear model and the adjoint of the main loop, checked on the
host CPU with the library's own code (the generic step, the hand-written
reverse of every physics function and every stage, the checkpoint driver),
compiled for the CPU by tests/hostcheck/build.py.

* every adjoint function against the tangent-linear model of the same
  function (dot-product test, random inputs covering the limiter, supersonic,
  HLLE-fallback and degenerate-field branches);
* the generic step (the recorded forward step of the adjoint) against the
  oracle restatement, bit for bit;
* the full loop: <ybar, TLM xdot> == <ADJ ybar, xdot> for the objective
  J = sum (B1c^2 + B2c^2)/2, on smooth and white-noise states, Roe and HLLE,
  periodic / outflow / reflecting boundaries, with the tlim clamp active;
* every checkpoint schedule (from no free slot to one per step) gives the
  same gradient bit for bit;
* the tangent against central finite differences of the oracle.
"""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

import adjoint_host as ah
import oracle_cpu
import refutil
from athena_cuda_b200 import Params, configs, problem_state

CASES = {
    # name: (problem or "random:<smooth>", blocks, steps)
    "blast_periodic": ("blast", configs.blast(16, 12), 6),
    "blast_mixed_bc": ("blast", configs.blast(14, 10, bc=(1, 2, 4, 2)), 6),
    "blast_reflect_hlle": ("blast", configs.blast(12, 12, bc=(1, 1, 1, 1), flux="hlle"), 5),
    "field_loop": ("field_loop", configs.field_loop(16, 8), 5),
    "random_smooth": ("random:1", configs.field_loop(14, 10), 4),
    "random_noise": ("random:0", configs.field_loop(12, 10), 3),
    "random_noise_hlle": ("random:0", configs.field_loop(12, 10, flux="hlle"), 3),
    "cpaw_tlim_clamp": ("cpaw2d", configs.cpaw2d(16, 8, tlim=0.05), 40),
}


def _setup(name):
    problem, blocks, steps = CASES[name]
    p = Params.from_blocks(blocks)
    cfg = p.config()
    if problem.startswith("random"):
        S0 = refutil.random_state(np.random.default_rng(77), cfg.nx1, cfg.nx2, problem.endswith("1"))
    else:
        S0 = problem_state(problem, p)
    return cfg, S0, steps


def test_adjoint_functions_dot_product():
    exe = ah.paths()["pieces"]
    out = subprocess.run([str(exe), "20000"], capture_output=True, text=True, check=True).stdout
    rows = {}
    for line in out.splitlines():
        m = re.match(r"(\S+)\s+trials=(\d+) worst_rel=\S+ worst_vs_terms=(\S+)", line)
        if m:
            rows[m.group(1)] = (int(m.group(2)), float(m.group(3)))
    for name in ("cons_to_prim", "prim_to_cons", "esys_prim", "plm_cell", "flux_roe", "flux_hlle", "corner_emf",
                 "cell_dti", "flux_hlle_degen"):
        n, err = rows[name]
        assert n > 1000 and err < 1e-12, (name, n, err)
    # b2 = b3 = 0 with b1 != 0: alpha_s is the root of a rounding residue in
    # both linearisations (esys_prim, the Roe eigenvectors)
    for name in ("esys_prim_degen", "flux_roe_degen"):
        n, err = rows[name]
        assert n > 1000 and err < 1e-6, (name, n, err)
    assert "hlle-fallback" in out and re.search(r"hlle-fallback [1-9]", out)


@pytest.mark.parametrize("name", ["blast_periodic", "blast_mixed_bc", "blast_reflect_hlle", "field_loop",
                                  "random_noise"])
def test_generic_step_bit_exact_against_oracle(name):
    cfg, S0, n = _setup(name)
    got, dt, t, steps = ah.forward(cfg, S0, n)
    dx1 = (cfg.x1max - cfg.x1min) / cfg.nx1
    dx2 = (cfg.x2max - cfg.x2min) / cfg.nx2
    want = oracle_cpu.run(S0, dx1, dx2, (cfg.bc_ix1, cfg.bc_ox1, cfg.bc_ix2, cfg.bc_ox2), cfg.gamma, cfg.cour_no,
                          cfg.tlim, n, cfg.flux, -1)
    assert steps == want[3]
    assert np.array_equal(got, want[0]), refutil.mismatch_report(want[0], got, [str(k) for k in range(11)])
    assert (dt, t) == (want[1], want[2])


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_loop_dot_product(name):
    cfg, S0, n = _setup(name)
    J, g, steps, _ = ah.adjoint(cfg, S0, n, n + 1)
    assert steps >= 1
    rng = np.random.default_rng(11)
    for planes in (range(11), [0], [1, 2], [4], [8, 9]):
        d = ah.interior_direction(rng, cfg, planes)
        J2, dJ, _, _ = ah.tlm(cfg, S0, d, steps)
        assert J2 == J
        ip = float(np.sum(g * d))
        scale = float(np.sum(np.abs(g * d)))
        assert abs(ip - dJ) <= 1e-12 * max(scale, abs(dJ), 1e-300), (name, list(planes), ip, dJ)
    # the gradient is zero on the ghost zones (they are functions of the interior)
    mask = ah.interior_direction(rng, cfg) != 0
    assert np.all(g[~mask] == 0.0)


def test_clamp_case_reaches_tlim():
    cfg, S0, n = _setup("cpaw_tlim_clamp")
    _, _, t, steps = ah.forward(cfg, S0, n)
    assert steps < n and t == cfg.tlim   # the last step was clamped to tlim


@pytest.mark.parametrize("name", ["blast_mixed_bc", "random_smooth"])
def test_checkpoint_schedules_give_identical_gradients(name):
    cfg, S0, n = _setup(name)
    n = 7
    J0, g0, _, adv0 = ah.adjoint(cfg, S0, n, n + 1)
    assert adv0 == n   # every state stored: one forward sweep
    seen = set()
    for slots in (1, 2, 3, 5):
        J, g, _, adv = ah.adjoint(cfg, S0, n, slots)
        assert J == J0 and np.array_equal(g, g0), slots
        seen.add(adv)
        # binomial checkpointing: the fewest forward steps for the slots
        # (Griewank's bound; slot 0 holds S^0)
    assert len(seen) == 4
    # tape mode: every step's intermediates kept by the first sweep
    J, g, _, adv = ah.adjoint(cfg, S0, n, -1)
    assert J == J0 and np.array_equal(g, g0) and adv == 0


def test_tangent_matches_oracle_finite_differences():
    """The TLM is the derivative of the reference algorithm: central
    differences of the oracle along the same direction agree to 1e-6."""
    cfg, S0, n = _setup("random_smooth")
    rng = np.random.default_rng(3)
    d = ah.interior_direction(rng, cfg, [0, 1, 2, 4])
    J, dJ, _, _ = ah.tlm(cfg, S0, d, n)
    dx1 = (cfg.x1max - cfg.x1min) / cfg.nx1
    dx2 = (cfg.x2max - cfg.x2min) / cfg.nx2
    bc = (cfg.bc_ix1, cfg.bc_ox1, cfg.bc_ix2, cfg.bc_ox2)
    eps = 1e-6
    Jpm = []
    for s in (1.0, -1.0):
        P = oracle_cpu.run(S0 + s * eps * d, dx1, dx2, bc, cfg.gamma, cfg.cour_no, cfg.tlim, n, cfg.flux, -1)[0]
        Jpm.append(ah.objective(P, cfg))
    fd = (Jpm[0] - Jpm[1]) / (2 * eps)
    assert abs(fd - dJ) <= 1e-6 * abs(dJ), (fd, dJ)


@pytest.mark.parametrize("name", sorted(CASES))
def test_seeded_adjoint_is_the_transpose_of_the_tlm(name):
    """athb_adjoint_vjp's code: for a random cotangent w of the final state,
    <(dS^N/dS^0)^T w, d> = <w, dS^N(d)> (the TLM's final tangent state), and
    J = <w, S^N>; the magnetic energy's seed (B1c, B2c) gives the plain
    adjoint's gradient bit for bit."""
    cfg, S0, n = _setup(name)
    _, g0, steps, _ = ah.adjoint(cfg, S0, n, n + 1)
    rng = np.random.default_rng(23)
    w = ah.interior_direction(rng, cfg)
    Jw, gw, steps_w = ah.adjoint_seed(cfg, S0, w, n, n + 1)
    assert steps_w == steps
    d = ah.interior_direction(rng, cfg)
    _, _, SN, dSN = ah.tlm(cfg, S0, d, steps)
    mask = ah.interior_direction(np.random.default_rng(0), cfg) != 0
    assert abs(Jw - float(np.sum((w * SN)[mask]))) <= 1e-12 * float(np.sum(np.abs(w * SN)))
    lhs, rhs = float(np.sum(gw * d)), float(np.sum((w * dSN)[mask]))
    scale = max(float(np.sum(np.abs(gw * d))), float(np.sum(np.abs(w * dSN))))
    assert abs(lhs - rhs) <= 1e-11 * scale, (name, lhs, rhs)
    # the magnetic-energy seed reproduces the plain adjoint
    seed = np.zeros_like(S0)
    seed[5:7, 4:4 + cfg.nx2, 4:4 + cfg.nx1] = SN[5:7, 4:4 + cfg.nx2, 4:4 + cfg.nx1]
    _, gm, _ = ah.adjoint_seed(cfg, S0, seed, n, 3)
    assert np.array_equal(gm, g0)
