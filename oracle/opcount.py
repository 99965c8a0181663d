"""Count the algorithmic FP64 operations of one main-loop iteration of the
reference step, per stage, with the counting instantiation of the oracle
restatement (oracle/mhd_oracle.cpp) -- TEST/MEASUREMENT INFRASTRUCTURE ONLY.

Counted: every binary + - * / and every sqrt on a Real value that the
reference algorithm performs (dense 7x7 eigenmatrices, the reference's work
ranges, the dead cc_pos of step 7 and the discarded fast speeds of new_dt
included); unary negation reported separately.  The restatement is bit-exact
against the reference (tests/test_oracle_pin.py), so these are the
reference's operations.

Usage: python oracle/opcount.py --problem field_loop --nx 2048 --ny 2048 --steps 3
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--problem", default="field_loop")
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    import oracle_cpu
    from athena_cuda_b200 import Params, configs, problem_state, write_athinput

    with tempfile.TemporaryDirectory() as td:
        ath = write_athinput(Path(td) / "a", configs.BUILDERS[a.problem](a.nx, a.ny))
        p = Params(ath)
        cfg = p.config()
        P = problem_state(a.problem, p)
    c, n = oracle_cpu.opcount(P, (cfg.x1max - cfg.x1min) / a.nx, (cfg.x2max - cfg.x2min) / a.ny,
                              (cfg.bc_ix1, cfg.bc_ox1, cfg.bc_ix2, cfg.bc_ox2), cfg.gamma, cfg.cour_no,
                              cfg.tlim, cfg.nlim, cfg.flux, a.steps)
    zc = a.nx * a.ny * n
    per = {s: {k: v / zc for k, v in d.items()} for s, d in c.items()}
    tot = {s: sum(v for k, v in d.items() if k != "neg") for s, d in per.items()}
    print(json.dumps({"problem": a.problem, "nx": a.nx, "ny": a.ny, "steps": n, "per_zone_cycle": per,
                      "ops_per_zone_cycle_by_stage": tot,
                      "integrate_2d": sum(v for s, v in tot.items() if s != "new_dt"),
                      "step_total": sum(tot.values())}, indent=1))


if __name__ == "__main__":
    main()
