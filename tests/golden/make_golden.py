"""Regenerate the golden fixtures in tests/golden/ from the reference CPU path.

Each fixture is the final state (all 11 planes, ghost zones included), dt,
time and nstep of the reference's own CPU step (oracle/_ref, compiled from the
reference sources by oracle/build_ref.py) after a fixed number of main-loop
iterations of a small configuration.  The fixtures let the GPU tests and
smoke() check parity on machines where the reference sources are absent.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import refutil  # noqa: E402
from athena_cuda_b200 import configs, write_athinput  # noqa: E402

FIXTURES = {
    # name: (problem, flux, blocks, steps)
    "field_loop_32x16_roe_10": ("field_loop", "roe", configs.field_loop(32, 16), 10),
    "blast_24x36_roe_15": ("blast", "roe", configs.blast(24, 36), 15),
    "blast_20x20_mixedbc_roe_12": ("blast", "roe", configs.blast(20, 20, bc=(1, 2, 2, 1)), 12),
    "cpaw2d_16x8_hlle_period": ("cpaw2d", "hlle", configs.cpaw2d(16, 8, flux="hlle"), None),
}


def main() -> None:
    for name, (problem, flux, blocks, steps) in FIXTURES.items():
        with tempfile.TemporaryDirectory() as td:
            ath = write_athinput(Path(td) / "athinput", blocks)
            text = ath.read_text()
            r = refutil.run_ref(problem, flux, ath, td, steps=steps)
        np.savez_compressed(HERE / f"{name}.npz", planes=r["planes"], dt=r["dt"], time=r["time"],
                            nstep=r["nstep"], problem=problem, flux=flux,
                            steps=-1 if steps is None else steps, athinput=text)
        print(name, r["nstep"], r["time"])


if __name__ == "__main__":
    main()
