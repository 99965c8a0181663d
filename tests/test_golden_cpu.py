"""The golden fixtures are what the reference CPU path produces today
(re-run here when the reference build is available)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES

GOLDEN = sorted((Path(__file__).parent / "golden").glob("*.npz"))


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_golden_matches_reference(path, tmp_path):
    f = np.load(path)
    problem, flux = str(f["problem"]), str(f["flux"])
    if not refutil.have_ref(problem, flux):
        pytest.skip("oracle/_ref not built")
    ath = tmp_path / "athinput"
    ath.write_text(str(f["athinput"]))
    steps = int(f["steps"])
    r = refutil.run_ref(problem, flux, ath, tmp_path, steps=None if steps < 0 else steps)
    assert refutil.mismatch_report(f["planes"], r["planes"], PLANES) == ""
    assert (r["nstep"], r["time"], r["dt"]) == (int(f["nstep"]), float(f["time"]), float(f["dt"]))
