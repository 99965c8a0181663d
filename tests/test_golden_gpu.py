"""GPU step against the committed golden fixtures (outputs of the reference's
own CPU path, tests/golden/make_golden.py): bit-exact, no reference build needed."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Grid

pytestmark = pytest.mark.gpu
GOLDEN = sorted((Path(__file__).parent / "golden").glob("*.npz"))


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_golden_bit_exact(path, tmp_path):
    f = np.load(path)
    ath = tmp_path / "athinput"
    ath.write_text(str(f["athinput"]))
    g = Grid.from_athinput(ath, str(f["problem"]))
    steps = int(f["steps"])
    g.run(steps if steps >= 0 else 1_000_000)
    planes, dt, t, n = g.download()
    g.close()
    rep = refutil.mismatch_report(f["planes"], planes, PLANES)
    assert rep == "", rep
    assert (n, t, dt) == (int(f["nstep"]), float(f["time"]), float(f["dt"]))
