"""The example athinput files parse with the reference's rules and name a
built-in problem generator the command-line driver can take from them."""
from __future__ import annotations

from pathlib import Path

import pytest

from athena_cuda_b200 import Params

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("name", ["blast", "field_loop", "cpaw2d"])
def test_example_parses(name):
    path = ROOT / "examples" / f"athinput.{name}"
    p = Params(path)
    cfg = p.config()
    assert cfg.nx1 > 0 and cfg.nx2 > 0 and cfg.tlim > 0 and cfg.gamma > 1
    text = path.read_text()
    assert f"config = --with-problem={name}" in text
    assert p.geti("job", "maxout") >= 1
