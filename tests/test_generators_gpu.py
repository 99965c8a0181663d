"""Initial conditions formed on the GPU (athb_generate, athb_batch_generate)
equal the host generators bit for bit -- and those equal the reference's
(tests/test_host_cpu.py) -- including after set_bvals and the first new_dt."""
from __future__ import annotations

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Batch, Grid, Params, configs, problem_state, write_athinput

pytestmark = pytest.mark.gpu

def _loop(nx1, nx2, rad=0.3, amp=1e-3):
    b = configs.field_loop(nx1, nx2)
    b["problem"]["rad"], b["problem"]["amp"] = rad, amp
    return b


CASES = [
    ("blast", configs.blast(60, 40, b0=1.5, angle=30.0, bc=(2, 2, 1, 1))),
    ("blast", configs.blast(33, 47, prat=1000.0, radius=0.15)),
    ("field_loop", _loop(50, 34)),
    ("field_loop", _loop(64, 64, rad=0.45, amp=2e-3)),
]


def _host_grid(name, blocks):
    p = Params.from_blocks(blocks)
    g = Grid.create(p.config())
    g.upload(problem_state(name, p))
    g.set_bvals()
    g.new_dt()
    return g


@pytest.mark.parametrize("name,blocks", CASES, ids=[f"{c[0]}-{i}" for i, c in enumerate(CASES)])
def test_device_generator_equals_host(name, blocks, tmp_path):
    dev = Grid.from_athinput(write_athinput(tmp_path / "athinput", blocks), name)  # device path
    host = _host_grid(name, blocks)
    a, b = dev.download(), host.download()
    assert refutil.mismatch_report(b[0], a[0], PLANES) == ""
    assert a[1:] == b[1:]
    # and one step later
    dev.run(1)
    host.run(1)
    assert refutil.mismatch_report(host.download()[0], dev.download()[0], PLANES) == ""
    dev.close()
    host.close()


def test_batch_device_generator_equals_upload():
    items = CASES + [("cpaw2d", configs.cpaw2d(16, 8))]  # cpaw2d: host upload path
    b_dev = Batch.from_problems(items)
    params = [Params.from_blocks(bl) for _, bl in items]
    b_host = Batch([p.config() for p in params])
    for k, ((name, _), p) in enumerate(zip(items, params)):
        b_host.upload(k, problem_state(name, p))
    b_host.prepare()
    for k in range(len(items)):
        x, y = b_dev.download(k), b_host.download(k)
        assert refutil.mismatch_report(y[0], x[0], PLANES) == ""
        assert x[1:] == y[1:]
    b_dev.close()
    b_host.close()
