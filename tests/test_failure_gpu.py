"""Failure detection without a GPU fault: the persistent kernel's bounded
barrier wait runs out and reports instead of hanging, and a non-finite state
is reported as ATHB_ERR_STATE by a single grid and by a batch (the device's
CFL check sets an error flag that the host reads).  Every case leaves the
device usable."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from athena_cuda_b200 import AthbError, Batch, Grid, configs, ensemble, lib, write_athinput

pytestmark = pytest.mark.gpu


def _usable(tmp_path):
    g = Grid.from_athinput(write_athinput(tmp_path / "ok", configs.field_loop(16, 8)), "field_loop")
    g.run(3)
    assert g.status()["nstep"] == 3
    g.close()


def test_barrier_wait_runs_out_and_reports(tmp_path):
    f = lib().athb_batch_selftest_barrier
    f.restype, f.argtypes = C.c_int, [C.c_int, C.c_longlong, C.POINTER(C.c_int)]
    out = C.c_int(-1)
    t0 = time.perf_counter()
    assert f(0, 1_000_000, C.byref(out)) == 0, lib().athb_last_error().decode()
    assert out.value == 1  # the wait gave up
    assert time.perf_counter() - t0 < 60.0
    _usable(tmp_path)


def test_non_finite_state_is_reported(tmp_path):
    g = Grid.from_athinput(write_athinput(tmp_path / "a", configs.field_loop(32, 16)), "field_loop")
    planes, dt, t, n = g.download()
    planes[0, 10, 10] = np.nan  # density of one interior cell
    g.upload(planes, dt, t, n)
    with pytest.raises(AthbError) as e:
        g.run(5)
    assert e.value.code == 3 and "non-finite" in str(e.value)
    g.close()
    _usable(tmp_path)


def test_batch_reports_the_non_finite_instance(tmp_path):
    items = ensemble.instances(3, seed=1, sizes=(12, 16), tlim=0.02)
    b = Batch.from_problems(items)
    planes, dt, t, n = b.download(1)
    planes[0, 6, 6] = np.nan  # density of one interior cell (a bad energy alone is floored by P >= 1e-20)
    b.upload(1, planes, dt, t, n)
    with pytest.raises(AthbError) as e:
        b.run(1000)
    assert e.value.code == 3 and "instance 1" in str(e.value)
    b.close()
    _usable(tmp_path)
