"""Initial conditions formed on the GPU (athb_generate, athb_batch_generate)
equal the host generators bit for bit -- and those equal the reference's
(tests/test_host_cpu.py) -- including after set_bvals and the first new_dt.

The cpaw2d device generator (athb_generate_device) takes CUDA's sin/cos
(within 2 ulp) where the host generator takes libm's, so it is checked at a
stated tolerance: the momenta, B3 and the centred B3c to 8 ulp of the
plane's largest value; the face fields (differences of the vector potential
A3 over dx) and what is formed from them (B1c, B2c, E) to
8 * eps * max|A3| / dx: a cos a few ulp apart can move A3's rounding by an
ulp of A3, and the difference quotient carries that over dx."""
from __future__ import annotations

import numpy as np
import pytest

import refutil
import math

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


CPAW_SIZES = [(32, 16), (64, 32), (100, 50), (512, 256)]
EPS = np.finfo(np.float64).eps


def _cpaw_tolerances(blocks, nx1, nx2):
    dx = min(1.0 / nx1, 0.5 / nx2)
    k_par = 2.0 * math.pi * math.sqrt(5.0)   # wavelength 1/sqrt(5) on this box
    pr = blocks["problem"]
    a3max = pr["b_par"] * (1.0 + 0.5) + pr["b_perp"] / k_par   # |A3| on [0,1] x [0,0.5]
    return 8.0 * EPS * a3max / dx


@pytest.mark.parametrize("nx1,nx2", CPAW_SIZES, ids=[f"{a}x{b}" for a, b in CPAW_SIZES])
def test_cpaw2d_device_generator_within_tolerance(nx1, nx2):
    blocks = configs.cpaw2d(nx1, nx2)
    p = Params.from_blocks(blocks)
    host = problem_state("cpaw2d", p)
    g = Grid.create(p.config())
    g.generate_device("cpaw2d", p)
    dev = g.download()[0]
    face = _cpaw_tolerances(blocks, nx1, nx2)
    ng = 4
    sl = (slice(ng, ng + nx2 + 1), slice(ng, ng + nx1 + 1))   # faces up to ie+1, je+1
    cells = (slice(ng, ng + nx2), slice(ng, ng + nx1))
    worst = {}
    for k, name in enumerate(PLANES):
        region = sl if k >= 8 else cells
        a, b = dev[k][region], host[k][region]
        if name in ("B1i", "B2i", "B1c", "B2c"):
            tol = face
        elif name == "E":
            tol = 4.0 * face * max(1.0, float(np.max(np.abs(host[5][cells]))))
        else:
            tol = 8.0 * EPS * max(float(np.max(np.abs(b))), 1e-300)
        err = float(np.max(np.abs(a - b)))
        worst[name] = err / tol
        assert err <= tol, (name, err, tol)
    # the ghost zones stay zero, as a fresh host array leaves them
    assert not dev[0][:ng].any() and not dev[0][:, :ng].any()
    print({k: round(v, 3) for k, v in worst.items()})
    g.close()


def test_cpaw2d_device_generator_one_period_same_l1(tmp_path):
    """One period from the device-formed state: the L1 error against its own
    initial state agrees with the host-formed run's to 6 digits."""
    blocks = configs.cpaw2d(64, 32)
    ath = write_athinput(tmp_path / "athinput", blocks)
    p = Params(ath)
    e = []
    for device in (False, True):
        g = Grid.create(p.config())
        (g.generate_device if device else g.generate)("cpaw2d", p)
        g.set_bvals()
        g.new_dt()
        g.run(1_000_000)
        e.append(g.cpaw2d_errors())
        g.close()
    np.testing.assert_allclose(e[1], e[0], rtol=1e-6)


def test_batch_cpaw2d_generator_matches_grid_device_generator():
    blocks = [configs.cpaw2d(32, 16), configs.cpaw2d(48, 24)]
    params = [Params.from_blocks(b) for b in blocks]
    b = Batch([p.config() for p in params])
    for k, p in enumerate(params):
        b.generate(k, "cpaw2d", p)
    b.prepare()
    for k, p in enumerate(params):
        g = Grid.create(p.config())
        g.generate_device("cpaw2d", p)
        g.set_bvals()
        g.new_dt()
        x, y = b.download(k), g.download()
        assert refutil.mismatch_report(y[0], x[0], PLANES) == ""
        assert x[1:] == y[1:]
        g.close()
    b.close()


@pytest.mark.parametrize("name,blocks", CASES[::2], ids=["blast", "field_loop"])
def test_generate_device_equals_generate(name, blocks):
    """athb_generate_device forms blast and the field loop exactly as
    athb_generate does (both on the GPU, bit-identical to the host)."""
    p = Params.from_blocks(blocks)
    a, b = Grid.create(p.config()), Grid.create(p.config())
    a.generate(name, p)
    b.generate_device(name, p)
    x, y = a.download(), b.download()
    assert np.array_equal(x[0], y[0]) and x[1:] == y[1:]
    a.close()
    b.close()
