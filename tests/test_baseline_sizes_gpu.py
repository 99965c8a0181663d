"""Bit-exact parity at the benchmark configurations' own sizes.

The smaller parity cases (test_parity_gpu.py) cover every branch; these cases
run the configurations the throughput numbers are quoted on, against the
reference CPU path compiled here (oracle/_ref), with zero tolerance on every
plane (ghosts included), dt, time and nstep:

* field-loop advection 1024x512 (10 steps) and 2048x2048 (2 steps)
  (src/field_loop.c:40-137);
* the circularly polarised Alfven wave at 256x128 and 512x256 over one full
  period, Roe and HLLE, together with the L1 errors the reference's
  Userwork_after_loop writes (src/cpaw2d.c:222-302);
* the 512-instance blast ensemble (seed 2024): every instance against the
  single-grid stepper at its own t = 0.1, and 16 instances spread over the
  size range against the reference (nlim-capped so the CPU side stays short).

The reference processes are started together at the beginning of the module
(one process each, in parallel) so the wall time is that of the longest.
"""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Batch, Grid, configs, ensemble, write_athinput

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

PLAIN = {
    # name: (problem, flux, blocks, steps)
    "field_loop_1024x512_10": ("field_loop", "roe", configs.field_loop(1024, 512), 10),
    "field_loop_2048x2048_2": ("field_loop", "roe", configs.field_loop(2048, 2048), 2),
    "cpaw2d_256x128_roe": ("cpaw2d", "roe", configs.cpaw2d(256, 128), None),
    "cpaw2d_256x128_hlle": ("cpaw2d", "hlle", configs.cpaw2d(256, 128, flux="hlle"), None),
    "cpaw2d_512x256_roe": ("cpaw2d", "roe", configs.cpaw2d(512, 256), None),
    "cpaw2d_512x256_hlle": ("cpaw2d", "hlle", configs.cpaw2d(512, 256, flux="hlle"), None),
}

ENSEMBLE_N, ENSEMBLE_SEED, ENSEMBLE_NLIM, ENSEMBLE_SAMPLES = 512, 2024, 12, 16


class _RefJob:
    """One reference CPU process started in the background."""

    def __init__(self, problem, flux, blocks, workdir: Path, steps=None, l1=False):
        workdir.mkdir(parents=True, exist_ok=True)
        self.workdir = workdir
        self.ath = write_athinput(workdir / "athinput", blocks)
        self.out = workdir / "ref.bin"
        cmd = [str(refutil.ref_binary(problem, flux)), "-i", str(self.ath), "--dump", str(self.out)]
        if steps is not None:
            cmd += ["--steps", str(steps)]
        if l1:
            cmd += ["--l1"]
        self.proc = subprocess.Popen(cmd, cwd=workdir, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)

    def result(self) -> dict:
        _, err = self.proc.communicate(timeout=900)
        assert self.proc.returncode == 0, err.decode()[-2000:]
        return refutil.read_raw(self.out)

    def l1_row(self) -> list[float]:
        row = [l for l in (self.workdir / "cpaw2d-errors.dat").read_text().splitlines()
               if not l.startswith("#")][-1]
        return [float(x) for x in row.split()[2:]]  # RMS d M1 M2 M3 E B1c B2c B3c


def _sampled(items) -> list[int]:
    """ENSEMBLE_SAMPLES instance indices spread over the cell-count range."""
    order = sorted(range(len(items)), key=lambda k: (items[k][1]["grid"]["Nx1"] * items[k][1]["grid"]["Nx2"], k))
    step = len(order) / ENSEMBLE_SAMPLES
    return [order[int(q * step)] for q in range(ENSEMBLE_SAMPLES - 1)] + [order[-1]]


def _capped(blocks: dict) -> dict:
    b = {k: dict(v) for k, v in blocks.items()}
    b["time"]["nlim"] = ENSEMBLE_NLIM
    return b


@pytest.fixture(scope="module")
def ref_jobs():
    missing = [p for p, f in {("field_loop", "roe"), ("cpaw2d", "roe"), ("cpaw2d", "hlle"), ("blast", "roe")}
               if not refutil.have_ref(p, f)]
    if missing:
        pytest.skip("oracle/_ref not built (python oracle/build_ref.py)")
    td = Path(tempfile.mkdtemp(prefix="athb_baseline_"))
    jobs = {}
    for name, (problem, flux, blocks, steps) in PLAIN.items():
        jobs[name] = _RefJob(problem, flux, blocks, td / name, steps=steps, l1=(problem == "cpaw2d"))
    items = ensemble.instances(ENSEMBLE_N, seed=ENSEMBLE_SEED)
    for k in _sampled(items):
        jobs[f"ens{k}"] = _RefJob("blast", "roe", _capped(items[k][1]), td / f"ens{k}")
    yield jobs
    for j in jobs.values():
        if j.proc.poll() is None:
            j.proc.kill()


def _compare(ref: dict, planes: np.ndarray, dt: float, t: float, n: int, what: str) -> None:
    rep = refutil.mismatch_report(ref["planes"], planes, PLANES)
    assert rep == "", f"{what}: state differs from the reference:\n{rep}"
    assert (n, t, dt) == (ref["nstep"], ref["time"], ref["dt"]), what


@pytest.mark.parametrize("name", list(PLAIN))
def test_plain_configuration_bit_exact(name, ref_jobs):
    problem, flux, blocks, steps = PLAIN[name]
    job = ref_jobs[name]
    g = Grid.from_athinput(job.ath, problem)
    g.run(steps if steps is not None else 1_000_000)
    planes, dt, t, n = g.download()
    l1 = g.cpaw2d_errors() if problem == "cpaw2d" else None
    g.close()
    _compare(job.result(), planes, dt, t, n, name)
    if l1 is not None:
        # the reference prints its errors with 6 significant digits (%e)
        theirs = job.l1_row()
        assert len(theirs) == 9
        for k, (mine, ref) in enumerate(zip(l1, theirs)):
            assert float(f"{mine:e}") == ref, (name, k, mine, ref)


def test_ensemble_512_every_instance_equals_single_grid():
    items = ensemble.instances(ENSEMBLE_N, seed=ENSEMBLE_SEED)
    b = Batch.from_problems(items)
    b.run(1_000_000)
    with tempfile.TemporaryDirectory() as td:
        for k, (problem, blocks) in enumerate(items):
            planes, dt, t, n = b.download(k)  # one at a time: the whole ensemble is ~2.5 GB on the host
            assert t == blocks["time"]["tlim"], (k, t)
            g = Grid.from_athinput(write_athinput(Path(td) / f"a{k}", blocks), problem)
            g.run(1_000_000)
            p2, dt2, t2, n2 = g.download()
            g.close()
            rep = refutil.mismatch_report(p2, planes, PLANES)
            assert rep == "", f"instance {k} differs from the single-grid run:\n{rep}"
            assert (n, t, dt) == (n2, t2, dt2), k
    b.close()


def test_ensemble_512_sampled_instances_equal_reference(ref_jobs):
    items = [(p, _capped(b)) for p, b in ensemble.instances(ENSEMBLE_N, seed=ENSEMBLE_SEED)]
    b = Batch.from_problems(items)
    b.run(1_000_000)
    sampled = _sampled(items)
    results = {k: b.download(k) for k in sampled}
    b.close()
    sizes = set()
    for k in sampled:
        planes, dt, t, n = results[k]
        assert n == ENSEMBLE_NLIM
        _compare(ref_jobs[f"ens{k}"].result(), planes, dt, t, n, f"instance {k}")
        sizes.add(items[k][1]["grid"]["Nx1"] * items[k][1]["grid"]["Nx2"])
    assert len(sizes) >= 8, sorted(sizes)
