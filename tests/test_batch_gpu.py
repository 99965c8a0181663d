"""Batched ensemble: independent grids of different sizes, parameters and
boundary conditions advanced by one persistent launch per step.  Every
instance must equal the single-grid stepper and the reference CPU path bit
for bit, and each must stop at its own end time."""
from __future__ import annotations

import numpy as np
import pytest

import refutil
from athena_cuda_b200 import PLANES, Batch, Grid, configs, ensemble, write_athinput

pytestmark = pytest.mark.gpu


def _items():
    items = ensemble.instances(6, seed=7, sizes=(8, 12, 16, 24, 40), tlim=0.06)
    # different boundary kinds and problems in the same batch
    items.append(("blast", configs.blast(20, 12, tlim=0.05, bc=(1, 2, 2, 1))))
    items.append(("field_loop", configs.field_loop(32, 16, tlim=0.04)))
    items.append(("cpaw2d", configs.cpaw2d(16, 8, tlim=0.05)))
    return items


def test_batch_matches_single_grid_and_reference(tmp_path):
    items = _items()
    b = Batch.from_problems(items)
    launches = b.run(10_000)
    assert launches > 0
    results = [b.download(k) for k in range(b.n)]
    b.close()
    nsteps = set()
    for k, (problem, blocks) in enumerate(items):
        planes, dt, t, n = results[k]
        assert t == blocks["time"]["tlim"], (k, t)
        nsteps.add(n)
        ath = write_athinput(tmp_path / f"a{k}", blocks)
        g = Grid.from_athinput(ath, problem)
        g.run(1_000_000)
        p2, dt2, t2, n2 = g.download()
        g.close()
        rep = refutil.mismatch_report(p2, planes, PLANES)
        assert rep == "", f"instance {k} differs from the single-grid run:\n{rep}"
        assert (n, t, dt) == (n2, t2, dt2)
        if refutil.have_ref(problem):
            ref = refutil.run_ref(problem, "roe", ath, tmp_path)
            assert refutil.mismatch_report(ref["planes"], planes, PLANES) == ""
            assert (n, t, dt) == (ref["nstep"], ref["time"], ref["dt"])
    assert len(nsteps) > 1, "instances should take different numbers of steps"


def test_batch_partial_runs_and_tuning_keep_results(tmp_path):
    """Re-tuned segment lengths and persistent grid sizes change only the
    schedule: results after the same number of launches are identical."""
    items = _items()[:5]
    ref = Batch.from_problems(items)
    ref.run(12)
    want = [ref.download(k)[0] for k in range(ref.n)]
    ref.close()
    b = Batch.from_problems(items)
    for k in range(b.n):
        b.set_ly(k, 4 + 3 * k)
    b.commit()
    b.set_grid(37)
    b.run_async(5)
    b.synchronize()
    b.run(7)
    for k in range(b.n):
        assert refutil.mismatch_report(want[k], b.download(k)[0], PLANES) == ""
    b.close()


def test_autotuner_returns_a_candidate():
    from athena_cuda_b200 import autotune

    ly, times = autotune.tune_class(40, nx1=24, launches=1)
    assert ly in autotune.LY_CANDIDATES and ly in times and all(t > 0 for t in times.values())


def test_phased_mode_matches_persistent():
    """One launch per phase gives the same bits as the persistent kernel."""
    items = _items()
    want = Batch.from_problems(items)
    assert want.mode == Batch.PHASED   # the default
    want.mode = Batch.PERSISTENT
    want.run(10_000)
    ref = [want.download(k) for k in range(want.n)]
    want.close()
    b = Batch.from_problems(items)
    b.mode = Batch.PHASED
    assert b.mode == Batch.PHASED
    b.timing(1)
    b.run(10_000)
    assert all(v >= 0.0 for v in b.timing(0).values())
    for k in range(b.n):
        planes, dt, t, n = b.download(k)
        assert refutil.mismatch_report(ref[k][0], planes, PLANES) == ""
        assert (dt, t, n) == ref[k][1:]
    b.close()


@pytest.mark.parametrize("mode", [Batch.PERSISTENT, Batch.PHASED])
def test_hlle_batch_matches_reference(mode, tmp_path):
    """A batch whose instances all use HLLE (src/flux_hlle.c) equals the
    reference CPU path built with flux_hlle, instance by instance."""
    items = ensemble.instances(4, seed=11, sizes=(8, 16, 24), tlim=0.04, flux="hlle")
    b = Batch.from_problems(items)
    b.mode = mode
    b.run(10_000)
    for k, (problem, blocks) in enumerate(items):
        planes, dt, t, n = b.download(k)
        if refutil.have_ref(problem, "hlle"):
            ref = refutil.run_ref(problem, "hlle", write_athinput(tmp_path / f"a{k}", blocks), tmp_path)
            assert refutil.mismatch_report(ref["planes"], planes, PLANES) == ""
            assert (n, t, dt) == (ref["nstep"], ref["time"], ref["dt"])
        else:
            g = Grid.from_athinput(write_athinput(tmp_path / f"a{k}", blocks), problem)
            g.run(1_000_000)
            assert refutil.mismatch_report(g.download()[0], planes, PLANES) == ""
            g.close()
    b.close()


@pytest.mark.parametrize("nt", [64, 256])
def test_threads_per_unit_give_the_same_bits(nt):
    """64- and 256-thread work units (the phased launches' block size, which
    the autotuner picks) give the 128-thread result bit for bit."""
    items = _items()
    want = Batch.from_problems(items)
    assert want.threads == 128
    want.run(10_000)
    ref = [want.download(k) for k in range(want.n)]
    want.close()
    b = Batch.from_problems(items)
    b.threads = nt
    for k in range(b.n):
        b.set_ly(k, 3 + 5 * k)
    b.commit()
    b.run(10_000)
    for k in range(b.n):
        planes, dt, t, n = b.download(k)
        assert refutil.mismatch_report(ref[k][0], planes, PLANES) == ""
        assert (dt, t, n) == ref[k][1:]
    from athena_cuda_b200 import AthbError
    with pytest.raises(AthbError, match="128-thread"):
        b.mode = Batch.PERSISTENT
    b.close()


def test_autotuner_picks_threads_and_segments(tmp_path):
    from athena_cuda_b200 import autotune

    items = _items()
    b = Batch.from_problems(items)
    sizes = [(bl["grid"]["Nx1"], bl["grid"]["Nx2"]) for _, bl in items]
    table = autotune.tune_batch(b, sizes, cache=tmp_path / "tune.json")
    assert table["threads"] in autotune.NT_CANDIDATES and b.threads == table["threads"]
    assert set(table["estimated_ms_per_launch_by_threads"]) == {"64", "128", "256"}
    b.close()
