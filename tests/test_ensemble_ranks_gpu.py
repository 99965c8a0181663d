"""An ensemble bin-packed over ranks (ensemble.partition, one Batch per rank,
no communication) gives every instance the same bits as one Batch of all of
them.  Two ranks share this one GPU here; their kernels never wait on each
other."""
from __future__ import annotations

import os
import pickle
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _items():
    sys.path.insert(0, str(ROOT))
    from athena_cuda_b200 import ensemble

    return ensemble.instances(7, seed=3, sizes=(12, 20, 28), tlim=0.03)


def _rank(rank, ranks, outdir):
    sys.path.insert(0, str(ROOT))
    from athena_cuda_b200 import Batch, ensemble

    items = _items()
    mine = ensemble.partition(items, ranks)[rank]
    b = Batch.from_problems([items[k] for k in mine])
    b.mode = Batch.PHASED
    b.run(100000)
    res = {k: b.download(i) for i, k in enumerate(mine)}
    b.close()
    (Path(outdir) / f"r{rank}.pkl").write_bytes(pickle.dumps(res))


def test_partitioned_equals_one_batch(tmp_path):
    from athena_cuda_b200 import Batch

    ranks = 2
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, ranks, str(tmp_path))) for r in range(ranks)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = {}
    for r in range(ranks):
        got.update(pickle.loads((tmp_path / f"r{r}.pkl").read_bytes()))
    items = _items()
    assert sorted(got) == list(range(len(items)))
    b = Batch.from_problems(items)
    b.run(100000)
    for k in range(len(items)):
        want = b.download(k)
        assert np.array_equal(got[k][0], want[0]) and got[k][1:] == want[1:], k
    b.close()
