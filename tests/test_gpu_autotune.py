"""GPU check of the autotuner: tuning a small batch returns valid launch parameters, and the batch
run with them gives the oracle's rows."""
import numpy as np
import pytest

from jhelp import dev_t
from oracle import oracle as O
from sirius_b200 import autotune as A
from sirius_b200 import batch as B

pytestmark = pytest.mark.gpu


def test_tune_batch_small(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("SJ_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    rng = np.random.default_rng(2)
    host, specs = [], []
    for j in range(24):
        nb = int(rng.integers(100, 20000))
        bk = rng.permutation(nb).astype(np.int32)
        pk = rng.integers(0, int(1.2 * nb), 10 * nb).astype(np.int32)
        host.append((bk, pk))
        specs.append(B.BatchJoinSpec(dev_t(bk, cuda), dev_t(pk, cuda)))
    best = A.tune_batch(specs, rounds=1)
    for k, space in A.BATCH_SPACE.items():
        assert best[k] in space
    assert A.tune_batch(specs) == best  # second call served from the cache
    with B.BatchPlan(specs, B.batch_params(**A._public(best))) as plan:
        plan.launch()
        counts, err = plan.counts()
        assert int(err.item()) == 0
        for (bk, pk), c in zip(host, counts.cpu().numpy()):
            assert c == O.hash_join_count(bk, pk)
