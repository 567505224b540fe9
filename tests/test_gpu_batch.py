"""GPU parity of the batched persistent join: every join of a batch (uneven sizes, duplicates,
NULL keys, int32 and int64 keys) against the CPU oracle, bit-exact, for the persistent launch,
its CUDA-graph replay and the one-launch-per-join comparison path."""
import numpy as np
import pytest
import torch

from jhelp import dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import batch as B

pytestmark = pytest.mark.gpu


def _specs(dev, seed, n_joins, dtype, dup=True, nulls=True, pay=(np.int32, np.int64), max_build=6000):
    rng = np.random.default_rng(seed)
    host, specs = [], []
    for j in range(n_joins):
        nb = int(np.exp(rng.uniform(np.log(1), np.log(max_build))))
        npr = int(rng.integers(0, 4 * nb + 3))
        bk = (rng.integers(0, max(1, nb // 2), nb) if (dup and j % 3 == 0) else rng.permutation(nb)).astype(dtype)
        pk = rng.integers(-2, int(1.3 * nb) + 2, npr).astype(dtype)
        bv = O.pack_validity(rng.random(nb) > 0.1) if (nulls and j % 4 == 1) else None
        pv = O.pack_validity(rng.random(npr) > 0.1) if (nulls and j % 5 == 2) else None
        bp = rng.integers(0, 1 << 30, nb).astype(pay[0])
        pp = rng.integers(0, 1 << 40, npr).astype(pay[1])
        cnt = O.hash_join_count(bk, pk, bv, pv)
        host.append((bk, pk, bv, pv, bp, pp, cnt))
        specs.append(B.BatchJoinSpec(dev_t(bk, dev), dev_t(pk, dev), dev_t(bp, dev), dev_t(pp, dev),
                                     dev_valid(bv, dev), dev_valid(pv, dev), capacity=cnt))
    return host, specs


def _check(host, plan):
    counts, err = plan.counts()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    counts = counts.cpu().numpy()
    for (bk, pk, bv, pv, bp, pp, cnt), s, c in zip(host, plan.specs, counts):
        assert c == cnt
        ref = O.hash_join(bk, pk, bv, pv, probe_payload=[pp], build_payload=[bp])
        got = O.canonical(s.out.probe_rid[:c].cpu().numpy(), s.out.build_rid[:c].cpu().numpy(),
                          s.out.probe_payload[:c].cpu().numpy(), s.out.build_payload[:c].cpu().numpy())
        exp = O.canonical(ref.probe_rid, ref.build_rid, ref.probe_payload[0], ref.build_payload[0])
        for a, b in zip(got, exp):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("gw", [1, 2, 4, 8])
def test_batch_persistent_launch(cuda, dtype, gw):
    host, specs = _specs(cuda, 3 + gw, 48, dtype)
    with B.BatchPlan(specs, B.batch_params(group_width=gw, tile_rows=512)) as plan:
        plan.launch()
        _check(host, plan)


@pytest.mark.parametrize("block", [128, 512])
def test_batch_block_sizes_and_load_factor(cuda, block):
    host, specs = _specs(cuda, 17, 32, np.int32)
    with B.BatchPlan(specs, B.batch_params(block_size=block, load_factor=0.8, tile_rows=64)) as plan:
        plan.launch()
        _check(host, plan)


def test_batch_graph_replay_and_per_join(cuda):
    host, specs = _specs(cuda, 23, 40, np.int32)
    s = torch.cuda.Stream()
    with B.BatchPlan(specs, B.batch_params(tile_rows=1024), stream=s) as plan:
        for _ in range(3):   # capture once, replay three times: each replay resets and reruns the batch
            plan.replay(s)
        s.synchronize()
        _check(host, plan)
        plan.launch_per_join()
        _check(host, plan)


def test_batch_empty_joins(cuda):
    e = torch.zeros(0, dtype=torch.int32, device=cuda)
    k = torch.arange(100, dtype=torch.int32, device=cuda)
    specs = [B.BatchJoinSpec(e, k, capacity=0), B.BatchJoinSpec(k, e, capacity=0), B.BatchJoinSpec(k, k)]
    with B.BatchPlan(specs) as plan:
        plan.launch()
        counts, err = plan.counts()
        torch.cuda.synchronize()
        assert counts.tolist() == [0, 0, 100] and int(err.item()) == 0


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_batch_staged_output_shapes(cuda, width, dtype, block):
    """Both payloads of one width (4 or 8 bytes, no payload NULLs) and both row ids: the compile-time
    shape whose warps stage matches in shared memory and reserve output once per flush. Joins up to
    60K build rows (several flushes per warp), duplicates and NULL keys mixed in."""
    t = np.int32 if width == 4 else np.int64
    host, specs = _specs(cuda, 31 + width + block, 40, dtype, pay=(t, t), max_build=60_000)
    s = torch.cuda.Stream()
    with B.BatchPlan(specs, B.batch_params(block_size=block, tile_rows=4096), stream=s) as plan:
        plan.launch(s)
        s.synchronize()
        _check(host, plan)
        for _ in range(2):
            plan.replay(s)
        s.synchronize()
        _check(host, plan)
        plan.launch_per_join(s)
        s.synchronize()
        _check(host, plan)


SENTINEL, GUARD = -7, 512


def test_batch_staged_capacity_below_count(cuda):
    """Capacities below the match count: every count is still reported in full, nothing is written
    past a join's capacity, and the rows written are real matches."""
    rng = np.random.default_rng(77)
    host, specs = [], []
    for j in range(24):
        nb = int(rng.integers(1000, 40_000))
        bk = rng.permutation(nb).astype(np.int32)
        pk = rng.integers(0, nb, 8 * nb).astype(np.int32)   # every probe row matches
        bp = rng.integers(0, 1 << 30, nb).astype(np.int32)
        pp = rng.integers(0, 1 << 30, len(pk)).astype(np.int32)
        cap = int(len(pk) * rng.uniform(0.1, 0.95))
        # outputs with GUARD rows past the capacity, which must keep their SENTINEL
        out = B.BatchJoinOutput(*[torch.full((cap + GUARD,), SENTINEL, dtype=torch.int32, device=cuda)
                                  for _ in range(4)])
        sp = B.BatchJoinSpec(dev_t(bk, cuda), dev_t(pk, cuda), dev_t(bp, cuda), dev_t(pp, cuda), capacity=cap,
                             out=out)
        host.append((bk, pk, bp, pp, cap))
        specs.append(sp)
    with B.BatchPlan(specs, B.batch_params(tile_rows=4096)) as plan:
        plan.launch()
        counts, err = plan.counts()
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        for (bk, pk, bp, pp, cap), s, c in zip(host, plan.specs, counts.cpu().numpy()):
            assert c == len(pk)
            cols = [x.cpu().numpy() for x in (s.out.probe_rid, s.out.build_rid, s.out.probe_payload,
                                              s.out.build_payload)]
            for x in cols:
                assert (x[cap:] == SENTINEL).all(), "a row was written past the capacity"
            prid, brid, ppo, bpo = [x[:cap] for x in cols]
            assert np.array_equal(pk[prid], bk[brid])
            assert np.array_equal(ppo, pp[prid])
            assert np.array_equal(bpo, bp[brid])
            assert len(np.unique(prid)) == cap   # distinct probe rows, no row written twice
