"""The partitioned probe's output contract at sizes that take the tile-local partition and the
run-walking probe: the output against the oracle, under both output reservations (AUTO and one
atomicAdd per CTA chunk), at match rates from none to all, with capacities equal to the match
count, above it and below it. Below it the full count is reported, nothing past the capacity is
written, and every row written is a real match."""
import numpy as np
import pytest
import torch

from jhelp import assert_same_rows, dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import datagen as D
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu
SENTINEL = -7


def _input(n_build, n_probe, hit, null_frac, seed, four_byte=False):
    r = np.random.default_rng(seed)
    bk = (r.permutation(n_build * 3)[:n_build]).astype(np.int64)
    pk = np.where(r.random(n_probe) < hit, bk[r.integers(0, n_build, n_probe)],
                  n_build * 3 + r.integers(0, n_build, n_probe)).astype(np.int64)
    pv = O.pack_validity(r.random(n_probe) >= null_frac) if null_frac else None
    t = np.int32 if four_byte else np.int64
    bp = [r.integers(-2**30, 2**30, n_build).astype(t) for _ in range(2)]
    pp = [r.integers(-2**30, 2**30, n_probe).astype(t)]
    return D.JoinInput(f"blocks{seed}", bk, pk, bp, pp, None, pv)


def _run(inp, cuda, aggregation, capacity=None, attach=True, guard=0):
    bk, pk = dev_t(inp.build_keys, cuda), dev_t(inp.probe_keys, cuda)
    pv = dev_valid(inp.probe_validity, cuda)
    bp = [dev_t(c, cuda) for c in inp.build_payload]
    pp = [dev_t(c, cuda) for c in inp.probe_payload]
    with J.HashTable(bk, attach=bp if attach else (), partition_bits=4, aggregation=aggregation) as t:
        assert t.info().partition_bits == 4
        cap = len(inp.probe_keys) if capacity is None else capacity
        out = J.allocate_output(cap + guard, pp, bp, cuda)
        for c in [out.probe_rid, out.build_rid] + list(out.probe_payload) + list(out.build_payload):
            c.fill_(SENTINEL)
        d = torch.zeros(1, dtype=torch.int64, device=cuda)
        if attach:
            t.probe_gather(pk, pv, pp, attached=True, out=out, capacity=cap, d_count=d, sync=False)
        else:
            t.probe_gather(pk, pv, pp, bp, out=out, capacity=cap, d_count=d, sync=False)
        torch.cuda.synchronize()
    m = int(d.item())
    cols = [out.probe_rid, out.build_rid] + list(out.probe_payload) + list(out.build_payload)
    if guard:
        for c in cols:
            assert bool((c[cap:] == SENTINEL).all()), "a row was written past the capacity"
    return m, [c[:min(m, cap)].cpu().numpy() for c in cols]


@pytest.mark.parametrize("n_probe", [65_536, 300_001, 2_000_000])
@pytest.mark.parametrize("hit", [0.0, 0.003, 0.5, 1.0])
def test_partitioned_probe_matches_oracle(cuda, n_probe, hit):
    inp = _input(200_000, n_probe, hit, 0.0, seed=n_probe + int(hit * 1000))
    ref = O.hash_join(inp.build_keys, inp.probe_keys, None, inp.probe_validity, probe_payload=inp.probe_payload,
                      build_payload=inp.build_payload)
    exp = [ref.probe_rid, ref.build_rid] + ref.probe_payload + ref.build_payload
    m, got = _run(inp, cuda, L.SJ_AGG_AUTO, guard=4096)
    assert m == len(exp[0])
    assert_same_rows(got, exp)
    m2, cta = _run(inp, cuda, L.SJ_AGG_CTA)
    assert m2 == m
    assert_same_rows(cta, exp)


@pytest.mark.parametrize("extra", [0, 1, 12_345])
def test_capacity_at_and_above_the_count(cuda, extra):
    """Capacity M, M + 1 and M + 12,345, with 5 % NULL probe keys."""
    inp = _input(150_000, 1_000_000, 0.9, 0.05, seed=11)
    ref = O.hash_join(inp.build_keys, inp.probe_keys, None, inp.probe_validity, probe_payload=inp.probe_payload,
                      build_payload=inp.build_payload)
    exp = [ref.probe_rid, ref.build_rid] + ref.probe_payload + ref.build_payload
    m, got = _run(inp, cuda, L.SJ_AGG_AUTO, capacity=ref.rows + extra, guard=2048)
    assert m == ref.rows
    assert_same_rows(got, exp)


def test_caller_payloads_of_four_bytes(cuda):
    """The run-time output shape: 4-byte caller payloads gathered by build row id."""
    inp = _input(120_000, 700_000, 0.7, 0.0, seed=5, four_byte=True)
    ref = O.hash_join(inp.build_keys, inp.probe_keys, probe_payload=inp.probe_payload,
                      build_payload=inp.build_payload)
    exp = [ref.probe_rid, ref.build_rid] + ref.probe_payload + ref.build_payload
    m, got = _run(inp, cuda, L.SJ_AGG_AUTO, attach=False, guard=1024)
    assert m == ref.rows
    assert_same_rows(got, exp)


@pytest.mark.parametrize("frac", [0.5, 0.999])
def test_capacity_below_the_count(cuda, frac):
    """M > capacity: the full count is reported and nothing past the capacity is written; every
    row that was written below the capacity is a real match."""
    inp = _input(100_000, 500_000, 1.0, 0.0, seed=3)
    ref_rows = len(inp.probe_keys)
    cap = int(ref_rows * frac)
    m, got = _run(inp, cuda, L.SJ_AGG_AUTO, capacity=cap, guard=4096)
    assert m == ref_rows
    prid, brid = got[0], got[1]
    written = prid != SENTINEL
    assert written.sum() > 0
    assert np.array_equal(inp.probe_keys[prid[written]], inp.build_keys[brid[written]])
