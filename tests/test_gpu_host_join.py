"""GPU parity of the one-shot join from host memory (sj_inner_join_host) against the CPU oracle:
the probe side streamed in many chunks (a partial last one), NULL keys on both sides with validity
words at chunk boundaries, DISTINCT and GROUPED tables, partitioned and not, composite keys, and
the capacity contract (rows past capacity not written, the full count reported)."""
import numpy as np
import pytest
import torch

from jhelp import assert_same_rows
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


def _h(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def _hv(v):
    return None if v is None else torch.from_numpy(v.view(np.int32)).pin_memory()


def _rows(out):
    c = out.count
    return [out.probe_rid[:c].numpy(), out.build_rid[:c].numpy()] + [t[:c].numpy() for t in out.probe_payload] + \
        [t[:c].numpy() for t in out.build_payload]


@pytest.mark.parametrize("pbits", [-1, 3])
@pytest.mark.parametrize("chunk", [65_536, 1 << 20])
def test_distinct_with_nulls_matches_oracle(cuda, pbits, chunk):
    rng = np.random.default_rng(21)
    nb, npr = 300_001, 1_000_003
    bk = rng.permutation(3 * nb)[:nb].astype(np.int64)
    pk = bk[rng.integers(0, nb, npr)]
    miss = rng.random(npr) < 0.2
    pk[miss] = 3 * nb + rng.integers(0, 1000, int(miss.sum()))
    bv = O.pack_validity(rng.random(nb) > 0.03)
    pv = O.pack_validity(rng.random(npr) > 0.05)
    pp = [rng.integers(-2**40, 2**40, npr).astype(np.int64)]
    bp = [rng.integers(-2**40, 2**40, nb).astype(np.int64), rng.integers(-2**31, 2**31 - 1, nb).astype(np.int32)]
    out = J.inner_join_host(_h(bk), _h(pk), _hv(bv), _hv(pv), [_h(c) for c in pp], [_h(c) for c in bp],
                            chunk_rows=chunk, partition_bits=pbits)
    r = O.hash_join(bk, pk, bv, pv, probe_payload=pp, build_payload=bp)
    assert out.count == r.rows
    assert_same_rows(_rows(out), [r.probe_rid, r.build_rid] + r.probe_payload + r.build_payload)


def test_grouped_composite_keys_match_oracle(cuda):
    rng = np.random.default_rng(22)
    nb, npr = 60_000, 400_001
    b = [rng.integers(0, 300, nb).astype(np.int32), rng.integers(-5, 40, nb).astype(np.int64)]
    p = [rng.integers(-3, 303, npr).astype(np.int32), rng.integers(-5, 42, npr).astype(np.int64)]
    bvw = [O.pack_validity(rng.random(nb) > 0.02), None]
    pvw = [None, O.pack_validity(rng.random(npr) > 0.02)]
    bi, pi, bvi, pvi = O.composite_keys(b, p, bvw, pvw)
    ref = O.hash_join(bi, pi, bvi, pvi, build_payload=[b[1]])
    out = J.inner_join_host([(_h(c), _hv(v)) for c, v in zip(b, bvw)], [(_h(c), _hv(v)) for c, v in zip(p, pvw)],
                            build_payload=[_h(b[1])], capacity=ref.rows, chunk_rows=50_000)
    assert out.count == ref.rows
    assert_same_rows(_rows(out), [ref.probe_rid, ref.build_rid] + ref.build_payload)


def test_capacity_reports_the_full_count(cuda):
    rng = np.random.default_rng(23)
    bk = np.arange(50_000, dtype=np.int64)
    pk = np.concatenate([bk, bk, bk])  # 150,000 matches
    rng.shuffle(pk)
    cap = 100_000
    out = J.JoinOutput(0, torch.full((cap,), -1, dtype=torch.int32).pin_memory(),
                       torch.full((cap,), -1, dtype=torch.int32).pin_memory(), [], [])
    with pytest.raises(L.SjError) as e:
        J.inner_join_host(_h(bk), _h(pk), capacity=cap, out=out, chunk_rows=40_000)
    assert "150000 matches" in str(e.value)
    # the rows that were written are real matches, each probe row at most once
    pr, br = out.probe_rid.numpy(), out.build_rid.numpy()
    assert np.all(pr >= 0) and np.all(pk[pr] == bk[br])
    assert len(np.unique(pr)) == cap


def test_empty_probe_and_empty_build(cuda):
    k = _h(np.arange(1000, dtype=np.int64))
    e = _h(np.zeros(0, dtype=np.int64))
    assert J.inner_join_host(k, e, capacity=0).count == 0
    assert J.inner_join_host(e, k).count == 0
