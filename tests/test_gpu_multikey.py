"""GPU parity of composite (multi-column) equi-join keys against the CPU oracle: 2..4 key columns
packed into one 64-bit key, DISTINCT and GROUPED tables, partitioned and not, NULL components under
both NULL rules, probe values outside the build's ranges, every join type; and the refusal of key
ranges that do not pack into 63 bits."""
import numpy as np
import pytest
import torch

from jhelp import assert_same_rows, dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


def _cols(seed, nb, npr, dup, dtypes=(np.int32, np.int32), nulls=True):
    rng = np.random.default_rng(seed)
    b, p, bv, pv = [], [], [], []
    for c, dt in enumerate(dtypes):
        span = 60 if dup else 400
        off = -7 if c == 0 else 1_000_000_000 * (dt == np.int64)
        b.append((rng.integers(0, span, nb) + off).astype(dt))
        p.append((rng.integers(-5, span + 5, npr) + off).astype(dt))  # some values outside the build range
        bv.append(O.pack_validity(rng.random(nb) > 0.05) if nulls else None)
        pv.append(O.pack_validity(rng.random(npr) > 0.05) if nulls else None)
    if not dup:  # unique build tuples: keep the first row of each tuple
        _, first = np.unique(np.stack([x.astype(np.int64) for x in b], axis=1), axis=0, return_index=True)
        keep = np.sort(first)
        b = [x[keep] for x in b]
        bv = [None] * len(b) if not nulls else [O.pack_validity(np.ones(len(keep), bool)) for _ in b]
    return b, p, bv, pv


def _pairs(cols, valid, dev):
    return [(dev_t(c, dev), dev_valid(v, dev)) for c, v in zip(cols, valid)]


@pytest.mark.parametrize("dup", [False, True])
@pytest.mark.parametrize("pbits", [-1, 3])
@pytest.mark.parametrize("dtypes", [(np.int32, np.int32), (np.int64, np.int32, np.int32)])
def test_composite_inner(cuda, dup, pbits, dtypes):
    b, p, bv, pv = _cols(41 + dup, 50_000, 200_003, dup, dtypes)
    bi, pi, bvw, pvw = O.composite_keys(b, p, bv, pv)
    rng = np.random.default_rng(3)
    bp = [rng.integers(0, 1 << 40, len(b[0])).astype(np.int64)]
    pp = [rng.integers(0, 1 << 30, len(p[0])).astype(np.int32)]
    with J.HashTable(_pairs(b, bv, cuda), partition_bits=pbits) as t:
        out = t.probe_gather(_pairs(p, pv, cuda), None, [dev_t(pp[0], cuda)], [dev_t(bp[0], cuda)]).trimmed()
    got = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy(), out.probe_payload[0].cpu().numpy(),
           out.build_payload[0].cpu().numpy()]
    r = O.hash_join(bi, pi, bvw, pvw, probe_payload=pp, build_payload=bp)
    assert_same_rows(got, [r.probe_rid, r.build_rid] + r.probe_payload + r.build_payload)


@pytest.mark.parametrize("kind", ["left", "semi", "anti"])
def test_composite_join_kinds(cuda, kind):
    b, p, bv, pv = _cols(51, 30_000, 120_001, True)
    bi, pi, bvw, pvw = O.composite_keys(b, p, bv, pv)
    code = {"left": L.SJ_JOIN_LEFT, "semi": L.SJ_JOIN_SEMI, "anti": L.SJ_JOIN_ANTI}[kind]
    with J.HashTable(_pairs(b, bv, cuda)) as t:
        out = t.probe_join(code, _pairs(p, pv, cuda))
    ep, eb = O.kind_join(kind, bi, pi, bvw, pvw)
    gp = out.probe_rid[:out.count].cpu().numpy()
    if kind == "left":
        gb = out.build_rid[:out.count].cpu().numpy()
        g, e = O.canonical(gp, gb), O.canonical(ep, eb)
        assert np.array_equal(g[0], e[0]) and np.array_equal(g[1], e[1])
    else:
        assert np.array_equal(np.sort(gp), np.sort(ep))


def test_composite_mark(cuda):
    b, p, bv, pv = _cols(52, 20_000, 80_001, True)
    bi, pi, bvw, pvw = O.composite_keys(b, p, bv, pv)
    with J.HashTable(_pairs(b, bv, cuda)) as t:
        out = t.probe_join(L.SJ_JOIN_MARK, _pairs(p, pv, cuda))
    m, v = O.mark_join(bi, pi, bvw, pvw)
    assert np.array_equal(out.mark.cpu().numpy().astype(bool), m)
    assert np.array_equal(O.unpack_validity(out.mark_validity.cpu().numpy().view(np.uint32), len(pi)), v)


def test_composite_nulls_equal(cuda):
    b, p, bv, pv = _cols(53, 20_000, 80_001, True)
    bi, pi, _, _ = O.composite_keys(b, p, bv, pv, nulls_equal=True)
    with J.HashTable(_pairs(b, bv, cuda), null_equality=L.SJ_NULLS_EQUAL) as t:
        out = t.probe_gather(_pairs(p, pv, cuda)).trimmed()
    r = O.hash_join(bi, pi)
    assert_same_rows([out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()], [r.probe_rid, r.build_rid])


def test_composite_refuses_unpackable_ranges(cuda):
    rng = np.random.default_rng(1)
    b = [rng.integers(-2**62, 2**62, 1000), rng.integers(-2**62, 2**62, 1000)]
    with pytest.raises(L.SjError):
        J.HashTable([dev_t(c, cuda) for c in b])


def test_probe_key_count_must_match(cuda):
    b = [np.arange(100, dtype=np.int32), np.arange(100, dtype=np.int32)]
    with J.HashTable([dev_t(c, cuda) for c in b]) as t:
        with pytest.raises(L.SjError):
            t.probe_gather(dev_t(b[0], cuda))
