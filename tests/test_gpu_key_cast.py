"""GPU parity of single-column probe keys of the other integer type than the table's (the
reference's key casts, prepare_join_keys: src/op/sirius_physical_hash_join.cpp:1234-1291):
int32 probes into an int64 table widen exactly; int64 probes into an int32 table narrow in range
and never match out of range, without becoming NULL (LEFT, ANTI and MARK keep them as rows
without a match). Checked against the oracle on both sides widened to int64."""
import numpy as np
import pytest

from jhelp import assert_same_rows, dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


def _inputs(seed, build_dtype, probe_dtype, nb=60_000, npr=300_001):
    rng = np.random.default_rng(seed)
    bk = (rng.permutation(200_000)[:nb] - 100_000).astype(build_dtype)
    pk = rng.integers(-120_000, 120_000, npr).astype(np.int64)
    if probe_dtype == np.int64:  # values beyond the int32 range, some of them equal to a build key mod 2^32
        far = rng.random(npr) < 0.2
        pk[far] = bk[rng.integers(0, nb, int(far.sum()))].astype(np.int64) + (1 << 32) * rng.choice([-1, 1], int(far.sum()))
    pv = O.pack_validity(rng.random(npr) > 0.05)
    return bk, pk.astype(probe_dtype), pv


@pytest.mark.parametrize("build_dtype,probe_dtype", [(np.int64, np.int32), (np.int32, np.int64)])
@pytest.mark.parametrize("pbits", [-1, 3])
def test_inner_with_cast_probe_keys(cuda, build_dtype, probe_dtype, pbits):
    bk, pk, pv = _inputs(61, build_dtype, probe_dtype)
    bp = [np.arange(len(bk), dtype=np.int64) * 7]
    with J.HashTable(dev_t(bk, cuda), attach=[dev_t(bp[0], cuda)], partition_bits=pbits) as t:
        out = t.probe_gather(dev_t(pk, cuda), dev_valid(pv, cuda), attached=True).trimmed()
    r = O.hash_join(bk.astype(np.int64), pk.astype(np.int64), None, pv, build_payload=bp)
    got = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy(), out.build_payload[0].cpu().numpy()]
    assert_same_rows(got, [r.probe_rid, r.build_rid] + r.build_payload)


@pytest.mark.parametrize("kind", ["left", "anti", "semi"])
def test_outer_kinds_keep_out_of_range_rows_unmatched(cuda, kind):
    bk, pk, pv = _inputs(62, np.int32, np.int64)
    code = {"left": L.SJ_JOIN_LEFT, "anti": L.SJ_JOIN_ANTI, "semi": L.SJ_JOIN_SEMI}[kind]
    with J.HashTable(dev_t(bk, cuda)) as t:
        out = t.probe_join(code, dev_t(pk, cuda), dev_valid(pv, cuda))
    ep, eb = O.kind_join(kind, bk.astype(np.int64), pk, None, pv)
    gp = out.probe_rid[:out.count].cpu().numpy()
    if kind == "left":
        g = O.canonical(gp, out.build_rid[:out.count].cpu().numpy())
        e = O.canonical(ep, eb)
        assert np.array_equal(g[0], e[0]) and np.array_equal(g[1], e[1])
    else:
        assert np.array_equal(np.sort(gp), np.sort(ep))


def test_mark_of_out_of_range_rows_is_false_not_null(cuda):
    bk, pk, pv = _inputs(63, np.int32, np.int64)
    with J.HashTable(dev_t(bk, cuda)) as t:
        out = t.probe_join(L.SJ_JOIN_MARK, dev_t(pk, cuda), dev_valid(pv, cuda))
    m, v = O.mark_join(bk.astype(np.int64), pk, None, pv)
    assert np.array_equal(out.mark.cpu().numpy().astype(bool), m)
    assert np.array_equal(O.unpack_validity(out.mark_validity.cpu().numpy().view(np.uint32), len(pk)), v)


def test_narrowing_into_a_full_range_int32_table_is_refused(cuda):
    bk = np.array([-2**31, 0, 2**31 - 1], dtype=np.int32)
    with J.HashTable(dev_t(bk, cuda)) as t:
        with pytest.raises(L.SjError):
            t.probe_gather(dev_t(np.array([1, 2**40], dtype=np.int64), cuda), capacity=2)
        # widening the other way round is always exact
    with J.HashTable(dev_t(bk.astype(np.int64), cuda)) as t:
        out = t.probe_gather(dev_t(np.array([0, -2**31, 5], dtype=np.int32), cuda), capacity=3).trimmed()
        assert sorted(out.build_rid.cpu().numpy().tolist()) == [0, 1]
