"""The CPU oracle pinned against the reference's known answers, and its two restatements
(C chained hash join, numpy sort-merge) cross-checked on seeded inputs. No GPU needed."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = json.loads((Path(__file__).parent / "golden" / "join_known_answers.json").read_text())


def _col(values, dtype=np.int32):
    valid = np.array([v is not None for v in values], bool)
    data = np.array([0 if v is None else v for v in values], dtype)
    return data, O.pack_validity(valid)


def _fixture(dtype=np.int32):
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"], dtype)
    rk, rv = _col(fx["r"]["k"], dtype)
    lid = np.array(fx["l"]["id"], np.int32)
    rid = np.array(fx["r"]["id"], np.int32)
    return fx, lk, lv, rk, rv, lid, rid


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("threads", [1, 4])
def test_inner_known_answer_hash(dtype, threads):
    fx, lk, lv, rk, rv, lid, rid = _fixture(dtype)
    r = O.hash_join(rk, lk, rv, lv, probe_payload=[lid], build_payload=[rid], threads=threads)
    got = sorted(zip(r.probe_payload[0].tolist(), r.build_payload[0].tolist()))
    assert got == [tuple(p) for p in fx["inner"]]


def test_inner_known_answer_sort_merge():
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    pr, br = O.sort_merge_join(rk, lk, rv, lv)
    got = sorted(zip(lid[pr].tolist(), rid[br].tolist()))
    assert got == [tuple(p) for p in fx["inner"]]


def test_inner_where_probe_key_null_is_empty():
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    r = O.hash_join(rk, lk, rv, lv)
    lvalid = O.unpack_validity(lv, len(lk))
    assert not np.any(~lvalid[r.probe_rid])
    assert fx["inner_where_lk_null"] == []


def test_semi_anti_known_answers_from_inner_rows():
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    r = O.hash_join(rk, lk, rv, lv)
    matched = sorted(set(lid[r.probe_rid].tolist()))
    assert matched == fx["semi"]
    assert sorted(set(lid.tolist()) - set(matched)) == fx["anti"]


def test_null_safe_known_answer():
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    r = O.hash_join(rk, lk, rv, lv, nulls_equal=True)
    got = sorted(zip(lid[r.probe_rid].tolist(), rid[r.build_rid].tolist()))
    assert got == [tuple(p) for p in fx["inner_null_safe"]]
    pr, br = O.sort_merge_join(rk, lk, rv, lv, nulls_equal=True)
    assert sorted(zip(lid[pr].tolist(), rid[br].tolist())) == got


@pytest.mark.parametrize("case", GOLDEN["mark_cases"], ids=lambda c: c["name"])
def test_mark_cases_semi_set(case):
    """The MARK cases' TRUE rows are exactly the probe rows with an INNER match."""
    lk, lv = _col(case["left"])
    rk, rv = _col(case["right"]) if case["right"] else (np.zeros(0, np.int32), None)
    r = O.hash_join(rk, lk, rv, lv)
    matched = set(r.probe_rid.tolist())
    expect_true = {i for i, m in enumerate(case["mark"]) if m is True}
    assert matched == expect_true


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("nulls_equal", [False, True])
def test_hash_matches_sort_merge(seed, nulls_equal):
    rng = np.random.default_rng(seed)
    nb, np_ = 3000, 20000
    bk = rng.integers(-50, 500, nb).astype(np.int64)
    pk = rng.integers(-60, 600, np_).astype(np.int64)
    bv = O.pack_validity(rng.random(nb) > 0.1)
    pv = O.pack_validity(rng.random(np_) > 0.1)
    r = O.hash_join(bk, pk, bv, pv, nulls_equal=nulls_equal, threads=3)
    pr, br = O.sort_merge_join(bk, pk, bv, pv, nulls_equal=nulls_equal)
    a = O.canonical(r.probe_rid, r.build_rid)
    b = O.canonical(pr, br)
    assert len(a[0]) == len(b[0])
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert O.hash_join_count(bk, pk, bv, pv, nulls_equal=nulls_equal) == len(pr)


def test_capacity_truncates_but_reports_total():
    bk = np.array([1, 1, 1], np.int32)
    pk = np.array([1, 1], np.int32)
    r = O.hash_join(bk, pk, capacity=4)
    assert r.rows == 4
    assert O.hash_join_count(bk, pk) == 6


def test_payload_gather_and_checksum():
    rng = np.random.default_rng(7)
    bk = rng.permutation(1000).astype(np.int32)
    pk = rng.integers(0, 1100, 5000).astype(np.int32)
    bp = [rng.integers(-9, 9, 1000).astype(np.int64), rng.random(1000).astype(np.float32)]
    pp = [rng.integers(0, 100, 5000).astype(np.int16)]
    r = O.hash_join(bk, pk, probe_payload=pp, build_payload=bp)
    assert np.array_equal(r.build_payload[0], bp[0][r.build_rid])
    assert np.array_equal(r.build_payload[1], bp[1][r.build_rid])
    assert np.array_equal(r.probe_payload[0], pp[0][r.probe_rid])
    assert np.array_equal(bk[r.build_rid], pk[r.probe_rid])
    perm = rng.permutation(r.rows)
    c1 = O.multiset_checksum(r.probe_rid, r.build_rid, r.build_payload[0])
    c2 = O.multiset_checksum(r.probe_rid[perm], r.build_rid[perm], r.build_payload[0][perm])
    assert c1 == c2
    c3 = O.multiset_checksum(r.probe_rid, r.build_rid, r.build_payload[0] + 1)
    assert c3 != c1


def test_empty_sides():
    e32 = np.zeros(0, np.int32)
    assert O.hash_join_count(e32, np.array([1, 2], np.int32)) == 0
    assert O.hash_join_count(np.array([1, 2], np.int32), e32) == 0
    assert O.hash_join(e32, e32).rows == 0


def _pairs(pr, br, lid, rid):
    key = lambda x: (x[0] is None, x[0] or 0, x[1] is None, x[1] or 0)  # noqa: E731
    return sorted([(None if p == O.NO_ROW else int(lid[p]), None if b == O.NO_ROW else int(rid[b]))
                   for p, b in zip(pr, br)], key=key)


@pytest.mark.parametrize("kind", ["left", "full"])
def test_outer_known_answers(kind):
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    pr, br = O.kind_join(kind, rk, lk, rv, lv)
    exp = sorted([tuple(p) for p in fx[kind]], key=lambda x: (x[0] is None, x[0] or 0, x[1] is None, x[1] or 0))
    assert _pairs(pr, br, lid, rid) == exp


@pytest.mark.parametrize("kind", ["semi", "anti"])
def test_semi_anti_known_answers(kind):
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    pr, _ = O.kind_join(kind, rk, lk, rv, lv)
    assert sorted(lid[pr].tolist()) == fx[kind]


def test_mark_known_answers():
    fx, lk, lv, rk, rv, lid, rid = _fixture()
    m, v = O.mark_join(rk, lk, rv, lv)
    assert [[int(lid[i]), bool(m[i]) if v[i] else None] for i in range(len(lk))] == fx["mark_with_null_build"]
    keep = np.array([k is not None for k in fx["r"]["k"]])
    m, v = O.mark_join(rk[keep], lk, None, lv)
    assert [[int(lid[i]), bool(m[i]) if v[i] else None] for i in range(len(lk))] == fx["mark_null_free_build"]


@pytest.mark.parametrize("case", GOLDEN["mark_cases"], ids=lambda c: c["name"])
def test_mark_cases(case):
    lk, lv = _col(case["left"])
    rk, rv = _col(case["right"]) if case["right"] else (np.zeros(0, np.int32), None)
    m, v = O.mark_join(rk, lk, rv, lv)
    assert [bool(m[i]) if v[i] else None for i in range(len(lk))] == case["mark"]


def test_kind_join_partitions_the_probe_rows():
    """semi + anti = every probe row once; left rows = inner rows + anti rows."""
    rng = np.random.default_rng(5)
    bk = rng.integers(0, 300, 1000).astype(np.int64)
    pk = rng.integers(-20, 400, 4000).astype(np.int64)
    bv = O.pack_validity(rng.random(1000) > 0.1)
    pv = O.pack_validity(rng.random(4000) > 0.1)
    s, _ = O.kind_join("semi", bk, pk, bv, pv)
    a, _ = O.kind_join("anti", bk, pk, bv, pv)
    assert np.array_equal(np.sort(np.concatenate([s, a])), np.arange(4000))
    pr, br = O.kind_join("left", bk, pk, bv, pv)
    assert len(pr) == O.hash_join_count(bk, pk, bv, pv) + len(a)
    pr, br = O.kind_join("full", bk, pk, bv, pv)
    assert np.all(np.isin(np.arange(1000), br))  # every build row appears in a FULL join


def test_composite_keys_reduce_tuples_to_ids():
    b = [np.array([1, 1, 2, 2], np.int64), np.array([10, 20, 10, 20], np.int32)]
    p = [np.array([1, 2, 2, 3], np.int64), np.array([20, 10, 30, 10], np.int32)]
    bv = [None, O.pack_validity(np.array([True, True, False, True]))]
    bi, pi, bvw, pvw = O.composite_keys(b, p, bv, None)
    r = O.hash_join(bi, pi, bvw, pvw)
    pairs = sorted(zip(r.probe_rid.tolist(), r.build_rid.tolist()))
    assert pairs == [(0, 1)]  # (1,20) matches build row 1; build row 2 has a NULL component
    bi, pi, _, _ = O.composite_keys(b, p, bv, None, nulls_equal=True)
    r = O.hash_join(bi, pi)
    assert sorted(zip(r.probe_rid.tolist(), r.build_rid.tolist())) == [(0, 1)]
