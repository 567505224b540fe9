"""GPU parity of LEFT / SEMI / ANTI / MARK / FULL (``sj_probe_join``) and of the RIGHT family
(``join.right_join``: the sides swapped, as the reference's STANDARD mode runs RIGHT / RIGHT_SEMI /
RIGHT_ANTI) against the CPU oracle:
the reference's own known answers (NULL fixture and the MARK operator cases), then seeded inputs
over DISTINCT and GROUPED tables, int32 and int64 keys, partitioned and unpartitioned tables,
NULL keys on both sides and NULL payloads — row ids bit-exact after a canonical sort, gathered
payloads and their validity equal row by row, MARK bytes and validity bits equal."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from jhelp import dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "join_known_answers.json").read_text())
KINDS = {"left": L.SJ_JOIN_LEFT, "full": L.SJ_JOIN_FULL, "semi": L.SJ_JOIN_SEMI, "anti": L.SJ_JOIN_ANTI}


def _col(values, dtype=np.int32):
    valid = np.array([v is not None for v in values], bool)
    return np.array([0 if v is None else v for v in values], dtype), O.pack_validity(valid)


def _bits(words, n):
    return O.unpack_validity(words.cpu().numpy().view(np.uint32), n)


def _check_rows(kind, out, bk, pk, bv, pv, bp, pp, bpv=None, ppv=None):
    n = out.count
    ep, eb = O.kind_join(kind, bk, pk, bv, pv)
    gp = out.probe_rid[:n].cpu().numpy()
    if kind in ("semi", "anti"):
        assert np.array_equal(np.sort(gp), np.sort(ep))
        for c, col in enumerate(pp):
            vals = out.probe_payload[c][:n].cpu().numpy()
            assert np.array_equal(vals, col[gp])
        return
    gb = out.build_rid[:n].cpu().numpy()
    g = O.canonical(gp, gb, np.arange(n))
    e = O.canonical(ep, eb)
    assert np.array_equal(g[0], e[0]) and np.array_equal(g[1], e[1])
    order = g[2]
    for c, col in enumerate(bp):
        ev, em = O.gather_nullable(col, g[1], bpv[c] if bpv else None)
        gv = out.build_payload[c][:n].cpu().numpy()[order]
        gm = _bits(out.build_payload_validity[c], n)[order]
        assert np.array_equal(gm, em), f"build payload {c} validity differs"
        assert np.array_equal(gv[gm], ev[em]), f"build payload {c} values differ"
    for c, col in enumerate(pp):
        ev, em = O.gather_nullable(col, g[0], ppv[c] if ppv else None)
        gv = out.probe_payload[c][:n].cpu().numpy()[order]
        if out.probe_payload_validity[c] is not None:
            gm = _bits(out.probe_payload_validity[c], n)[order]
            assert np.array_equal(gm, em), f"probe payload {c} validity differs"
        else:
            assert em.all()
            gm = em
        assert np.array_equal(gv[gm], ev[em]), f"probe payload {c} values differ"


@pytest.mark.parametrize("kind", list(KINDS))
def test_known_answers_nulls_fixture(cuda, kind):
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"])
    rk, rv = _col(fx["r"]["k"])
    lid = np.array(fx["l"]["id"], np.int32)
    rid = np.array(fx["r"]["id"], np.int32)
    with J.HashTable(dev_t(rk, cuda), dev_valid(rv, cuda)) as t:
        bp = [dev_t(rid, cuda)] if kind in ("left", "full") else []
        out = t.probe_join(KINDS[kind], dev_t(lk, cuda), dev_valid(lv, cuda), [dev_t(lid, cuda)], bp)
    n = out.count
    gp = out.probe_rid[:n].cpu().numpy()
    if kind in ("semi", "anti"):
        assert sorted(lid[gp].tolist()) == fx[kind]
        return
    gb = out.build_rid[:n].cpu().numpy()
    got = [(None if p == O.NO_ROW else int(lid[p]), None if b == O.NO_ROW else int(rid[b])) for p, b in zip(gp, gb)]
    key = lambda x: (x[0] is None, x[0] or 0, x[1] is None, x[1] or 0)  # noqa: E731
    assert sorted(got, key=key) == sorted([tuple(x) for x in fx[kind]], key=key)
    # the gathered id payloads say the same thing, with NULL where the side is missing
    bvals = out.build_payload[0][:n].cpu().numpy()
    bmask = _bits(out.build_payload_validity[0], n)
    pmask = _bits(out.probe_payload_validity[0], n) if out.probe_payload_validity[0] is not None else np.ones(n, bool)
    pvals = out.probe_payload[0][:n].cpu().numpy()
    via_payload = [(int(pv) if pm else None, int(bv) if bm else None) for pv, pm, bv, bm in zip(pvals, pmask, bvals, bmask)]
    assert sorted(via_payload, key=key) == sorted([tuple(x) for x in fx[kind]], key=key)


def test_known_answers_mark(cuda):
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"])
    lid = fx["l"]["id"]
    for name, rvals in (("mark_with_null_build", fx["r"]["k"]),
                        ("mark_null_free_build", [v for v in fx["r"]["k"] if v is not None])):
        rk, rv = _col(rvals)
        with J.HashTable(dev_t(rk, cuda), dev_valid(rv, cuda)) as t:
            out = t.probe_join(L.SJ_JOIN_MARK, dev_t(lk, cuda), dev_valid(lv, cuda))
        m = out.mark.cpu().numpy()
        v = _bits(out.mark_validity, len(lk))
        assert [[lid[i], bool(m[i]) if v[i] else None] for i in range(len(lk))] == fx[name]


@pytest.mark.parametrize("case", GOLDEN["mark_cases"], ids=lambda c: c["name"])
def test_mark_operator_cases(cuda, case):
    lk, lv = _col(case["left"])
    if case["right"]:
        rk, rv = _col(case["right"])
    else:
        rk, rv = np.zeros(0, np.int32), None
    with J.HashTable(dev_t(rk, cuda), dev_valid(rv, cuda)) as t:
        out = t.probe_join(L.SJ_JOIN_MARK, dev_t(lk, cuda), dev_valid(lv, cuda))
    m = out.mark.cpu().numpy()
    v = _bits(out.mark_validity, len(lk))
    assert [bool(m[i]) if v[i] else None for i in range(len(lk))] == case["mark"]


def _seeded(seed, dtype, dup, nulls):
    rng = np.random.default_rng(seed)
    nb, np_ = 40_000, 150_001
    bk = (rng.integers(0, nb // 3, nb) if dup else rng.permutation(nb * 2)[:nb]).astype(dtype)
    pk = rng.integers(-100, int(nb * (0.7 if dup else 2.4)), np_).astype(dtype)
    bv = O.pack_validity(rng.random(nb) > 0.07) if nulls else None
    pv = O.pack_validity(rng.random(np_) > 0.05) if nulls else None
    bp = [rng.integers(-2**31, 2**31 - 1, nb).astype(np.int32), rng.integers(-2**40, 2**40, nb).astype(np.int64)]
    bpv = [O.pack_validity(rng.random(nb) > 0.2) if nulls else None, None]
    pp = [rng.integers(-2**40, 2**40, np_).astype(np.int64)]
    return bk, pk, bv, pv, bp, bpv, pp


@pytest.mark.parametrize("kind", list(KINDS) + ["mark"])
@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("dup", [False, True])
@pytest.mark.parametrize("pbits", [-1, 3])
def test_kinds_match_oracle(cuda, kind, dtype, dup, pbits):
    bk, pk, bv, pv, bp, bpv, pp = _seeded(21 + dup, dtype, dup, nulls=True)
    bpd = [(dev_t(c, cuda), dev_valid(v, cuda)) for c, v in zip(bp, bpv)]
    with J.HashTable(dev_t(bk, cuda), dev_valid(bv, cuda), partition_bits=pbits) as t:
        if kind == "mark":
            out = t.probe_join(L.SJ_JOIN_MARK, dev_t(pk, cuda), dev_valid(pv, cuda))
            m, v = O.mark_join(bk, pk, bv, pv)
            assert np.array_equal(out.mark.cpu().numpy().astype(bool), m)
            assert np.array_equal(_bits(out.mark_validity, len(pk)), v)
            return
        out = t.probe_join(KINDS[kind], dev_t(pk, cuda), dev_valid(pv, cuda), [dev_t(c, cuda) for c in pp],
                           bpd if kind in ("left", "full") else [])
    _check_rows(kind, out, bk, pk, bv, pv, bp if kind in ("left", "full") else [], pp,
                bpv if kind in ("left", "full") else None)


@pytest.mark.parametrize("dup", [False, True])
def test_left_with_attached_payloads(cuda, dup):
    bk, pk, bv, pv, bp, bpv, pp = _seeded(31 + dup, np.int64, dup, nulls=True)
    with J.HashTable(dev_t(bk, cuda), dev_valid(bv, cuda), partition_bits=3,
                     attach=[(dev_t(c, cuda), dev_valid(v, cuda)) for c, v in zip(bp, bpv)]) as t:
        out = t.probe_join(L.SJ_JOIN_LEFT, dev_t(pk, cuda), dev_valid(pv, cuda), [dev_t(c, cuda) for c in pp],
                           attached=True)
    _check_rows("left", out, bk, pk, bv, pv, bp, pp, bpv)


def test_full_rejects_attached_payloads(cuda):
    bk = np.arange(100, dtype=np.int64)
    with J.HashTable(dev_t(bk, cuda), attach=[dev_t(bk, cuda)]) as t:
        with pytest.raises(L.SjError):
            t.probe_join(L.SJ_JOIN_FULL, dev_t(bk, cuda), attached=True)


def test_right_join_known_answer(cuda):
    """RIGHT JOIN of the NULL fixture (test_gpu_execution_join_nulls.cpp:67-72): every right row,
    with its left matches or a NULL left side."""
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"])
    rk, rv = _col(fx["r"]["k"])
    lid = np.array(fx["l"]["id"], np.int32)
    rid = np.array(fx["r"]["id"], np.int32)
    out = J.right_join(J.JOIN_RIGHT, dev_t(lk, cuda), dev_t(rk, cuda), dev_valid(lv, cuda), dev_valid(rv, cuda),
                       [dev_t(lid, cuda)], [dev_t(rid, cuda)])
    n = out.count
    r_rows = out.probe_rid[:n].cpu().numpy()
    l_rows = out.build_rid[:n].cpu().numpy()
    l_ids = out.build_payload[0][:n].cpu().numpy()
    l_ok = _bits(out.build_payload_validity[0], n)
    got = [((int(l_ids[i]) if l_ok[i] else None), int(rid[r_rows[i]])) for i in range(n)]
    assert all((l_rows[i] == L.SJ_NO_ROW) == (not l_ok[i]) for i in range(n))
    key = lambda r: tuple((0, 0) if x is None else (1, x) for x in r)  # noqa: E731
    assert sorted(got, key=key) == sorted([tuple(r) for r in fx["right"]], key=key)
    # RIGHT_SEMI / RIGHT_ANTI: right rows with / without a left match
    semi = J.right_join(J.JOIN_RIGHT_SEMI, dev_t(lk, cuda), dev_t(rk, cuda), dev_valid(lv, cuda), dev_valid(rv, cuda))
    anti = J.right_join(J.JOIN_RIGHT_ANTI, dev_t(lk, cuda), dev_t(rk, cuda), dev_valid(lv, cuda), dev_valid(rv, cuda))
    assert sorted(rid[semi.probe_rid[:semi.count].cpu().numpy()].tolist()) == [1, 2, 3]
    assert sorted(rid[anti.probe_rid[:anti.count].cpu().numpy()].tolist()) == [4, 5]


@pytest.mark.parametrize("kind", [J.JOIN_RIGHT, J.JOIN_RIGHT_SEMI, J.JOIN_RIGHT_ANTI])
@pytest.mark.parametrize("dup", [False, True])
def test_right_family_matches_oracle(cuda, kind, dup):
    rng = np.random.default_rng(31 + dup)
    n_l, n_r = 50_000, 300_000
    lk = (rng.integers(0, n_l // 4, n_l) if dup else rng.permutation(n_l)).astype(np.int64) * 3 + 5
    rk = rng.integers(0, n_l + n_l // 5, n_r).astype(np.int64) * 3 + 5
    lv = O.pack_validity(rng.random(n_l) > 0.03)
    rv = O.pack_validity(rng.random(n_r) > 0.05)
    lp = rng.integers(-2**31, 2**31 - 1, n_l).astype(np.int32)
    rp = rng.integers(-2**40, 2**40, n_r).astype(np.int64)
    out = J.right_join(kind, dev_t(lk, cuda), dev_t(rk, cuda), dev_valid(lv, cuda), dev_valid(rv, cuda),
                       [dev_t(lp, cuda)] if kind == J.JOIN_RIGHT else (), [dev_t(rp, cuda)])
    # the swapped join: left is the build side, right the probe side
    inner = {J.JOIN_RIGHT: "left", J.JOIN_RIGHT_SEMI: "semi", J.JOIN_RIGHT_ANTI: "anti"}[kind]
    _check_rows(inner, out, lk, rk, lv, rv, [lp] if kind == J.JOIN_RIGHT else [], [rp])


def _left_raw(t, pk, pp, capacity, dev):
    """sj_probe_join LEFT with probe row ids, build row ids and caller-sized outputs; returns the
    device count and the outputs (no capacity check)."""
    lib = L.load()
    kcols, nkeys, _ = J._keys(pk)
    words = (capacity + 31) // 32
    prid = torch.empty(capacity, dtype=torch.int32, device=dev)
    brid = torch.empty(capacity, dtype=torch.int32, device=dev)
    pout = torch.empty(capacity, dtype=pp.dtype, device=dev)
    bouts = [torch.empty(capacity, dtype=c.dtype, device=dev) for c, _ in t.attached]
    bvs = [torch.empty(words, dtype=torch.int32, device=dev) for _ in t.attached]
    dc = torch.zeros(1, dtype=torch.int64, device=dev)
    L.check(lib.sj_probe_join(t.handle, L.SJ_JOIN_LEFT, kcols, nkeys, J._cols([J.make_column(pp)]), 1, None,
                              len(t.attached), prid.data_ptr(), brid.data_ptr(),
                              J._cols([J._mut(pout, None)], L.SjMutColumn),
                              J._cols([J._mut(b, v) for b, v in zip(bouts, bvs)], L.SjMutColumn), capacity,
                              None, None, None, None, dc.data_ptr()), "sj_probe_join")
    torch.cuda.synchronize()
    return int(dc.item()), prid, brid, pout, bouts, bvs


@pytest.mark.parametrize("frac_absent", [0.0, 0.3, 1.0])
def test_left_partitioned_plain_payloads(cuda, frac_absent):
    """LEFT on a partitioned DISTINCT table with attached payloads without NULLs: the unmatched probe
    rows come from a bitmask of the INNER rows' probe row ids. NULL probe keys are unmatched rows."""
    rng = np.random.default_rng(41)
    nb, np_ = 200_000, 700_001
    bk = rng.permutation(nb * 3)[:nb].astype(np.int64)
    pk = bk[rng.integers(0, nb, np_)]
    absent = rng.random(np_) < frac_absent
    pk = np.where(absent, pk + (1 << 40), pk).astype(np.int64)
    pv = O.pack_validity(rng.random(np_) > 0.02)
    bp = [rng.integers(-2**40, 2**40, nb).astype(np.int64), rng.integers(-2**30, 2**30, nb).astype(np.int64)]
    pp = [rng.integers(-2**40, 2**40, np_).astype(np.int64)]
    with J.HashTable(dev_t(bk, cuda), partition_bits=4, attach=[dev_t(c, cuda) for c in bp]) as t:
        out = t.probe_join(L.SJ_JOIN_LEFT, dev_t(pk, cuda), dev_valid(pv, cuda), [dev_t(c, cuda) for c in pp],
                           attached=True)
    assert out.count == np_
    _check_rows("left", out, bk, pk, None, pv, bp, pp)


def test_left_count_exact_when_inner_rows_overflow(cuda):
    """A capacity below the INNER rows: the INNER rows past it are not written, so the matched-row
    bits would be incomplete; the unmatched pass then looks the rows up again and the LEFT count
    stays exact (every probe row once for a DISTINCT table)."""
    rng = np.random.default_rng(43)
    nb, np_ = 150_000, 500_000
    bk = rng.permutation(nb * 2)[:nb].astype(np.int64)
    pk = np.where(rng.random(np_) < 0.2, bk[rng.integers(0, nb, np_)] + (1 << 40),
                  bk[rng.integers(0, nb, np_)]).astype(np.int64)
    bp = [rng.integers(0, 1 << 30, nb).astype(np.int64)]
    pp = torch.from_numpy(rng.integers(0, 1 << 30, np_).astype(np.int64)).to(cuda)
    with J.HashTable(dev_t(bk, cuda), partition_bits=4, attach=[dev_t(c, cuda) for c in bp]) as t:
        full, *_ = _left_raw(t, dev_t(pk, cuda), pp, np_, cuda)
        small, *_ = _left_raw(t, dev_t(pk, cuda), pp, np_ // 3, cuda)
    assert full == np_ and small == np_
