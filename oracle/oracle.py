"""CPU oracle for the INNER equi-join — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module, and only as the checker / the timed CPU reference; the product (``sirius_b200``) never
calls it.

Two independent restatements of the semantics of Sirius's INNER hash join
(``src/op/sirius_physical_hash_join.cpp:1871-1874`` for INNER, ``:252-264`` for the NULL rule,
``:1299-1359`` for the gathered output columns):

* ``hash_join`` — the multithreaded C chained-hash join in ``oracle.c`` (also the CPU baseline);
* ``sort_merge_join`` — a numpy sort-merge join, used to cross-check the C oracle;
* ``kind_join`` / ``mark_join`` — LEFT, FULL, SEMI, ANTI and MARK restated from the INNER pairs
  (``:1640-1700``, ``resolve_mark_join_result`` ``:1461-1525``).

Parity pinning: ``tests/golden/`` restates the known answers of the reference's own join tests
(``test/cpp/integration/test_gpu_execution_join_nulls.cpp:42-58`` and
``test/cpp/operator/test_physical_mark_join.cpp:245-530``); both oracles must reproduce them.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_lib = None


def build() -> Path:
    """Compile oracle.c (gcc) into oracle/_build/liboracle.so."""
    src = HERE / "oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        L.oracle_join_count.restype = i64
        L.oracle_join_count.argtypes = [vp, vp, i64, i64, vp, vp, i64, i64, i32, i32, i32]
        L.oracle_inner_join.restype = i64
        L.oracle_inner_join.argtypes = [vp, vp, i64, i64, vp, vp, i64, i64, i32, i32, i32,
                                        vp, vp, i64,
                                        i32, vp, vp, vp,
                                        i32, vp, vp, vp]
        _lib = L
    return _lib


def default_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def _ptr(a):
    return None if a is None else a.ctypes.data


@dataclass
class JoinResult:
    probe_rid: np.ndarray
    build_rid: np.ndarray
    probe_payload: list
    build_payload: list

    @property
    def rows(self) -> int:
        return int(self.probe_rid.shape[0])


def _valid_or_none(v):
    if v is None:
        return None
    v = np.ascontiguousarray(v, dtype=np.uint32)
    return v


def hash_join_count(bkeys, pkeys, bvalid=None, pvalid=None, nulls_equal=False, threads=None) -> int:
    bkeys = np.ascontiguousarray(bkeys)
    pkeys = np.ascontiguousarray(pkeys)
    assert bkeys.dtype == pkeys.dtype and bkeys.dtype in (np.int32, np.int64)
    bvalid, pvalid = _valid_or_none(bvalid), _valid_or_none(pvalid)
    n = lib().oracle_join_count(_ptr(bkeys), _ptr(bvalid), 0, len(bkeys), _ptr(pkeys), _ptr(pvalid), 0,
                                len(pkeys), bkeys.dtype.itemsize, int(nulls_equal),
                                threads or default_threads())
    if n < 0:
        raise MemoryError("oracle allocation failed")
    return int(n)


def hash_join(bkeys, pkeys, bvalid=None, pvalid=None, probe_payload=(), build_payload=(),
              nulls_equal=False, threads=None, capacity=None) -> JoinResult:
    """Multithreaded C hash join. Returns rows in probe-row order (within a probe row, in build
    chain order)."""
    bkeys = np.ascontiguousarray(bkeys)
    pkeys = np.ascontiguousarray(pkeys)
    assert bkeys.dtype == pkeys.dtype and bkeys.dtype in (np.int32, np.int64)
    bvalid, pvalid = _valid_or_none(bvalid), _valid_or_none(pvalid)
    threads = threads or default_threads()
    if capacity is None:
        capacity = hash_join_count(bkeys, pkeys, bvalid, pvalid, nulls_equal, threads)
    pp = [np.ascontiguousarray(c) for c in probe_payload]
    bp = [np.ascontiguousarray(c) for c in build_payload]
    prid = np.empty(capacity, np.int32)
    brid = np.empty(capacity, np.int32)
    opp = [np.empty(capacity, c.dtype) for c in pp]
    obp = [np.empty(capacity, c.dtype) for c in bp]

    def arr(ptrs):
        return (ctypes.c_void_p * max(1, len(ptrs)))(*[p.ctypes.data for p in ptrs])

    def widths(cols):
        return (ctypes.c_int * max(1, len(cols)))(*[c.dtype.itemsize for c in cols])

    m = lib().oracle_inner_join(_ptr(bkeys), _ptr(bvalid), 0, len(bkeys), _ptr(pkeys), _ptr(pvalid), 0,
                                len(pkeys), bkeys.dtype.itemsize, int(nulls_equal), threads,
                                prid.ctypes.data, brid.ctypes.data, capacity,
                                len(pp), arr(pp), widths(pp), arr(opp),
                                len(bp), arr(bp), widths(bp), arr(obp))
    if m < 0:
        raise MemoryError("oracle allocation failed")
    k = min(m, capacity)
    return JoinResult(prid[:k], brid[:k], [c[:k] for c in opp], [c[:k] for c in obp])


# ------------------------------------------------------------------------------------------------
# Independent numpy sort-merge oracle
# ------------------------------------------------------------------------------------------------
def unpack_validity(mask, n, offset=0):
    """Bitmask words (bit i%32 of word i/32) -> bool array of n rows."""
    if mask is None:
        return np.ones(n, bool)
    bits = np.unpackbits(np.ascontiguousarray(mask, np.uint32).view(np.uint8), bitorder="little")
    return bits[offset:offset + n].astype(bool)


def pack_validity(valid):
    """bool array -> uint32 bitmask words (cuDF layout)."""
    valid = np.asarray(valid, bool)
    n = len(valid)
    words = (n + 31) // 32
    padded = np.zeros(words * 32, bool)
    padded[:n] = valid
    return np.packbits(padded, bitorder="little").view(np.uint32).copy()


def sort_merge_join(bkeys, pkeys, bvalid=None, pvalid=None, nulls_equal=False):
    """All (probe_rid, build_rid) with equal keys, NULL semantics per nulls_equal. numpy only."""
    bkeys = np.asarray(bkeys)
    pkeys = np.asarray(pkeys)
    bv = unpack_validity(bvalid, len(bkeys))
    pv = unpack_validity(pvalid, len(pkeys))
    b_idx = np.nonzero(bv)[0]
    order = b_idx[np.argsort(bkeys[b_idx], kind="stable")]
    sk = bkeys[order]
    p_idx = np.nonzero(pv)[0]
    lo = np.searchsorted(sk, pkeys[p_idx], side="left")
    hi = np.searchsorted(sk, pkeys[p_idx], side="right")
    cnt = hi - lo
    prid = np.repeat(p_idx, cnt)
    starts = np.repeat(lo, cnt)
    within = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    brid = order[starts + within]
    if nulls_equal:
        bn = np.nonzero(~bv)[0]
        pn = np.nonzero(~pv)[0]
        if len(bn) and len(pn):
            prid = np.concatenate([prid, np.repeat(pn, len(bn))])
            brid = np.concatenate([brid, np.tile(bn, len(pn))])
    return prid.astype(np.int32), brid.astype(np.int32)


# ------------------------------------------------------------------------------------------------
# The other join types, restated from the INNER pairs (numpy)
# ------------------------------------------------------------------------------------------------
NO_ROW = np.int32(-(1 << 31))  # the missing side of an outer row (cuDF's JoinNoneValue)


def kind_join(kind, bkeys, pkeys, bvalid=None, pvalid=None, nulls_equal=False):
    """Row-id pairs of a LEFT / FULL / SEMI / ANTI join, following the operator's join types
    (src/op/sirius_physical_hash_join.cpp:1640-1700: filtered_join semi/anti, hash_join left/full):
    semi = probe rows with a match; anti = the others (NULL keys included: NOT EXISTS);
    left = INNER pairs + (unmatched probe row, NO_ROW); full = left + (NO_ROW, unmatched build row),
    NULL-key build rows included. Returns (prid, brid) int32 arrays (brid None for semi/anti)."""
    pr, br = sort_merge_join(bkeys, pkeys, bvalid, pvalid, nulls_equal=nulls_equal)
    n_p, n_b = len(pkeys), len(bkeys)
    p_hit = np.zeros(n_p, bool)
    p_hit[pr] = True
    if kind == "semi":
        return np.nonzero(p_hit)[0].astype(np.int32), None
    if kind == "anti":
        return np.nonzero(~p_hit)[0].astype(np.int32), None
    miss_p = np.nonzero(~p_hit)[0].astype(np.int32)
    prid = np.concatenate([pr, miss_p])
    brid = np.concatenate([br, np.full(len(miss_p), NO_ROW, np.int32)])
    if kind == "left":
        return prid, brid
    if kind == "full":
        b_hit = np.zeros(n_b, bool)
        b_hit[br] = True
        miss_b = np.nonzero(~b_hit)[0].astype(np.int32)
        return (np.concatenate([prid, np.full(len(miss_b), NO_ROW, np.int32)]), np.concatenate([brid, miss_b]))
    raise ValueError(kind)


def mark_join(bkeys, pkeys, bvalid=None, pvalid=None):
    """MARK join (resolve_mark_join_result, src/op/sirius_physical_hash_join.cpp:1461-1525): for
    every probe row (mark, valid): mark = it has a match; an unmatched row is NULL when its key is
    NULL or when the build side has a NULL key (the IN rule; NULLs compare unequal)."""
    pr, _ = sort_merge_join(bkeys, pkeys, bvalid, pvalid)
    n_p = len(pkeys)
    mark = np.zeros(n_p, bool)
    mark[pr] = True
    pv = unpack_validity(pvalid, n_p) if pvalid is not None else np.ones(n_p, bool)
    build_has_null = bvalid is not None and not unpack_validity(bvalid, len(bkeys)).all()
    valid = mark | (pv if not build_has_null else np.zeros(n_p, bool))
    return mark, valid


def gather_nullable(col, rid, valid=None):
    """Payload column gathered by row id with NULLs for NO_ROW (and for NULL inputs): (values,
    validity bool). Values at NULL rows are 0."""
    rid = np.asarray(rid)
    ok = rid != NO_ROW
    v = np.zeros(len(rid), col.dtype)
    v[ok] = col[rid[ok]]
    m = ok.copy()
    if valid is not None:
        m[ok] &= unpack_validity(valid, len(col))[rid[ok]]
    v[~m] = 0
    return v, m


def composite_keys(build_cols, probe_cols, build_valid=None, probe_valid=None, nulls_equal=False):
    """Equi-join on several key columns reduced to one: each distinct tuple of key values (over both
    sides) gets an int64 id. Returns (build ids, probe ids, build validity words, probe validity
    words). NULLs unequal: a row with any NULL key column has a NULL id; NULLs equal: a NULL is one
    more value of its column (IS NOT DISTINCT FROM on every column)."""
    nb, npr = len(build_cols[0]), len(probe_cols[0])
    build_valid = build_valid or [None] * len(build_cols)
    probe_valid = probe_valid or [None] * len(probe_cols)
    parts, all_valid = [], np.ones(nb + npr, bool)
    for bc, pc, bv, pv in zip(build_cols, probe_cols, build_valid, probe_valid):
        vals = np.concatenate([np.asarray(bc, np.int64), np.asarray(pc, np.int64)])
        ok = np.concatenate([unpack_validity(bv, nb) if bv is not None else np.ones(nb, bool),
                             unpack_validity(pv, npr) if pv is not None else np.ones(npr, bool)])
        parts += [np.where(ok, vals, 0), (~ok).astype(np.int64)]
        all_valid &= ok
    _, ids = np.unique(np.stack(parts, axis=1), axis=0, return_inverse=True)
    ids = ids.reshape(-1).astype(np.int64)
    if nulls_equal:
        return ids[:nb], ids[nb:], None, None
    return ids[:nb], ids[nb:], pack_validity(all_valid[:nb]), pack_validity(all_valid[nb:])


def partition_ids(key_cols, key_valid=None, num_partitions=1):
    """Partition of every row under the partition operator's rule: the top log2(P) bits of mix64 of
    the key — the key itself for one column without NULLs, else the fold k0, mix64(h) ^ k_c, with
    0 for a row with any NULL key column."""
    n = len(key_cols[0])
    key_valid = key_valid or [None] * len(key_cols)
    bits = int(num_partitions).bit_length() - 1
    vals = [np.asarray(c).astype(np.int64).view(np.uint64) for c in key_cols]
    if len(key_cols) == 1 and key_valid[0] is None:
        h = vals[0]
    else:
        h = vals[0].copy()
        for v in vals[1:]:
            h = _mix(h) ^ v
        null = np.zeros(n, bool)
        for kv in key_valid:
            if kv is not None:
                null |= ~unpack_validity(kv, n)
        h[null] = np.uint64(0)
    if bits == 0:
        return np.zeros(n, np.int64)
    return (_mix(h) >> np.uint64(64 - bits)).astype(np.int64)


def bloom_mask(bkeys, pkeys, bvalid=None, pvalid=None, bits_per_key=16):
    """The blocked Bloom filter's answer per probe row (uint8), restated in numpy: 2^b blocks of 8
    32-bit words (the smallest b with 256 * 2^b >= keys * bits_per_key), block = top b bits of
    mix64(key), bit of word w = bits [5w, 5w+5) of mix64(mix64(key) + 0x9E3779B97F4A7C15); NULL keys
    are not inserted and test 0."""
    nb, npr = len(bkeys), len(pkeys)
    want = max(nb, 1) * bits_per_key
    b = 0
    while b < 40 and (256 << b) < want:
        b += 1
    words = np.zeros((1 << b) * 8, np.uint32)

    def locate(keys):
        h = _mix(np.asarray(keys).astype(np.int64).view(np.uint64))
        block = (h >> np.uint64(64 - b)) if b else np.zeros(len(h), np.uint64)
        with np.errstate(over="ignore"):
            bits = _mix(h + np.uint64(0x9E3779B97F4A7C15))
        return block.astype(np.int64), bits

    ok = unpack_validity(bvalid, nb) if bvalid is not None else np.ones(nb, bool)
    blk, bits = locate(bkeys)
    for w in range(8):
        bit = ((bits >> np.uint64(5 * w)) & np.uint64(31)).astype(np.uint32)
        np.bitwise_or.at(words, blk[ok] * 8 + w, (np.uint32(1) << bit[ok]))
    pok = unpack_validity(pvalid, npr) if pvalid is not None else np.ones(npr, bool)
    blk, bits = locate(pkeys)
    hit = pok.copy()
    for w in range(8):
        bit = ((bits >> np.uint64(5 * w)) & np.uint64(31)).astype(np.uint32)
        hit &= ((words[blk * 8 + w] >> bit) & 1).astype(bool)
    return hit.astype(np.uint8)


# ------------------------------------------------------------------------------------------------
# Canonical form and order-independent checksum
# ------------------------------------------------------------------------------------------------
def canonical_order(prid, brid):
    """Permutation sorting rows by (probe_rid, build_rid); an INNER join never repeats a pair."""
    key = (np.asarray(prid, np.int64).astype(np.uint64) << np.uint64(32)) | \
        np.asarray(brid, np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    return np.argsort(key, kind="stable")


def canonical(prid, brid, *cols):
    o = canonical_order(prid, brid)
    return (np.asarray(prid)[o], np.asarray(brid)[o]) + tuple(np.asarray(c)[o] for c in cols)


_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(x):
    x = x ^ (x >> np.uint64(30))
    x = x * _M1
    x = x ^ (x >> np.uint64(27))
    x = x * _M2
    return x ^ (x >> np.uint64(31))


def multiset_checksum(*cols) -> int:
    """Order-independent 64-bit checksum of a multiset of rows: sum over rows of a mix of the row's
    columns (as raw 64-bit values), mod 2^64."""
    if not cols or len(cols[0]) == 0:
        return 0
    with np.errstate(over="ignore"):
        h = np.zeros(len(cols[0]), np.uint64)
        for i, c in enumerate(cols):
            c = np.asarray(c)
            v = c.view(np.uint32).astype(np.uint64) if c.dtype.itemsize == 4 else c.view(np.uint64)
            h = _mix(h ^ (v + np.uint64(0x9E3779B97F4A7C15) * np.uint64(i + 1)))
        return int(h.sum(dtype=np.uint64))
