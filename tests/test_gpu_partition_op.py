"""GPU parity of the hash partition operator (``sj_hash_partition``) against the oracle's partition
rule: every input row appears once, in the partition the oracle assigns it, with its column values
and NULLs carried along; one and several key columns, NULL keys (partition 0), 1..1024 partitions,
and equal keys of two different tables landing in the same partition."""
import numpy as np
import pytest
import torch

from jhelp import dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


def _check(cuda, key_cols, key_valid, cols, col_valid, P):
    n = len(key_cols[0])
    rid = np.arange(n, dtype=np.int32)
    keys = ([(dev_t(c, cuda), dev_valid(v, cuda)) for c, v in zip(key_cols, key_valid)]
            if (len(key_cols) > 1 or key_valid[0] is not None) else dev_t(key_cols[0], cuda))
    ins = [dev_t(rid, cuda)] + [(dev_t(c, cuda), dev_valid(v, cuda)) for c, v in zip(cols, col_valid)]
    outs, vouts, off = J.hash_partition(keys, ins, P)
    off = off.cpu().numpy()
    assert off[0] == 0 and off[-1] == n and np.all(np.diff(off) >= 0)
    orid = outs[0].cpu().numpy()
    assert np.array_equal(np.sort(orid), rid), "not a permutation of the input rows"
    part = O.partition_ids(key_cols, key_valid, P)
    for p in range(P):
        assert np.all(part[orid[off[p]:off[p + 1]]] == p), f"rows in partition {p} belong elsewhere"
    for c, (col, v) in enumerate(zip(cols, col_valid)):
        got = outs[c + 1].cpu().numpy()
        assert np.array_equal(got, col[orid])
        if v is not None:
            gv = O.unpack_validity(vouts[c + 1].cpu().numpy().view(np.uint32), n)
            assert np.array_equal(gv, O.unpack_validity(v, n)[orid])
    return part


@pytest.mark.parametrize("P", [1, 8, 64, 1024])
def test_single_key_no_nulls(cuda, P):
    rng = np.random.default_rng(P)
    n = 1_000_003
    k = rng.integers(-2**40, 2**40, n).astype(np.int64)
    cols = [rng.integers(0, 1 << 30, n).astype(np.int64), rng.random(n).astype(np.float32)]
    _check(cuda, [k], [None], cols, [None, None], P)


@pytest.mark.parametrize("P", [4, 32])
def test_null_keys_and_nullable_columns(cuda, P):
    rng = np.random.default_rng(7)
    n = 300_001
    k = rng.integers(0, 50_000, n).astype(np.int32)
    kv = O.pack_validity(rng.random(n) > 0.1)
    cols = [rng.integers(-100, 100, n).astype(np.int16), rng.integers(0, 9, n).astype(np.int32),
            rng.random(n), rng.integers(0, 2, n).astype(np.int8)]
    cv = [O.pack_validity(rng.random(n) > 0.3), None, O.pack_validity(rng.random(n) > 0.5), None]
    part = _check(cuda, [k], [kv], cols, cv, P)
    assert np.all(part[~O.unpack_validity(kv, n)] == 0)


def test_composite_keys_and_cross_table_consistency(cuda):
    rng = np.random.default_rng(9)
    a = [rng.integers(0, 300, 200_000).astype(np.int64), rng.integers(0, 300, 200_000).astype(np.int32)]
    b = [rng.integers(0, 300, 150_000).astype(np.int64), rng.integers(0, 300, 150_000).astype(np.int32)]
    pa = _check(cuda, a, [None, None], [a[0], a[1]], [None, None], 16)
    pb = _check(cuda, b, [None, None], [b[0], b[1]], [None, None], 16)
    # a tuple present in both tables lands in the same partition in both
    ta = {(x, y): p for x, y, p in zip(a[0].tolist(), a[1].tolist(), pa.tolist())}
    for x, y, p in zip(b[0].tolist(), b[1].tolist(), pb.tolist()):
        if (x, y) in ta:
            assert ta[(x, y)] == p


def test_int32_and_int64_keys_of_equal_value_share_partitions(cuda):
    """The reference casts partition keys of mixed-type joins so both sides hash alike
    (gpu_partition_impl.cpp:45-60); here the partition function sign-extends keys to 64 bits, so
    equal values land in the same partition whatever their integer type."""
    rng = np.random.default_rng(12)
    v = rng.integers(-2**31, 2**31 - 1, 100_000)
    a = _check(cuda, [v.astype(np.int32)], [None], [], [], 64)
    b = _check(cuda, [v.astype(np.int64)], [None], [], [], 64)
    assert np.array_equal(a, b)
