"""Seeded random configurations of the INNER join against the CPU oracle, bit-exact after a
canonical sort. Each case draws: key type; build and probe sizes from empty and single rows up to
partitioned-probe sizes; unique, duplicated, full-range or negative keys; NULL keys on either side
(none, some, all); the NULL rule; load factor; radix partition bits; attached or caller build
payloads of 1-8 bytes; the DISTINCT probe's write-out kernel. The configuration is part of every
failure message, so a failing case can be replayed alone."""
import numpy as np
import pytest

from jhelp import assert_same_rows, gpu_join, oracle_join
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import datagen as D

pytestmark = pytest.mark.gpu

N_CASES = 320
MAX_OUT = 4_000_000
PAYLOAD_TYPES = [np.int8, np.int16, np.int32, np.int64, np.float32, np.float64]


def _case(seed):
    r = np.random.default_rng(1000 + seed)
    dtype = np.int32 if r.random() < 0.4 else np.int64
    size_class = r.choice(["empty", "one", "small", "medium", "partitioned"], p=[0.05, 0.05, 0.4, 0.3, 0.2])
    nb = {"empty": 0, "one": 1}.get(size_class, int(r.integers(2, 60_000 if size_class != "partitioned" else 150_000)))
    np_ = {"empty": int(r.integers(0, 100)), "one": int(r.integers(1, 1000))}.get(
        size_class, int(r.integers(1, 200_000)) if size_class != "partitioned" else int(r.integers(70_000, 400_000)))
    keys = r.choice(["unique", "dups", "full_range", "negative"])
    if keys == "unique":
        bk = (r.permutation(max(nb, 1) * 2)[:nb]).astype(dtype)
    elif keys == "dups":
        bk = r.integers(0, max(1, nb // int(r.integers(2, 50))), nb).astype(dtype)
    elif keys == "full_range" and dtype == np.int64:
        bk = r.integers(-2**63, 2**63 - 1, nb, dtype=np.int64)
    else:
        hi = 2**31 - 1 if dtype == np.int32 else 2**40
        bk = r.integers(-hi, hi, nb).astype(dtype)
    hit = r.random()
    pk = np.empty(np_, dtype)
    if nb:
        from_build = r.random(np_) < hit
        pk[from_build] = bk[r.integers(0, nb, int(from_build.sum()))]
        miss = ~from_build
        if keys == "full_range" and dtype == np.int64:
            pk[miss] = r.integers(-2**63, 2**63 - 1, int(miss.sum()), dtype=np.int64)
        else:  # around and inside the build's key range
            lo, hi = int(bk.min()), int(bk.max())
            span = max(1, hi - lo)
            off = r.integers(-(span // 4) - 1, span + span // 4 + 2, int(miss.sum()), dtype=np.int64)
            info = np.iinfo(dtype)
            pk[miss] = np.clip(off + lo, info.min, info.max).astype(dtype)
    else:
        pk[:] = r.integers(-1000, 1000, np_).astype(dtype)
    null_b = r.choice([0.0, 0.0, 0.05, 1.0])
    null_p = r.choice([0.0, 0.0, 0.1, 1.0])
    bmask = r.random(nb) >= null_b
    pmask = r.random(np_) >= null_p
    nbp, npp = int(r.integers(0, 3)), int(r.integers(0, 3))
    bp = [r.integers(-100, 100, nb).astype(PAYLOAD_TYPES[int(r.integers(0, 6))]) for _ in range(nbp)]
    pp = [r.integers(-100, 100, np_).astype(PAYLOAD_TYPES[int(r.integers(0, 6))]) for _ in range(npp)]
    null_equality = int(r.random() < 0.25)
    # NULL = NULL over many NULL rows, or heavy duplicates, multiply into billions of output rows:
    # keep every case's output under MAX_OUT rows (NULLs distinct first, then fewer probe rows)
    out = O.hash_join_count(bk, pk, O.pack_validity(bmask), O.pack_validity(pmask), nulls_equal=bool(null_equality))
    if out > MAX_OUT and null_equality:
        null_equality = 0
        out = O.hash_join_count(bk, pk, O.pack_validity(bmask), O.pack_validity(pmask))
    if out > MAX_OUT:
        np_ = max(1, np_ * MAX_OUT // out)
        pk, pmask, pp = pk[:np_], pmask[:np_], [c[:np_] for c in pp]
    bv = O.pack_validity(bmask) if null_b else None
    pv = O.pack_validity(pmask) if null_p else None
    params = dict(
        null_equality=null_equality,
        load_factor=float(r.choice([0.35, 0.5, 0.7, 0.9])),
        partition_bits=int(r.choice([-1, 0, 0, 2, 4, 6])),
        probe_kernel=int(r.choice([L.SJ_PROBE_KERNEL_AUTO, L.SJ_PROBE_KERNEL_STAGED, L.SJ_PROBE_KERNEL_DIRECT,
                                   L.SJ_PROBE_KERNEL_DIRECT_TMA])),
        force_wide=bool(r.random() < 0.15),
    )
    attach = bool(r.random() < 0.5)
    desc = dict(seed=seed, dtype=dtype.__name__, nb=nb, np=np_, keys=keys, hit=round(hit, 2), null_b=null_b,
                null_p=null_p, bpay=[t.dtype.name for t in bp], ppay=[t.dtype.name for t in pp], attach=attach,
                **params)
    return D.JoinInput(f"fuzz{seed}", bk, pk, bp, pp, bv, pv), params, attach, desc


@pytest.mark.parametrize("seed", range(N_CASES))
def test_random_inner_join_matches_oracle(cuda, seed):
    inp, params, attach, desc = _case(seed)
    got, info = gpu_join(inp, cuda, attach=attach, **params)
    exp = oracle_join(inp, nulls_equal=bool(params["null_equality"]))
    try:
        assert_same_rows(got, exp)
    except AssertionError as e:
        raise AssertionError(f"{desc}: {e}") from None
