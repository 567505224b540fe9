"""Shared helpers of the GPU parity tests: run a JoinInput through the C ABI and compare the
canonically sorted output with the CPU oracle, bit for bit."""
from __future__ import annotations

import numpy as np
import torch

from oracle import oracle as O


def dev_t(a, dev):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def dev_valid(words, dev):
    return None if words is None else torch.from_numpy(np.ascontiguousarray(words).view(np.int32)).to(dev)


def gpu_join(inp, dev, attach=False, **table_kw):
    """Build + fused probe/gather on the GPU; returns (host arrays tuple, table info).
    attach=True attaches the build payloads to the table (sj_build_ex) and gathers them from it."""
    from sirius_b200 import join as J
    bk, pk = dev_t(inp.build_keys, dev), dev_t(inp.probe_keys, dev)
    bv, pv = dev_valid(inp.build_validity, dev), dev_valid(inp.probe_validity, dev)
    bp = [dev_t(c, dev) for c in inp.build_payload]
    pp = [dev_t(c, dev) for c in inp.probe_payload]
    with J.HashTable(bk, bv, attach=bp if attach else (), **table_kw) as t:
        info = t.info()
        cnt = int(t.count(pk, pv).item())
        if attach:
            out = t.probe_gather(pk, pv, pp, attached=True).trimmed()
        else:
            out = t.probe_gather(pk, pv, pp, bp).trimmed()
    torch.cuda.synchronize()
    assert cnt == out.count, (cnt, out.count)
    host = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()]
    host += [c.cpu().numpy() for c in out.probe_payload] + [c.cpu().numpy() for c in out.build_payload]
    return host, info


def oracle_join(inp, nulls_equal=False):
    r = O.hash_join(inp.build_keys, inp.probe_keys, inp.build_validity, inp.probe_validity,
                    probe_payload=inp.probe_payload, build_payload=inp.build_payload, nulls_equal=nulls_equal)
    return [r.probe_rid, r.build_rid] + r.probe_payload + r.build_payload


def assert_same_rows(got, exp):
    assert len(got[0]) == len(exp[0]), f"row count {len(got[0])} != oracle {len(exp[0])}"
    g = O.canonical(*got)
    e = O.canonical(*exp)
    for i, (a, b) in enumerate(zip(g, e)):
        assert a.dtype == b.dtype, (i, a.dtype, b.dtype)
        if not np.array_equal(a, b):
            bad = np.nonzero(a != b)[0][:5]
            raise AssertionError(f"column {i} differs at canonical rows {bad}: {a[bad]} vs {b[bad]}")
