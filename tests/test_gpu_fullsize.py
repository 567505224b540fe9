"""Parity at the full workload sizes through size-independent properties: exact row counts,
joined keys equal, gathered payloads equal the source rows, every probe row of the 1:1 join
appears exactly once, and an order-independent multiset checksum equal to the CPU oracle's."""
import numpy as np
import pytest
import torch

from jhelp import dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import datagen as D
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


def test_large_full_size(cuda):
    inp = D.large(1)  # 16M build x 64M probe
    bk, pk = dev_t(inp.build_keys, cuda), dev_t(inp.probe_keys, cuda)
    bp = [dev_t(c, cuda) for c in inp.build_payload]
    pp = [dev_t(c, cuda) for c in inp.probe_payload]
    with J.HashTable(bk) as t:
        info = t.info()
        assert info.layout == 1 and info.slot_kind == 0 and info.rid_bits == 24
        assert info.distinct_keys == inp.n_build
        out = t.probe_gather(pk, None, pp, bp).trimmed()
    assert out.count == inp.n_probe
    # every probe row exactly once
    seen = torch.zeros(inp.n_probe, dtype=torch.int32, device=cuda)
    seen.index_add_(0, out.probe_rid.long(), torch.ones_like(out.probe_rid))
    assert bool((seen == 1).all())
    prid, brid = out.probe_rid.long(), out.build_rid.long()
    assert torch.equal(pk[prid], bk[brid])
    assert torch.equal(out.probe_payload[0], pp[0][prid])
    assert torch.equal(out.build_payload[0], bp[0][brid])
    assert torch.equal(out.build_payload[1], bp[1][brid])
    host = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy(), out.probe_payload[0].cpu().numpy(),
            out.build_payload[0].cpu().numpy(), out.build_payload[1].cpu().numpy()]
    del out, seen, prid, brid
    torch.cuda.empty_cache()
    ref = O.hash_join(inp.build_keys, inp.probe_keys, probe_payload=inp.probe_payload,
                      build_payload=inp.build_payload, capacity=inp.n_probe)
    assert ref.rows == inp.n_probe
    assert O.multiset_checksum(*host) == O.multiset_checksum(ref.probe_rid, ref.build_rid, *ref.probe_payload,
                                                             *ref.build_payload)


def test_skewed_full_size(cuda):
    inp = D.skewed(1)  # 8M build (Zipf 1.1 over 1M) x 32M probe (Zipf 0.8 over 2M, 5% NULL)
    m_ref = O.hash_join_count(inp.build_keys, inp.probe_keys, None, inp.probe_validity)
    bk, pk = dev_t(inp.build_keys, cuda), dev_t(inp.probe_keys, cuda)
    pv = dev_valid(inp.probe_validity, cuda)
    bp = [dev_t(c, cuda) for c in inp.build_payload]
    with J.HashTable(bk) as t:
        info = t.info()
        assert info.layout == 2
        assert info.max_group > 500_000  # the top Zipf(1.1) key holds ~12% of the build rows
        assert int(t.count(pk, pv).item()) == m_ref
        out = t.probe_gather(pk, pv, [], bp).trimmed()
    assert out.count == m_ref
    prid, brid = out.probe_rid.long(), out.build_rid.long()
    assert torch.equal(pk[prid], bk[brid])
    pvalid = torch.from_numpy(O.unpack_validity(inp.probe_validity, inp.n_probe)).to(cuda)
    assert bool(pvalid[prid].all()), "a NULL probe key matched"
    assert torch.equal(out.build_payload[0], bp[0][brid])
    host = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy(), out.build_payload[0].cpu().numpy()]
    del out, prid, brid
    torch.cuda.empty_cache()
    ref = O.hash_join(inp.build_keys, inp.probe_keys, None, inp.probe_validity, build_payload=inp.build_payload,
                      capacity=m_ref)
    assert O.multiset_checksum(*host) == O.multiset_checksum(ref.probe_rid, ref.build_rid, *ref.build_payload)
