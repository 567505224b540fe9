"""GPU parity of the dynamic Bloom filter (``sj_bloom_build`` / ``sj_bloom_contains``, and the same
filter filled by a table's insert pass, ``bloom_bits_per_key``) against the oracle's restatement:
the mask is deterministic, so it must equal the oracle's bit for bit (false positives included);
every build key tests positive; NULL probe keys test 0 with a NULL bit."""
import numpy as np
import pytest
import torch

from jhelp import dev_t, dev_valid
from oracle import oracle as O
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("bits", [4, 16, 40])
def test_bloom_matches_oracle(cuda, dtype, bits):
    rng = np.random.default_rng(bits)
    nb, npr = 200_003, 1_000_001
    hi = 2**31 - 1 if dtype == np.int32 else 2**50
    bk = rng.integers(-hi, hi, nb).astype(dtype)
    pk = np.concatenate([bk[rng.integers(0, nb, npr // 3)], rng.integers(-hi, hi, npr - npr // 3).astype(dtype)])
    bv = O.pack_validity(rng.random(nb) > 0.05)
    pv = O.pack_validity(rng.random(npr) > 0.05)
    with J.BloomFilter(dev_t(bk, cuda), dev_valid(bv, cuda), bits_per_key=bits) as f:
        mask, valid = f.contains(dev_t(pk, cuda), dev_valid(pv, cuda))
    got = mask.cpu().numpy()
    exp = O.bloom_mask(bk, pk, bv, pv, bits_per_key=bits)
    assert np.array_equal(got, exp)
    assert np.array_equal(O.unpack_validity(valid.cpu().numpy().view(np.uint32), npr), O.unpack_validity(pv, npr))


def test_bloom_has_no_false_negatives_at_scale(cuda):
    rng = np.random.default_rng(3)
    bk = rng.integers(0, 2**62, 16 << 20, dtype=np.int64)
    with J.BloomFilter(dev_t(bk, cuda)) as f:
        assert f.nbytes >= (16 << 20) * 16 // 8
        mask, _ = f.contains(dev_t(bk, cuda))
        assert int(mask.sum().item()) == len(bk)
        miss, _ = f.contains(dev_t(rng.integers(2**62, 2**63 - 1, 4 << 20, dtype=np.int64), cuda))
        assert miss.float().mean().item() < 0.01


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("dup", [False, True])
@pytest.mark.parametrize("pbits", [-1, 4])
def test_build_time_filter_equals_separate_build(cuda, dtype, dup, pbits):
    """The filter the table's insert pass fills (bloom_bits_per_key) is the filter sj_bloom_build makes
    from the same keys, bit for bit, and the oracle's restatement; the table still joins correctly.
    Covers unique and duplicated build keys (DISTINCT and GROUPED layouts), radix-partitioned tables
    (the insert walks the partitioned key copy) and NULL build keys."""
    from sirius_b200 import _lib as L
    rng = np.random.default_rng(7 + dup + pbits)
    nb, npr = 300_007, 900_001
    bk = (rng.integers(0, nb // 3, nb) if dup else rng.permutation(nb) * 5).astype(dtype)
    pk = rng.integers(0, 5 * nb, npr).astype(dtype)
    bv = O.pack_validity(rng.random(nb) > 0.04)
    pv = O.pack_validity(rng.random(npr) > 0.06)
    dbk, dpk, dbv, dpv = dev_t(bk, cuda), dev_t(pk, cuda), dev_valid(bv, cuda), dev_valid(pv, cuda)
    with J.HashTable(dbk, dbv, partition_bits=pbits, bloom_bits_per_key=12) as t:
        assert t.info().partition_bits == max(pbits, 0)
        f = t.bloom()
        assert f is not None and f.nbytes >= nb * 12 // 8
        got, gvalid = f.contains(dpk, dpv)
        assert int(t.count(dpk, dpv).item()) == O.hash_join_count(bk, pk, bv, pv)
    with J.BloomFilter(dbk, dbv, bits_per_key=12) as sep:
        exp, _ = sep.contains(dpk, dpv)
    assert torch.equal(got, exp)
    assert np.array_equal(got.cpu().numpy(), O.bloom_mask(bk, pk, bv, pv, bits_per_key=12))
    assert np.array_equal(O.unpack_validity(gvalid.cpu().numpy().view(np.uint32), npr), O.unpack_validity(pv, npr))
    with J.HashTable(dbk, dbv) as t:
        assert t.bloom() is None
    with pytest.raises(L.SjError):  # a composite key has no single key column to filter on
        J.HashTable([dbk, dbk], bloom_bits_per_key=8)
