"""GPU parity of the dynamic Bloom filter (``sj_bloom_build`` / ``sj_bloom_contains``) against the
oracle's restatement: the mask is deterministic, so it must equal the oracle's bit for bit (false
positives included); every build key tests positive; NULL probe keys test 0 with a NULL bit."""
import numpy as np
import pytest

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
