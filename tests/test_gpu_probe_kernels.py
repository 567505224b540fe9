"""GPU parity of every DISTINCT probe write-out (staged, direct, direct with TMA-staged inputs)
against the CPU oracle, bit-exact: partitioned and unpartitioned tables, int32 and int64 keys,
packed and wide slots, attached and caller build payloads, 4- and 8-byte probe payloads, probe
sizes that end in a partial tile, NULL probe keys, misses, and unaligned probe columns (which the
TMA variant must hand to the plain-load kernel)."""
import numpy as np
import pytest
import torch

from jhelp import assert_same_rows, dev_t, dev_valid, oracle_join
from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import datagen as D
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu

KERNELS = [L.SJ_PROBE_KERNEL_STAGED, L.SJ_PROBE_KERNEL_DIRECT, L.SJ_PROBE_KERNEL_DIRECT_TMA]


def _input(seed, dtype, nb, npr, pay_dtypes=(np.int64,), bpay_dtypes=(np.int64, np.int64), null_frac=0.0,
           full_range=False):
    rng = np.random.default_rng(seed)
    if full_range:
        bk = D.mix64(np.arange(nb, dtype=np.uint64) + np.uint64(seed << 40)).view(np.int64)
    else:
        bk = (rng.permutation(nb * 3)[:nb]).astype(dtype)
    pick = rng.integers(0, nb, npr)
    pk = bk[pick].copy()
    miss = rng.random(npr) < 0.2
    m = int(miss.sum())
    if full_range:  # indices past the table's range: distinct from every build key
        pk[miss] = D.mix64(np.arange(nb, nb + m, dtype=np.uint64) + np.uint64(seed << 40)).view(np.int64)
    else:
        pk[miss] = (bk.max() + 1 + rng.integers(0, 1000, m)).astype(pk.dtype)
    pv = O.pack_validity(rng.random(npr) >= null_frac) if null_frac else None
    pp = [rng.integers(-2**31, 2**31 - 1, npr).astype(t) for t in pay_dtypes]
    bp = [rng.integers(-2**40, 2**40, nb).astype(t) for t in bpay_dtypes]
    return D.JoinInput("probe-kernels", bk, pk, bp, pp, None, pv)


def _run(inp, dev, kernel, attach, **kw):
    bk, pk = dev_t(inp.build_keys, dev), dev_t(inp.probe_keys, dev)
    pv = dev_valid(inp.probe_validity, dev)
    bp = [dev_t(c, dev) for c in inp.build_payload]
    pp = [dev_t(c, dev) for c in inp.probe_payload]
    with J.HashTable(bk, attach=bp if attach else (), probe_kernel=kernel, **kw) as t:
        out = (t.probe_gather(pk, pv, pp, attached=True) if attach else t.probe_gather(pk, pv, pp, bp)).trimmed()
    torch.cuda.synchronize()
    return [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()] + \
        [c.cpu().numpy() for c in out.probe_payload] + [c.cpu().numpy() for c in out.build_payload]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("pbits", [-1, 3])
@pytest.mark.parametrize("attach", [False, True])
def test_kernels_match_oracle(cuda, kernel, dtype, pbits, attach):
    inp = _input(11, dtype, 200_003, 1_000_037)  # partial last tiles everywhere
    got = _run(inp, cuda, kernel, attach, partition_bits=pbits)
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("agg", [L.SJ_AGG_WARP, L.SJ_AGG_CTA, L.SJ_AGG_WARP_DYNAMIC])
def test_direct_output_reservation_modes(cuda, agg):
    inp = _input(15, np.int64, 300_001, 2_000_003)
    for pbits in (-1, 3):
        got = _run(inp, cuda, L.SJ_PROBE_KERNEL_DIRECT, True, partition_bits=pbits, aggregation=agg)
        assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("kernel", KERNELS)
def test_kernels_wide_slots_and_null_probe_keys(cuda, kernel):
    inp = _input(12, np.int64, 150_001, 700_001, null_frac=0.05, full_range=True)
    got = _run(inp, cuda, kernel, True, partition_bits=2)
    assert_same_rows(got, oracle_join(inp))
    got = _run(inp, cuda, kernel, True, partition_bits=-1)
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("shape", [((np.int32,), (np.int32,)), ((np.int32, np.int64), (np.int64,)),
                                   ((), ()), ((np.int64, np.int64), (np.int64, np.int64, np.int64))])
def test_kernels_payload_shapes(cuda, kernel, shape):
    pay, bpay = shape
    inp = _input(13, np.int64, 100_000, 513 * 1001, pay_dtypes=pay, bpay_dtypes=bpay)
    for attach in (False, True):
        got = _run(inp, cuda, kernel, attach, partition_bits=2)
        assert_same_rows(got, oracle_join(inp))


def test_tma_kernel_takes_unaligned_probe_columns(cuda):
    """A probe key column starting 8 bytes past a 16-byte boundary goes to the plain-load kernel."""
    inp = _input(14, np.int64, 120_000, 600_001)
    bk = dev_t(inp.build_keys, cuda)
    big = dev_t(np.concatenate([[0], inp.probe_keys]), cuda)
    pk = big[1:]
    assert pk.data_ptr() % 16 == 8
    pp = [dev_t(c, cuda) for c in inp.probe_payload]
    bp = [dev_t(c, cuda) for c in inp.build_payload]
    with J.HashTable(bk, attach=bp, probe_kernel=L.SJ_PROBE_KERNEL_DIRECT_TMA, partition_bits=-1) as t:
        out = t.probe_gather(pk, None, pp, attached=True).trimmed()
    got = [out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()] + \
        [c.cpu().numpy() for c in out.probe_payload] + [c.cpu().numpy() for c in out.build_payload]
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("l2", [L.SJ_L2_NORMAL, L.SJ_L2_EVICT_LAST])
@pytest.mark.parametrize("share_mb", [0, 1])
def test_table_l2_priority_and_probe_partition_share(cuda, l2, share_mb):
    """The L2 policy of the table loads and the probe's partition share change where lines live
    and how many probe partitions there are, never the result; wide slots cover the 128-bit loads."""
    for full_range in (False, True):
        inp = _input(16, np.int64, 400_001, 1_500_007, full_range=full_range)
        for attach in (False, True):
            got = _run(inp, cuda, L.SJ_PROBE_KERNEL_AUTO, attach, partition_bits=6, table_l2_priority=l2,
                       probe_partition_mb=share_mb)
            assert_same_rows(got, oracle_join(inp))


def test_l2_priority_and_share_are_validated(cuda):
    k = dev_t(np.arange(1000, dtype=np.int64), cuda)
    with pytest.raises(L.SjError):
        J.HashTable(k, table_l2_priority=3)
    with pytest.raises(L.SjError):
        J.HashTable(k, probe_partition_mb=-1)
