"""GPU parity: the sm_100a join (through the C ABI) against the CPU oracle, bit-exact on the
canonically sorted output rows (probe rid, build rid, probe payloads, build payloads)."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from jhelp import assert_same_rows, dev_t, dev_valid, gpu_join, oracle_join
from oracle import oracle as O
from sirius_b200 import datagen as D

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "join_known_answers.json").read_text())


def _col(values, dtype):
    valid = np.array([v is not None for v in values], bool)
    data = np.array([0 if v is None else v for v in values], dtype)
    return data, O.pack_validity(valid)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
@pytest.mark.parametrize("wide", [False, True])
@pytest.mark.parametrize("layout", [0, 2])
def test_known_answer_inner(cuda, dtype, wide, layout):
    """test_gpu_execution_join_nulls.cpp:50-58: NULL never matches, duplicates multiply."""
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"], dtype)
    rk, rv = _col(fx["r"]["k"], dtype)
    inp = D.JoinInput("nulls", rk, lk, [np.array(fx["r"]["id"], np.int32)], [np.array(fx["l"]["id"], np.int32)],
                      rv, lv)
    got, info = gpu_join(inp, cuda, force_wide=wide, layout=layout)
    pairs = sorted(zip(got[2].tolist(), got[3].tolist()))
    assert pairs == [tuple(p) for p in fx["inner"]]
    assert info.layout == 2  # duplicates on the build side -> grouped


@pytest.mark.parametrize("wide", [False, True])
def test_known_answer_null_safe(cuda, wide):
    fx = GOLDEN["nulls_fixture"]
    lk, lv = _col(fx["l"]["k"], np.int32)
    rk, rv = _col(fx["r"]["k"], np.int32)
    inp = D.JoinInput("nulls", rk, lk, [np.array(fx["r"]["id"], np.int32)], [np.array(fx["l"]["id"], np.int32)],
                      rv, lv)
    got, _ = gpu_join(inp, cuda, null_equality=1, force_wide=wide)
    assert sorted(zip(got[2].tolist(), got[3].tolist())) == [tuple(p) for p in fx["inner_null_safe"]]


@pytest.mark.parametrize("case", GOLDEN["mark_cases"], ids=lambda c: c["name"])
def test_known_answer_mark_cases_inner_rows(cuda, case):
    lk, lv = _col(case["left"], np.int32)
    if case["right"]:
        rk, rv = _col(case["right"], np.int32)
    else:
        rk, rv = np.zeros(0, np.int32), None
    inp = D.JoinInput("mark", rk, lk, [], [], rv, lv)
    got, _ = gpu_join(inp, cuda)
    assert set(got[0].tolist()) == {i for i, m in enumerate(case["mark"]) if m is True}


@pytest.mark.parametrize("seed", [1, 2])
def test_small_config_full_size(cuda, seed):
    inp = D.small(seed)
    got, info = gpu_join(inp, cuda)
    assert info.layout == 1 and info.slot_kind == 0
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("pbits", [0, 4])
def test_large_config_scaled(cuda, pbits):
    inp = D.large(5, n_build=1 << 20, n_probe=4 << 20)
    got, info = gpu_join(inp, cuda, partition_bits=pbits)
    assert info.layout == 1 and info.slot_kind == 0 and info.rid_bits == 20
    assert len(got[0]) == inp.n_probe
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("wide", [False, True])
def test_skewed_config_scaled(cuda, wide):
    inp = D.skewed(4, n_build=1 << 20, n_probe=4 << 20, build_values=1 << 17, probe_values=1 << 18)
    got, info = gpu_join(inp, cuda, force_wide=wide)
    assert info.layout == 2 and info.max_group > 1000
    assert info.distinct_keys == len(np.unique(inp.build_keys))
    assert_same_rows(got, oracle_join(inp))


def test_grouped_forced_on_unique_keys(cuda):
    inp = D.small(9, 5000, 40000)
    got, info = gpu_join(inp, cuda, layout=2)
    assert info.layout == 2 and info.max_group == 1
    assert_same_rows(got, oracle_join(inp))


def test_full_range_int64_uses_wide_slots(cuda):
    rng = np.random.default_rng(11)
    bk = D.mix64(np.arange(30000, dtype=np.uint64)).view(np.int64)
    pk = np.concatenate([bk[rng.integers(0, len(bk), 70000)], rng.integers(-2**63, 2**63 - 1, 30000)])
    bk = np.concatenate([bk, np.array([np.iinfo(np.int64).min, np.iinfo(np.int64).max], np.int64)])
    pk = np.concatenate([pk, np.array([np.iinfo(np.int64).max, np.iinfo(np.int64).min, -1, 0], np.int64)])
    inp = D.JoinInput("fullrange", bk, pk, [np.arange(len(bk), dtype=np.int64)], [np.arange(len(pk), dtype=np.int32)])
    got, info = gpu_join(inp, cuda)
    assert info.slot_kind == 1
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("nulls_equal", [0, 1])
def test_nulls_both_sides_random(cuda, nulls_equal):
    rng = np.random.default_rng(21)
    bk = rng.integers(-1000, 1000, 20000).astype(np.int64)
    pk = rng.integers(-1100, 1100, 50000).astype(np.int64)
    inp = D.JoinInput("nulls", bk, pk, [rng.integers(0, 9, 20000).astype(np.int8)],
                      [rng.random(50000).astype(np.float32)],
                      O.pack_validity(rng.random(20000) > 0.2), O.pack_validity(rng.random(50000) > 0.3))
    got, info = gpu_join(inp, cuda, null_equality=nulls_equal)
    assert_same_rows(got, oracle_join(inp, nulls_equal=bool(nulls_equal)))


def test_empty_inputs(cuda):
    from sirius_b200 import join as J
    e = torch.zeros(0, dtype=torch.int32, device=cuda)
    k = torch.arange(10, dtype=torch.int32, device=cuda)
    with J.HashTable(e) as t:
        assert t.info().valid_rows == 0
        assert t.probe_gather(k).count == 0
        assert int(t.count(k).item()) == 0
    with J.HashTable(k) as t:
        assert t.probe_gather(e).count == 0


def test_all_null_sides(cuda):
    from sirius_b200 import join as J
    k = torch.arange(64, dtype=torch.int64, device=cuda)
    none = torch.zeros(2, dtype=torch.int32, device=cuda)
    with J.HashTable(k, none) as t:
        assert t.info().null_rows == 64
        assert t.probe_gather(k).count == 0
    with J.HashTable(k) as t:
        assert t.probe_gather(k, none).count == 0
    with J.HashTable(k, none, null_equality=1) as t:  # NULL = NULL: 64 x 64 pairs
        assert t.probe_gather(k, none).count == 64 * 64


def test_capacity_overflow_reports_total(cuda):
    from sirius_b200 import join as J
    b = torch.tensor([7, 7, 7, 8], dtype=torch.int32, device=cuda)
    p = torch.tensor([7, 7, 8, 9], dtype=torch.int32, device=cuda)
    with J.HashTable(b) as t:
        out = J.allocate_output(4)
        d = torch.zeros(1, dtype=torch.int64, device=cuda)
        t.probe_gather(p, out=out, capacity=4, d_count=d, sync=False)
        torch.cuda.synchronize()
        assert int(d.item()) == 7
        with pytest.raises(Exception):
            t.probe_gather(p, capacity=4)
        full = t.probe_gather(p).trimmed()
        assert full.count == 7


def test_payload_validity_propagates(cuda):
    rng = np.random.default_rng(5)
    nb, np_ = 4000, 30000
    bk = rng.permutation(nb).astype(np.int32)
    pk = rng.integers(0, nb + 500, np_).astype(np.int32)
    bpv = rng.random(nb) > 0.4
    ppv = rng.random(np_) > 0.4
    bp = rng.integers(0, 1000, nb).astype(np.int64)
    pp = rng.integers(0, 1000, np_).astype(np.int32)
    from sirius_b200 import join as J
    for layout in (0, 2):
        with J.HashTable(dev_t(bk, cuda), layout=layout) as t:
            out = t.probe_gather(dev_t(pk, cuda), None, [(dev_t(pp, cuda), dev_valid(O.pack_validity(ppv), cuda))],
                                 [(dev_t(bp, cuda), dev_valid(O.pack_validity(bpv), cuda))]).trimmed()
        torch.cuda.synchronize()
        prid, brid = out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()
        n = out.count
        got_pv = O.unpack_validity(out.probe_payload_validity[0].cpu().numpy().view(np.uint32), n)
        got_bv = O.unpack_validity(out.build_payload_validity[0].cpu().numpy().view(np.uint32), n)
        assert np.array_equal(got_pv, ppv[prid])
        assert np.array_equal(got_bv, bpv[brid])
        assert np.array_equal(out.build_payload[0].cpu().numpy(), bp[brid])
        assert np.array_equal(out.probe_payload[0].cpu().numpy(), pp[prid])


def test_unaligned_and_offset_columns(cuda):
    """Key columns that start off a 16-byte boundary and validity with a bit offset."""
    from sirius_b200 import join as J
    from sirius_b200._lib import SjColumn  # noqa: F401
    rng = np.random.default_rng(8)
    bk = rng.permutation(3001).astype(np.int64)
    pk = rng.integers(0, 3500, 9001).astype(np.int64)
    pvalid = rng.random(9001) > 0.1
    bkt = dev_t(bk, cuda)[1:]      # 8-byte aligned, not 16
    pkt = dev_t(pk, cuda)[1:]
    words = dev_valid(O.pack_validity(pvalid), cuda)
    with J.HashTable(bkt) as t:
        key = J.make_column(pkt, words, validity_offset=1)
        d = torch.zeros(1, dtype=torch.int64, device=cuda)
        lib = t._lib
        import ctypes
        assert lib.sj_probe_count(t.handle, ctypes.byref(key), 1, None, torch.cuda.current_stream().cuda_stream,
                                  d.data_ptr()) == 0
        torch.cuda.synchronize()
    exp = O.hash_join_count(bk[1:], pk[1:], None, O.pack_validity(pvalid[1:]))
    assert int(d.item()) == exp


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.float32, np.float64, np.uint32])
def test_payload_widths(cuda, dtype):
    rng = np.random.default_rng(3)
    nb, np_ = 2000, 9000
    bk = rng.integers(0, 1500, nb).astype(np.int32)   # duplicates -> grouped
    pk = rng.integers(0, 1700, np_).astype(np.int32)
    def vals(n):
        return (rng.random(n) * 100).astype(dtype) if np.issubdtype(dtype, np.floating) else \
            rng.integers(0, 100, n).astype(dtype)
    inp = D.JoinInput("w", bk, pk, [vals(nb), vals(nb)], [vals(np_)])
    got, _ = gpu_join(inp, cuda)
    assert_same_rows(got, oracle_join(inp))


def test_concurrent_probes_one_table(cuda):
    """Many read-only probes of one built table on different streams (BUILD_PROBE pattern)."""
    from sirius_b200 import join as J
    inp = D.small(4, 50000, 100000)
    bk = dev_t(inp.build_keys, cuda)
    probes = [D.small(10 + i, 50000, 100000).probe_keys for i in range(4)]
    with J.HashTable(bk) as t:
        torch.cuda.synchronize()
        streams = [torch.cuda.Stream() for _ in range(4)]
        runs = []
        for s, p in zip(streams, probes):
            with torch.cuda.stream(s):
                pt = dev_t(p, cuda)
                d = torch.zeros(1, dtype=torch.int64, device=cuda)
                o = t.probe_gather(pt, stream=s, capacity=len(p), sync=False, d_count=d)
                runs.append((pt, d, o))
        torch.cuda.synchronize()
        for p, (_, d, o) in zip(probes, runs):
            n = int(d.item())
            r = O.hash_join(inp.build_keys, p)
            assert n == r.rows
            got = O.canonical(o.probe_rid[:n].cpu().numpy(), o.build_rid[:n].cpu().numpy())
            exp = O.canonical(r.probe_rid, r.build_rid)
            assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1])


@pytest.mark.parametrize("n_probe", [1, 2, 3, 31, 33, 255, 257, 1023, 1025, 2047, 2049, 4097, 31784, 262145])
def test_grouped_sizes_across_scan_blocks(cuda, n_probe):
    """Output offsets of the grouped probe come from a multi-block scan; sweep entry counts around
    its block and tile boundaries and check the exact row multiset."""
    rng = np.random.default_rng(n_probe)
    bk = rng.integers(0, 300, 2000).astype(np.int32)   # ~7 rows per key
    pk = rng.integers(0, 330, n_probe).astype(np.int32)
    inp = D.JoinInput("g", bk, pk, [rng.integers(0, 99, 2000).astype(np.int32)], [])
    got, info = gpu_join(inp, cuda)
    assert info.layout == 2
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("pbits", [1, 4, 7, 10])
@pytest.mark.parametrize("attach", [False, True])
def test_partitioned_distinct(cuda, pbits, attach):
    """Radix-partitioned table (segments = partitions) and the partitioned probe path."""
    inp = D.large(6, n_build=1 << 20, n_probe=3 << 20)
    got, info = gpu_join(inp, cuda, attach=attach, partition_bits=pbits)
    assert info.partition_bits == pbits and info.layout == 1
    assert_same_rows(got, oracle_join(inp))


def test_partitioned_auto_on_large_footprint(cuda):
    inp = D.large(7, n_build=4 << 20, n_probe=1 << 20)
    got, info = gpu_join(inp, cuda, attach=True)
    assert info.partition_bits > 0   # 4M keys: slots + attached payloads exceed the L2 budget
    assert_same_rows(got, oracle_join(inp))
    got, info = gpu_join(inp, cuda, attach=True, partition_bits=-1)
    assert info.partition_bits == 0
    assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("pbits", [-1, 3])
def test_partitioned_with_nulls_and_payload_validity(cuda, pbits):
    rng = np.random.default_rng(41)
    nb, np_ = 200_000, 900_000
    bk = rng.permutation(nb).astype(np.int64) * 3 - 100
    pk = (rng.integers(0, nb + 5000, np_) * 3 - 100).astype(np.int64)
    bpv, ppv = rng.random(nb) > 0.3, rng.random(np_) > 0.3
    bp = rng.integers(0, 1 << 40, nb).astype(np.int64)
    pp = rng.integers(0, 1 << 20, np_).astype(np.int32)
    kbv, kpv = rng.random(nb) > 0.05, rng.random(np_) > 0.05
    from sirius_b200 import join as J
    for attach in (False, True):
        bpay = [(dev_t(bp, cuda), dev_valid(O.pack_validity(bpv), cuda))]
        ppay = [(dev_t(pp, cuda), dev_valid(O.pack_validity(ppv), cuda))]
        with J.HashTable(dev_t(bk, cuda), dev_valid(O.pack_validity(kbv), cuda), partition_bits=pbits,
                         attach=bpay if attach else ()) as t:
            kw = dict(attached=True) if attach else dict(build_payload=bpay)
            out = t.probe_gather(dev_t(pk, cuda), dev_valid(O.pack_validity(kpv), cuda), ppay, **kw).trimmed()
        torch.cuda.synchronize()
        ref = O.hash_join(bk, pk, O.pack_validity(kbv), O.pack_validity(kpv))
        n = out.count
        assert n == ref.rows
        prid, brid = out.probe_rid.cpu().numpy(), out.build_rid.cpu().numpy()
        a = O.canonical(prid, brid)
        b = O.canonical(ref.probe_rid, ref.build_rid)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert np.array_equal(out.build_payload[0].cpu().numpy()[bpv[brid]], bp[brid][bpv[brid]])
        assert np.array_equal(out.probe_payload[0].cpu().numpy()[ppv[prid]], pp[prid][ppv[prid]])
        gv = O.unpack_validity(out.build_payload_validity[0].cpu().numpy().view(np.uint32), n)
        pvv = O.unpack_validity(out.probe_payload_validity[0].cpu().numpy().view(np.uint32), n)
        assert np.array_equal(gv, bpv[brid]) and np.array_equal(pvv, ppv[prid])


@pytest.mark.parametrize("pbits", [2, 6])
def test_partitioned_grouped(cuda, pbits):
    """Duplicated build keys in a partitioned table: grouped ranges hold table positions."""
    inp = D.skewed(8, n_build=1 << 19, n_probe=1 << 21, build_values=1 << 16, probe_values=1 << 17)
    for attach in (False, True):
        got, info = gpu_join(inp, cuda, attach=attach, partition_bits=pbits)
        assert info.layout == 2 and info.partition_bits == pbits
        assert_same_rows(got, oracle_join(inp))


def test_attached_with_null_group(cuda):
    """NULLs equal with NULL build keys: attached columns stay in row order."""
    rng = np.random.default_rng(12)
    bk = rng.integers(0, 50, 3000).astype(np.int32)
    pk = rng.integers(0, 60, 9000).astype(np.int32)
    inp = D.JoinInput("ng", bk, pk, [rng.integers(0, 1000, 3000).astype(np.int32)], [],
                      O.pack_validity(rng.random(3000) > 0.1), O.pack_validity(rng.random(9000) > 0.1))
    got, info = gpu_join(inp, cuda, attach=True, null_equality=1)
    assert info.layout == 2
    assert_same_rows(got, oracle_join(inp, nulls_equal=True))


@pytest.mark.parametrize("agg", [1, 2])
@pytest.mark.parametrize("pbits", [-1, 3])
def test_output_aggregation_modes(cuda, agg, pbits):
    """Per-warp and per-CTA output reservation give the same rows."""
    inp = D.small(13, 300_000, 2_000_000)
    for attach in (False, True):
        got, info = gpu_join(inp, cuda, attach=attach, aggregation=agg, partition_bits=pbits)
        assert_same_rows(got, oracle_join(inp))


@pytest.mark.parametrize("pdt", [np.int32, np.int64])
@pytest.mark.parametrize("pbits", [-1, 3])
@pytest.mark.parametrize("probe_nulls", [False, True])
def test_grouped_single_attached_payload_shapes(cuda, pdt, pbits, probe_nulls):
    """A GROUPED table with one attached 4- or 8-byte payload and no probe payload: the expand's
    compile-time record shapes (8- and 16-byte records). Skewed groups span many output tiles."""
    rng = np.random.default_rng(31)
    nb, npr = 200_000, 600_001
    bk = np.concatenate([rng.integers(0, 40_000, nb - 3000), np.full(3000, 7)]).astype(np.int64)
    rng.shuffle(bk)
    pk = rng.integers(-1000, 41_000, npr).astype(np.int64)
    pk[rng.random(npr) < 0.001] = 7  # a key with 3,000+ copies: one probe row spans several tiles
    bp = [rng.integers(-2**31, 2**31 - 1, nb).astype(pdt)]
    pv = O.pack_validity(rng.random(npr) > 0.1) if probe_nulls else None
    inp = D.JoinInput("grouped-shapes", bk, pk, bp, [], None, pv)
    got, info = gpu_join(inp, cuda, attach=True, partition_bits=pbits)
    assert info.layout == 2
    assert_same_rows(got, oracle_join(inp))
