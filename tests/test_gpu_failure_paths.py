"""Failure paths of the join, none of which faults or hangs the GPU:

* allocation refusals: an sj_alloc whose callback returns NULL on its Nth call, for every N from
  the first allocation until the call succeeds, across the build (partitioned row store, grouped
  layout with NULL keys), the partitioned probe's scratch, the grouped probe's match list and the
  one-shot join. Every refusal must come back as SJ_ERR_OOM (the status the adapter turns into
  rmm::out_of_memory, which Sirius reschedules: src/pipeline/gpu_pipeline_task.cpp:386-437), and
  the callback's ledger must show every byte the library took returned;
* SJ_ERR_TABLE_FULL: build keys whose hashes all fall into one of 1,024 table segments (found by
  inverting the hash on the host), more keys than that segment has slots;
* bounded device waits: the batched join's wait for a join's build and the TMA probe ring's
  mbarrier wait, run on conditions that never come true, give up and report it, and the context
  stays usable for a join afterwards."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu


class Ledger:
    """sj_alloc over torch's caching allocator that records live allocations and refuses call
    number `fail_at` (1-based; 0 = never)."""

    def __init__(self):
        self.live = {}
        self.calls = 0
        self.fail_at = 0
        self._a = L.ALLOC_FN(self._alloc)
        self._f = L.FREE_FN(self._free)
        self.alloc = L.SjAlloc(None, self._a, self._f)

    def _alloc(self, ctx, nbytes, stream):
        self.calls += 1
        if self.fail_at and self.calls == self.fail_at:
            return None
        s = stream if stream else torch.cuda.current_stream().cuda_stream
        p = torch.cuda.caching_allocator_alloc(max(int(nbytes), 1), torch.cuda.current_device(), s)
        self.live[p] = int(nbytes)
        return p

    def _free(self, ctx, ptr, nbytes, stream):
        assert ptr in self.live, "the library freed memory it did not get from this allocator"
        assert self.live.pop(ptr) == int(nbytes), "freed with another size than allocated"
        torch.cuda.caching_allocator_delete(ptr)

    @property
    def ref(self):
        return ctypes.byref(self.alloc)


def _sweep(run, ledger, max_n=200):
    """run() -> status with ledger.fail_at set to 1, 2, ... until it succeeds; every failure must be
    SJ_ERR_OOM with the ledger back where it was. Returns the number of refusals checked."""
    for n in range(1, max_n + 1):
        before = dict(ledger.live)
        ledger.calls = 0
        ledger.fail_at = n
        st = run()
        torch.cuda.synchronize()
        ledger.fail_at = 0
        if st == L.SJ_OK:
            assert ledger.calls < n, "a call succeeded although one of its allocations was refused"
            return n - 1
        assert st == L.SJ_ERR_OOM, (n, L.status_name(st), L.load().sj_last_error())
        assert ledger.live == before, f"refusal {n}: {len(ledger.live) - len(before)} allocations leaked"
    raise AssertionError("the call never succeeded")


def _build(ledger, keys, validity=None, attach=(), **params):
    lib = L.load()
    col = J.make_column(keys, validity)
    p = L.default_params(**params)
    h = ctypes.c_void_p()
    pay = [J.make_column(a) for a in attach]
    s = torch.cuda.current_stream().cuda_stream
    if pay:
        st = lib.sj_build_ex(ctypes.byref(col), 1, J._cols(pay), len(pay), ctypes.byref(p), ledger.ref, s,
                             ctypes.byref(h))
    else:
        st = lib.sj_build(ctypes.byref(col), 1, ctypes.byref(p), ledger.ref, s, ctypes.byref(h))
    return st, h


def _destroy(h):
    L.load().sj_table_destroy(h, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()


@pytest.mark.parametrize("case", ["partitioned_row_store", "grouped_with_nulls"])
def test_build_refusals_return_oom_and_free_everything(cuda, case):
    rng = np.random.default_rng(3)
    n = 300_000
    led = Ledger()
    if case == "partitioned_row_store":
        keys = torch.from_numpy(rng.permutation(n).astype(np.int64) * 11).to(cuda)
        pay = [torch.from_numpy(rng.integers(0, 2**40, n)).to(cuda) for _ in range(2)]
        valid, params = None, dict(partition_bits=3)
    else:
        keys = torch.from_numpy(rng.integers(0, n // 8, n).astype(np.int64)).to(cuda)
        pay = [torch.from_numpy(rng.integers(0, 2**31, n).astype(np.int32)).to(cuda)]
        valid = torch.from_numpy(O.pack_validity(rng.random(n) > 0.1).view(np.int32)).to(cuda)
        params = {}
    handles = []

    def run():
        st, h = _build(led, keys, valid, pay, **params)
        if st == L.SJ_OK:
            handles.append(h)
        return st

    refusals = _sweep(run, led)
    assert refusals >= 3
    _destroy(handles[-1])
    assert led.live == {}


@pytest.mark.parametrize("grouped", [False, True])
def test_probe_refusals_return_oom_and_free_everything(cuda, grouped):
    rng = np.random.default_rng(4)
    nb, np_ = 200_000, 1 << 18
    led = Ledger()
    bk = (rng.integers(0, nb // 4, nb) if grouped else rng.permutation(nb)).astype(np.int64)
    pk = rng.integers(0, nb, np_).astype(np.int64)
    bp = torch.from_numpy(rng.integers(0, 2**40, nb)).to(cuda)
    pp = torch.from_numpy(rng.integers(0, 2**40, np_)).to(cuda)
    st, h = _build(led, torch.from_numpy(bk).to(cuda), None, [bp], partition_bits=0 if grouped else 3)
    assert st == L.SJ_OK
    table_bytes = dict(led.live)
    exp = O.hash_join_count(bk, pk)
    pkd = torch.from_numpy(pk).to(cuda)
    out = J.allocate_output(exp, [pp], [bp], cuda)
    lib = L.load()
    d = torch.zeros(1, dtype=torch.int64, device=cuda)

    def run():
        return lib.sj_probe_gather(
            h, ctypes.byref(J.make_column(pkd)), 1, J._cols([J.make_column(pp)]), 1, None, 1,
            out.probe_rid.data_ptr(), out.build_rid.data_ptr(),
            J._cols([J._mut(out.probe_payload[0], None)], L.SjMutColumn),
            J._cols([J._mut(out.build_payload[0], None)], L.SjMutColumn), exp, led.ref,
            torch.cuda.current_stream().cuda_stream, d.data_ptr())

    _sweep(run, led)
    assert int(d.item()) == exp
    assert led.live == table_bytes  # the probe returned all of its scratch
    _destroy(h)
    assert led.live == {}


def test_one_shot_join_refusals(cuda):
    rng = np.random.default_rng(5)
    nb, np_ = 100_000, 400_000
    led = Ledger()
    bk = torch.from_numpy(rng.permutation(nb).astype(np.int32)).to(cuda)
    pk = torch.from_numpy(rng.integers(0, nb + nb // 10, np_).astype(np.int32)).to(cuda)
    lib = L.load()
    d = torch.zeros(1, dtype=torch.int64, device=cuda)
    prid = torch.empty(np_, dtype=torch.int32, device=cuda)
    brid = torch.empty(np_, dtype=torch.int32, device=cuda)

    def run():
        return lib.sj_inner_join(ctypes.byref(J.make_column(bk)), ctypes.byref(J.make_column(pk)), 1, None, 0, None,
                                 0, prid.data_ptr(), brid.data_ptr(), None, None, np_, None, led.ref,
                                 torch.cuda.current_stream().cuda_stream, d.data_ptr())

    assert _sweep(run, led) >= 2
    assert led.live == {}
    assert int(d.item()) == O.hash_join_count(bk.cpu().numpy(), pk.cpu().numpy())


# ---- SJ_ERR_TABLE_FULL ------------------------------------------------------------------------
M64 = (1 << 64) - 1
C1, C2 = 0xBF58476D1CE4E5B9, 0x94D049BB133111EB


def _mix64(x):
    x ^= x >> 30
    x = (x * C1) & M64
    x ^= x >> 27
    x = (x * C2) & M64
    x ^= x >> 31
    return x


def _unmix64(h):
    """Inverse of the splitmix64 finalizer the table hashes keys with."""
    h ^= (h >> 31) ^ (h >> 62)
    h = (h * pow(C2, -1, 1 << 64)) & M64
    h ^= (h >> 27) ^ (h >> 54)
    h = (h * pow(C1, -1, 1 << 64)) & M64
    h ^= (h >> 30) ^ (h >> 60)
    return h


def test_table_full_when_one_segment_overflows(cuda):
    # hashes 1..n all have their top 10 bits zero: every key lands in segment 0 of 1,024, whose
    # 2^(log2 buckets - 10) buckets hold far fewer than n keys
    n = 50_000
    keys = np.array([_unmix64(i) for i in range(1, n + 1)], dtype=np.uint64).view(np.int64)
    assert all(_mix64(int(k) & M64) == i + 1 for i, k in enumerate(keys[:100]))
    led = Ledger()
    st, h = _build(led, torch.from_numpy(keys).to(cuda), partition_bits=10)
    torch.cuda.synchronize()
    assert st == L.SJ_ERR_TABLE_FULL, L.status_name(st)
    assert b"ran out of slots" in L.load().sj_last_error()
    assert led.live == {}
    # the same keys spread over an unpartitioned table build fine
    st, h = _build(led, torch.from_numpy(keys).to(cuda), partition_bits=-1)
    assert st == L.SJ_OK
    _destroy(h)


# ---- bounded device waits -----------------------------------------------------------------------
def test_bounded_waits_give_up_and_the_context_survives(cuda):
    lib = L.load()
    status = torch.full((3,), -1, dtype=torch.int32, device=cuda)
    L.check(lib.sj_debug_wait_timeout(2000, torch.cuda.current_stream().cuda_stream, status.data_ptr()),
            "sj_debug_wait_timeout")
    torch.cuda.synchronize()
    assert status[:2].tolist() == [1, 1]  # both waits gave up
    # the GPU context still serves joins
    bk = torch.arange(1000, dtype=torch.int64, device=cuda)
    out = J.inner_join(bk, bk.flip(0))
    assert out.count == 1000
