"""GPU test of sj_inner_join_noalloc, the one-shot join for callers that cannot allocate device
memory (a fully committed memory reservation, a latency-critical thread that must not wait in the
driver's allocator, or a host whose allocator belongs to another component). It takes all scratch
from a 64 MiB static device array instead of allocating. The test calls it through the C ABI
twice in a row (the second call runs on the array the first one left behind) and checks both
results row for row against the allocating entry point sj_inner_join and the CPU oracle, that a
call after the first one takes no device memory from the driver or from torch's allocator, that
inputs at the documented limit are accepted and inputs past it refused with a clear error.
Collected last so that a failure here leaves every other test already run; it also passes alone in
a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _inputs(dev, seed, dup, nb=60_000, np_=400_000):
    rng = np.random.default_rng(seed)
    bk = (rng.integers(0, nb // 3, nb) if dup else rng.permutation(nb)).astype(np.int64) * 7 - 1000
    pk = (rng.integers(0, nb + nb // 10, np_)).astype(np.int64) * 7 - 1000
    pv = O.pack_validity(rng.random(np_) > 0.05)
    bp = rng.integers(-2**40, 2**40, nb).astype(np.int64)
    pp = rng.integers(-2**20, 2**20, np_).astype(np.int32)
    host = dict(bk=bk, pk=pk, pvalid=pv, bp=bp, pp=pp)
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    return host, (t(bk), t(pk), t(pv.view(np.int32)), t(bp), t(pp))


class _Call:
    """One join's C-ABI arguments and output buffers, allocated once so that repeated calls reuse them."""

    def __init__(self, dev, bk, pk, pv, bp, pp, capacity):
        from sirius_b200 import _lib
        from sirius_b200 import join as J
        self.lib = _lib.load()
        self.capacity = capacity
        self.keep = (bk, pk, pv, bp, pp)
        self.bcol = J.make_column(bk)
        self.pcol = J.make_column(pk, pv)
        self.pin = J._cols([J.make_column(pp)])
        self.bin = J._cols([J.make_column(bp)])
        self.out = J.allocate_output(capacity, [pp], [bp], dev)
        self.pout = J._cols([J._mut(self.out.probe_payload[0], None)], _lib.SjMutColumn)
        self.bout = J._cols([J._mut(self.out.build_payload[0], None)], _lib.SjMutColumn)
        self.d = torch.full((1,), -1, dtype=torch.int64, device=dev)

    def __call__(self, fn_name):
        from sirius_b200 import _lib
        s = torch.cuda.current_stream().cuda_stream
        args = [ctypes.byref(self.bcol), ctypes.byref(self.pcol), 1, self.pin, 1, self.bin, 1,
                self.out.probe_rid.data_ptr(), self.out.build_rid.data_ptr(), self.pout, self.bout, self.capacity, None]
        if fn_name == "sj_inner_join":
            st = self.lib.sj_inner_join(*args, None, s, self.d.data_ptr())
        else:
            st = self.lib.sj_inner_join_noalloc(*args, s, self.d.data_ptr())
        _lib.check(st, fn_name)
        torch.cuda.synchronize()
        return int(self.d.item())

    def rows(self, n):
        assert 0 < n <= self.capacity
        o = self.out
        return O.canonical(o.probe_rid[:n].cpu().numpy(), o.build_rid[:n].cpu().numpy(),
                           o.probe_payload[0][:n].cpu().numpy(), o.build_payload[0][:n].cpu().numpy())


def _oracle_rows(h):
    ref = O.hash_join(h["bk"], h["pk"], pvalid=h["pvalid"], probe_payload=[h["pp"]], build_payload=[h["bp"]])
    return O.canonical(ref.probe_rid, ref.build_rid, ref.probe_payload[0], ref.build_payload[0])


@pytest.mark.parametrize("dup", [False, True])
def test_noalloc_matches_allocating_join_twice(cuda, dup):
    h, cols = _inputs(cuda, 5 + dup, dup)
    capacity = 4 * cols[1].numel() if dup else cols[1].numel()
    c = _Call(cuda, *cols, capacity)
    ref = c.rows(c("sj_inner_join"))
    first = c.rows(c("sj_inner_join_noalloc"))
    # the second call: no device memory may be taken, from the driver or from torch's allocator
    free0, torch0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_stats()
    n2 = c("sj_inner_join_noalloc")
    free1, torch1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_stats()
    assert free1 == free0
    for k in ("allocation.all.allocated", "reserved_bytes.all.current", "allocated_bytes.all.current"):
        assert torch1.get(k) == torch0.get(k), k
    second = c.rows(n2)
    expect = _oracle_rows(h)
    for a, b, e, o in zip(ref, first, second, expect):
        assert np.array_equal(a, b)  # integer outputs: bit-exact is the tolerance
        assert np.array_equal(a, e)
        assert np.array_equal(a, o)


@pytest.mark.parametrize("nb,np_", [(1 << 19, 1_900_000), (1 << 20, 600_000)])
def test_noalloc_accepts_the_documented_limit(cuda, nb, np_):
    h, cols = _inputs(cuda, 11, False, nb=nb, np_=np_)
    c = _Call(cuda, *cols, np_)
    got = c.rows(c("sj_inner_join_noalloc"))
    for g, e in zip(got, _oracle_rows(h)):
        assert np.array_equal(g, e)


def test_noalloc_rejects_inputs_beyond_the_arena(cuda):
    from sirius_b200 import _lib
    from sirius_b200 import join as J
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    for nb, np_ in ((8 << 20, 8 << 20), (1 << 20, 700_000), ((1 << 19) + 1, 1_900_000)):
        bk = torch.zeros(nb, dtype=torch.int64, device=cuda)
        pk = torch.zeros(np_, dtype=torch.int64, device=cuda)
        bcol, pcol = J.make_column(bk), J.make_column(pk)
        d = torch.zeros(1, dtype=torch.int64, device=cuda)
        st = lib.sj_inner_join_noalloc(ctypes.byref(bcol), ctypes.byref(pcol), 1, None, 0, None, 0, None, None,
                                       None, None, 0, None, s, d.data_ptr())
        assert st == _lib.SJ_ERR_INVALID, (nb, np_)
        assert b"static arena holds" in lib.sj_last_error()
