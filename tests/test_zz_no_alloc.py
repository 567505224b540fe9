"""GPU test of sj_inner_join_noalloc, the one-shot join for callers that cannot allocate device
memory (a fully committed memory reservation, a latency-critical thread that must not wait in the
driver's allocator, or a host whose allocator belongs to another component). It takes all scratch
from a 64 MiB static device array instead of allocating. The test calls it through the C ABI
twice in a row (the second call runs on the array the first one left behind) and checks both
results row for row against the allocating entry point sj_inner_join, and that an input too
large for the array is refused with a clear error. Collected last so that a failure here leaves
every other test already run; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _inputs(dev, seed, dup):
    rng = np.random.default_rng(seed)
    nb, np_ = 60_000, 400_000
    bk = (rng.integers(0, nb // 3, nb) if dup else rng.permutation(nb)).astype(np.int64) * 7 - 1000
    pk = (rng.integers(0, nb + nb // 10, np_)).astype(np.int64) * 7 - 1000
    pv = O.pack_validity(rng.random(np_) > 0.05)
    bp = rng.integers(-2**40, 2**40, nb).astype(np.int64)
    pp = rng.integers(-2**20, 2**20, np_).astype(np.int32)
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    return t(bk), t(pk), t(pv.view(np.int32)), t(bp), t(pp)


def _run(fn_name, dev, bk, pk, pv, bp, pp, capacity):
    from sirius_b200 import _lib
    from sirius_b200 import join as J
    lib = _lib.load()
    bcol = J.make_column(bk)
    pcol = J.make_column(pk, pv)
    pin = J._cols([J.make_column(pp)])
    bin_ = J._cols([J.make_column(bp)])
    out = J.allocate_output(capacity, [pp], [bp], dev)
    pout = J._cols([J._mut(out.probe_payload[0], None)], _lib.SjMutColumn)
    bout = J._cols([J._mut(out.build_payload[0], None)], _lib.SjMutColumn)
    d = torch.full((1,), -1, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    args = [ctypes.byref(bcol), ctypes.byref(pcol), 1, pin, 1, bin_, 1, out.probe_rid.data_ptr(),
            out.build_rid.data_ptr(), pout, bout, capacity, None]
    if fn_name == "sj_inner_join":
        st = lib.sj_inner_join(*args, None, s, d.data_ptr())
    else:
        st = lib.sj_inner_join_noalloc(*args, s, d.data_ptr())
    _lib.check(st, fn_name)
    torch.cuda.synchronize()
    n = int(d.item())
    assert 0 < n <= capacity
    return O.canonical(out.probe_rid[:n].cpu().numpy(), out.build_rid[:n].cpu().numpy(),
                       out.probe_payload[0][:n].cpu().numpy(), out.build_payload[0][:n].cpu().numpy())


@pytest.mark.parametrize("dup", [False, True])
def test_noalloc_matches_allocating_join_twice(cuda, dup):
    bk, pk, pv, bp, pp = _inputs(cuda, 5 + dup, dup)
    capacity = 4 * pk.numel() if dup else pk.numel()
    ref = _run("sj_inner_join", cuda, bk, pk, pv, bp, pp, capacity)
    first = _run("sj_inner_join_noalloc", cuda, bk, pk, pv, bp, pp, capacity)
    second = _run("sj_inner_join_noalloc", cuda, bk, pk, pv, bp, pp, capacity)
    for a, b, c in zip(ref, first, second):
        assert np.array_equal(a, b)  # integer outputs: bit-exact is the tolerance
        assert np.array_equal(a, c)


def test_noalloc_rejects_inputs_beyond_the_arena(cuda):
    from sirius_b200 import _lib
    from sirius_b200 import join as J
    lib = _lib.load()
    big = torch.zeros(8 << 20, dtype=torch.int64, device=cuda)
    col = J.make_column(big)
    d = torch.zeros(1, dtype=torch.int64, device=cuda)
    st = lib.sj_inner_join_noalloc(ctypes.byref(col), ctypes.byref(col), 1, None, 0, None, 0, None, None, None, None,
                                   0, None, torch.cuda.current_stream().cuda_stream, d.data_ptr())
    assert st == _lib.SJ_ERR_INVALID
    assert b"static arena holds" in lib.sj_last_error()
