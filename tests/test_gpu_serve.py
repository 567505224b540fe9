"""GPU tests of the join server: every request's result is the same alone (one request on the GPU
at a time, no batching) and in the mix (several slots, requests admitted as slots and memory free
up, small requests batched into shared launches), and equal to the CPU oracle; small requests
really share launches; admission under a small memory budget; requests larger than the budget are
refused; closing a server whose queue cannot drain cancels the queued requests."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sirius_b200 import _lib as L
from sirius_b200 import datagen as D
from sirius_b200 import serve as S

pytestmark = pytest.mark.gpu

TABLE_ROWS = [1 << 20, 300_000, 3 << 20]


def _tables(dev, seed=5):
    out = []
    for t, n in enumerate(TABLE_ROWS):
        k, p = D.served_table_device(seed, t, n, dev)
        out.append((k, p))
    return out


def _requests(dev, tables, n, seed=9, lo=1e3, hi=1.5e6):
    ts, sizes, starts = D.served_requests(seed, n, len(tables), lo, hi)
    pools = [D.served_probe_pool(seed, t, k, int(hi) + 1) for t, (k, _) in enumerate(tables)]
    reqs = []
    for i in range(n):
        t, m = int(ts[i]), int(sizes[i])
        off = int(starts[i] * (pools[t].numel() - m))
        reqs.append((t, pools[t][off:off + m].contiguous()))
    torch.cuda.synchronize()
    return reqs


def _result_rows(r):
    """Host copy of a result, canonically sorted (probe rid, build rid, payload)."""
    c = int(r.count)
    cols = [r.probe_rid[:c].cpu().numpy(), r.build_rid[:c].cpu().numpy(), r.build_payload[0][:c].cpu().numpy()]
    return O.canonical(*cols)


def _run(server, tids, reqs, alone):
    got = {}
    if alone:
        for i, (t, pk) in enumerate(reqs):
            server.submit(tids[t], pk, i)
            res = []
            while not res:
                res = server.poll(4, wait_ms=1000)
            assert len(res) == 1 and res[0].request_id == i and res[0].status == L.SJ_OK
            got[i] = (res[0].count, _result_rows(res[0]))
            server.release(i)
        return got
    for i, (t, pk) in enumerate(reqs):
        server.submit(tids[t], pk, i, sync=(i == 0))
    while len(got) < len(reqs):
        for r in server.poll(64, wait_ms=1000):
            assert r.status == L.SJ_OK
            got[r.request_id] = (r.count, _result_rows(r))
            server.release(r.request_id)
    return got


def test_results_identical_alone_and_in_the_mix(cuda):
    tables = _tables(cuda)
    reqs = _requests(cuda, tables, 40)
    with S.JoinServer(slots=1, batch_small=False) as one:
        tids = [one.add_table(k, attach=[p], partition_bits=(3 if t == 2 else -1)) for t, (k, p) in enumerate(tables)]
        alone = _run(one, tids, reqs, alone=True)
    with S.JoinServer(slots=4) as many:
        tids = [many.add_table(k, attach=[p], partition_bits=(3 if t == 2 else -1))
                for t, (k, p) in enumerate(tables)]
        mixed = _run(many, tids, reqs, alone=False)
    assert sorted(alone) == sorted(mixed) == list(range(len(reqs)))
    for i in range(len(reqs)):
        assert alone[i][0] == mixed[i][0]
        for a, b in zip(alone[i][1], mixed[i][1]):
            assert np.array_equal(a, b), f"request {i} differs alone vs in the mix"
    # against the oracle, for a sample of requests
    host_tables = [(k.cpu().numpy(), p.cpu().numpy()) for k, p in tables]
    for i in range(0, len(reqs), 7):
        t, pk = reqs[i]
        bk, bp = host_tables[t]
        ref = O.hash_join(bk, pk.cpu().numpy(), build_payload=[bp], threads=8)
        assert ref.rows == alone[i][0]
        exp = O.canonical(ref.probe_rid, ref.build_rid, ref.build_payload[0])
        for a, b in zip(alone[i][1], exp):
            assert np.array_equal(a, b), f"request {i} differs from the oracle"


def test_small_requests_share_launches(cuda):
    """Hundreds of small requests (1K..60K rows) submitted at once run as a few batch launches: the
    requests of one batch complete together (one callback stamps them all). Each result equals the
    same request run alone without batching, and the oracle; wide (full-range int64) and packed
    (int32 key) tables are mixed in one batch."""
    tables = _tables(cuda)
    k32 = torch.randperm(200_000, device=cuda, dtype=torch.int64).to(torch.int32) * 3
    p32 = torch.randint(-2**60, 2**60, (200_000,), device=cuda, dtype=torch.int64)
    reqs = _requests(cuda, tables, 300, seed=21, lo=1e3, hi=6e4)
    g = torch.Generator(device=cuda)
    g.manual_seed(4)
    reqs += [(3, (torch.randint(0, 700_000, (int(n),), device=cuda, generator=g)).to(torch.int32))
             for n in np.random.default_rng(5).integers(1_000, 60_000, 60)]
    torch.cuda.synchronize()

    def serve(batch):
        with S.JoinServer(slots=4, batch_small=batch) as srv:
            tids = [srv.add_table(k, attach=[p], partition_bits=-1) for k, p in tables]
            tids.append(srv.add_table(k32, attach=[p32], partition_bits=-1))
            for i, (t, pk) in enumerate(reqs):
                srv.submit(tids[t], pk, i, sync=(i == 0))
            got, done_at = {}, {}
            while len(got) < len(reqs):
                for r in srv.poll(64, wait_ms=1000):
                    assert r.status == L.SJ_OK
                    got[r.request_id] = (r.count, _result_rows(r))
                    done_at[r.request_id] = r.t_done
                    srv.release(r.request_id)
        return got, done_at

    batched, done_at = serve(True)
    plain, _ = serve(False)
    groups = {}
    for i, t in done_at.items():
        groups.setdefault(t, []).append(i)
    assert len(groups) < len(reqs) // 4, f"{len(groups)} completion groups for {len(reqs)} requests"
    for i in range(len(reqs)):
        assert batched[i][0] == plain[i][0]
        for a, b in zip(batched[i][1], plain[i][1]):
            assert np.array_equal(a, b), f"request {i} differs batched vs alone"
    host = [(k.cpu().numpy(), p.cpu().numpy()) for k, p in tables] + [(k32.cpu().numpy(), p32.cpu().numpy())]
    for i in range(0, len(reqs), 11):
        t, pk = reqs[i]
        bk, bp = host[t]
        ref = O.hash_join(bk, pk.cpu().numpy(), build_payload=[bp], threads=8)
        assert ref.rows == batched[i][0]
        for a, b in zip(batched[i][1], O.canonical(ref.probe_rid, ref.build_rid, ref.build_payload[0])):
            assert np.array_equal(a, b), f"request {i} differs from the oracle"


def test_admission_under_a_small_budget(cuda):
    tables = _tables(cuda)[:2]
    reqs = _requests(cuda, tables, 24, seed=11, lo=5e4, hi=4e5)
    # outputs of the largest request: 2 x int32 rid + int64 payload per probe row
    largest = max(pk.numel() for _, pk in reqs) * 16
    budget = int(largest * 2.2)
    with S.JoinServer(slots=4, memory_budget_bytes=budget) as srv:
        tids = [srv.add_table(k, attach=[p], partition_bits=-1) for k, p in tables]
        for i, (t, pk) in enumerate(reqs):
            srv.submit(tids[t], pk, i, sync=(i == 0))
        done = {}
        while len(done) < len(reqs):
            for r in srv.poll(64, wait_ms=1000):
                assert r.status == L.SJ_OK
                done[r.request_id] = r
                srv.release(r.request_id)
        # outputs are held from admission past completion: the requests running at any admission
        # instant never hold more than the budget
        def a256(b):
            return (max(b, 16) + 255) // 256 * 256

        need = {i: 2 * a256(reqs[i][1].numel() * 4) + a256(reqs[i][1].numel() * 8) for i in done}
        for r in done.values():
            held = sum(need[q.request_id] for q in done.values() if q.t_admit <= r.t_admit < q.t_done)
            assert held <= budget
        with pytest.raises(L.SjError):
            big = torch.zeros(budget // 8, dtype=torch.int64, device=cuda)
            srv.submit(tids[0], big, 10_000)
    host_tables = [k.cpu().numpy() for k, _ in tables]
    for i, (t, pk) in enumerate(reqs):
        assert done[i].count == O.hash_join_count(host_tables[t], pk.cpu().numpy())


def test_close_cancels_requests_that_cannot_be_admitted(cuda):
    k, p = D.served_table_device(3, 0, 100_000, cuda)
    pk = k[:50_000].contiguous()
    torch.cuda.synchronize()
    srv = S.JoinServer(slots=2, memory_budget_bytes=50_000 * 16 + 4096)
    tid = srv.add_table(k, attach=[p], partition_bits=-1)
    srv.submit(tid, pk, 1)
    first = []
    while not first:
        first = srv.poll(1, wait_ms=1000)
    assert first[0].count == 50_000
    srv.submit(tid, pk, 2)  # cannot be admitted while request 1's outputs are held
    assert srv.poll(1, wait_ms=50) == []
    srv.close()  # returns: request 2 is cancelled
