"""Multi-process (world size 2, gloo, CPU) checks of the multi-GPU host logic: each rank's probe
shard is its own, every shard row matches the replicated build (checked with the CPU oracle),
and the job throughput uses the slowest rank's time (max over ranks)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import torch.distributed as dist
    from oracle import oracle as O
    from sirius_b200 import datagen as D
    from sirius_b200 import multigpu as M
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inp = D.large(3, n_build=1 << 14, n_probe=1 << 10)   # every rank: the same build side
        keys, pay = M.probe_shard(inp.build_keys, 50_000, 3, rank)
        m = O.hash_join_count(inp.build_keys, keys, threads=1)
        local_ms = 10.0 + rank * 5.0                          # a slower rank 1
        mx = M.max_over_ranks(local_ms)
        val = M.weak_scaling_value(50_000, 4, world, mx)
        shard_sum = int(keys.astype(np.int64).sum() & 0xFFFFFFFF)
        q.put((rank, m, mx, val, shard_sum, M.rank_info().world))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, mx0, v0, s0, w0), (r1, m1, mx1, v1, s1, w1) = res
    assert m0 == 50_000 and m1 == 50_000          # 1:1 workload: every shard row matches once
    assert mx0 == mx1 == 15.0                     # slowest rank's time on every rank
    assert v0 == v1 == pytest.approx(50_000 * 4 * 2 / 0.015 / 1e6)
    assert s0 != s1                               # each rank probes its own shard
    assert w0 == w1 == 2


def _exchange_worker(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from sirius_b200 import multigpu as M
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def cpu_partitioner(keys, columns, w):
        # the partition rule of sj_hash_partition (the oracle's restatement), applied on the host
        part = O.partition_ids([keys.numpy()], [None], w)
        order = np.argsort(part, kind="stable")
        counts = np.bincount(part, minlength=w)
        return [c[torch.from_numpy(order)] for c in columns], torch.from_numpy(counts.astype(np.int64))

    def local_join(bk, bc, pk, pc):
        r = O.hash_join(bk.numpy(), pk.numpy(), probe_payload=[pc[0].numpy()], build_payload=[bc[0].numpy()],
                        threads=1)
        return [r.probe_payload[0], r.build_payload[0]]

    try:
        rng = np.random.default_rng([9, rank])
        bk = rng.integers(0, 3000, 4000).astype(np.int64)       # duplicates across ranks
        pk = rng.integers(-50, 3500, 9000).astype(np.int64)
        bid = (rank * 10_000_000 + np.arange(len(bk))).astype(np.int64)  # global row ids as payloads
        pid = (rank * 10_000_000 + np.arange(len(pk))).astype(np.int64)
        out = M.partitioned_inner_join(torch.from_numpy(bk), [torch.from_numpy(bid)], torch.from_numpy(pk),
                                       [torch.from_numpy(pid)], local_join, partitioner=cpu_partitioner)
        q.put((rank, out[0].tolist(), out[1].tolist(), bk.tolist(), pk.tolist()))
    finally:
        dist.destroy_process_group()


def test_partitioned_exchange_join_gloo():
    """The union over ranks of the local joins after the hash exchange equals the global INNER join
    of the sharded tables (as (probe global id, build global id) pairs), with no pair twice."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import oracle as O
    got = sorted(pair for r in res for pair in zip(r[1], r[2]))
    bk = np.concatenate([np.array(r[3], np.int64) for r in res])
    pk = np.concatenate([np.array(r[4], np.int64) for r in res])
    bid = np.concatenate([r[0] * 10_000_000 + np.arange(len(r[3])) for r in res]).astype(np.int64)
    pid = np.concatenate([r[0] * 10_000_000 + np.arange(len(r[4])) for r in res]).astype(np.int64)
    ref = O.hash_join(bk, pk, threads=2)
    exp = sorted(zip(pid[ref.probe_rid].tolist(), bid[ref.build_rid].tolist()))
    assert got == exp and len(set(got)) == len(got)
