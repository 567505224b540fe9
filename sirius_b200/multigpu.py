"""Host logic of the multi-GPU join: one process per GPU, a replicated build and a sharded probe.

The INNER join's units of work are probe rows; with the build table replicated on every rank
(the reference's broadcast join for small builds, src/op/sirius_physical_hash_join.cpp:699-702)
every rank probes its own shard and no data moves between GPUs, so scaling is weak: per-rank work
is fixed and the job's throughput is all ranks' rows over the slowest rank's time.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class RankInfo:
    rank: int
    world: int
    local_rank: int


def rank_info() -> RankInfo:
    return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def probe_shard(build_keys: np.ndarray, n_probe: int, seed: int, rank: int):
    """Rank `rank`'s probe shard of the large 1:1 workload: keys drawn uniformly from the
    (replicated) build keys with the rank's own seeded stream, and an int64 payload."""
    rng = np.random.default_rng([seed, rank])
    keys = build_keys[rng.integers(0, len(build_keys), n_probe)]
    payload = rng.integers(-2**63, 2**63 - 1, n_probe, dtype=np.int64, endpoint=True)
    return keys, payload


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank scalar over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(rows_per_rank_per_step: int, steps: int, world: int, max_ms: float) -> float:
    """Job throughput in M rows/s: every rank's rows over the slowest rank's time."""
    return rows_per_rank_per_step * steps * world / (max_ms / 1e3) / 1e6


# ------------------------------------------------------------------------------------------------
# Hash-partitioned join across ranks: one all-to-all exchange, then independent local joins
# ------------------------------------------------------------------------------------------------
def gpu_partitioner(keys, columns, world: int):
    """Partition step on the GPU: sj_hash_partition over `world` partitions (a power of two).
    Returns (partitioned columns, per-partition row counts as a CPU int64 tensor)."""
    from . import join as J
    outs, _, offsets = J.hash_partition(keys, columns, world)
    return outs, (offsets[1:] - offsets[:-1]).cpu()


def exchange(keys, columns, partitioner=gpu_partitioner, group=None):
    """All-to-all by hash partition (the exchange step of a partitioned join: both sides hash-
    partitioned on h(key) mod world, one grouped all-to-all, then local joins — over NCCL on GPUs,
    any torch.distributed backend here). `keys` (one tensor, no NULLs) and `columns` (tensors of the
    same length) are this rank's rows; returns (keys, columns) of the rows every rank sent here,
    i.e. this rank's partition of the union. The partition counts go first (one small all-to-all),
    then each column in one all_to_all_single with those splits."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts, send_counts = partitioner(keys, [keys] + list(columns), world)
    send_counts = send_counts.to(torch.int64)
    dev = keys.device
    sc = send_counts.to(dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = rc.cpu()
    send_splits = [int(x) for x in send_counts]
    recv_splits = [int(x) for x in recv_counts]
    received = []
    for col in parts:
        out = torch.empty(sum(recv_splits), dtype=col.dtype, device=dev)
        dist.all_to_all_single(out, col.contiguous(), recv_splits, send_splits, group=group)
        received.append(out)
    return received[0], received[1:]


def partitioned_inner_join(build_keys, build_cols, probe_keys, probe_cols, local_join,
                           partitioner=gpu_partitioner, group=None):
    """INNER join of row-sharded tables across ranks (keys without NULLs: a NULL key never matches,
    so such rows are dropped before the exchange): exchange both sides by hash partition, then
    `local_join(build_keys, build_cols, probe_keys, probe_cols)` on this rank's partition. Every
    matching pair lands on exactly one rank (equal keys share a partition)."""
    bk, bc = exchange(build_keys, build_cols, partitioner, group)
    pk, pc = exchange(probe_keys, probe_cols, partitioner, group)
    return local_join(bk, bc, pk, pc)
