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
