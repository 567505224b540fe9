"""The partitioned multi-GPU join path on the GPU with a one-rank NCCL process group: the GPU
partition step (sj_hash_partition), the NCCL all-to-all of counts and columns, and the local join
on the GPU, against the oracle. (More ranks run the same code; this machine gives one GPU, and the
exchange logic across two ranks is tested with gloo in test_multiproc.py.)"""
import os
import tempfile

import numpy as np
import pytest
import torch

from jhelp import dev_t
from oracle import oracle as O
from sirius_b200 import join as J
from sirius_b200 import multigpu as M

pytestmark = pytest.mark.gpu


def test_partitioned_join_one_rank_nccl(cuda):
    import torch.distributed as dist
    store = dist.FileStore(os.path.join(tempfile.mkdtemp(), "store"), 1)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, device_id=cuda)
    try:
        rng = np.random.default_rng(4)
        bk = rng.permutation(200_000).astype(np.int64)
        pk = rng.integers(0, 250_000, 1_000_000).astype(np.int64)
        bp = rng.integers(0, 1 << 40, len(bk)).astype(np.int64)
        pp = rng.integers(0, 1 << 40, len(pk)).astype(np.int64)

        def local_join(k, c, q, d):
            with J.HashTable(k, attach=[c[0]]) as t:
                out = t.probe_gather(q, None, [d[0]], attached=True).trimmed()
            return out.probe_payload[0].cpu().numpy(), out.build_payload[0].cpu().numpy()

        got_p, got_b = M.partitioned_inner_join(dev_t(bk, cuda), [dev_t(bp, cuda)], dev_t(pk, cuda),
                                                [dev_t(pp, cuda)], local_join)
        ref = O.hash_join(bk, pk, probe_payload=[pp], build_payload=[bp])
        assert sorted(zip(got_p.tolist(), got_b.tolist())) == sorted(zip(ref.probe_payload[0].tolist(),
                                                                         ref.build_payload[0].tolist()))
    finally:
        dist.destroy_process_group()
