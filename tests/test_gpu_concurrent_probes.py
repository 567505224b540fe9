"""GPU stress test of partitioned probes running at the same time on several streams into one
resident table (the served case: sj_probe_* called concurrently on one built table). Every probe's
result must be the same as the same probe run alone, and its match count the oracle's. The
tile-local partition and the run-walking probe of a partitioned table are timing-sensitive (CTAs
take work items from a shared counter, per-tile run tables are built in shared memory), so the
probes are repeated with the streams competing for the SMs."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sirius_b200 import join as J

pytestmark = pytest.mark.gpu

N_BUILD = 1 << 24
N_PROBE = 3_000_001
STREAMS = 4
ROUNDS = 4


def _rows(out, count):
    return O.canonical(out.probe_rid[:count].cpu().numpy(), out.build_rid[:count].cpu().numpy(),
                       out.build_payload[0][:count].cpu().numpy())


def test_concurrent_partitioned_probes_match_alone(cuda):
    g = torch.Generator(device=cuda)
    g.manual_seed(11)
    bk = torch.randperm(2 * N_BUILD, device=cuda, generator=g)[:N_BUILD].to(torch.int64)
    bp = torch.randint(-2**40, 2**40, (N_BUILD,), device=cuda, generator=g, dtype=torch.int64)
    probes = []
    for _ in range(STREAMS):
        pk = bk[torch.randint(0, N_BUILD, (N_PROBE,), device=cuda, generator=g)]
        miss = torch.rand(N_PROBE, device=cuda, generator=g) < 0.25
        absent = torch.randint(2 * N_BUILD, 3 * N_BUILD, (N_PROBE,), device=cuda, generator=g)
        probes.append(torch.where(miss, absent, pk).contiguous())
    torch.cuda.synchronize()
    with J.HashTable(bk, partition_bits=6, attach=[bp]) as t:
        assert t.info().partition_bits > 0
        bkh = bk.cpu().numpy()
        alone = []
        for pk in probes:
            out = t.probe_gather(pk, attached=True)
            assert out.count == int(np.isin(pk.cpu().numpy(), bkh).sum())
            alone.append((out.count, _rows(out, out.count)))
        streams = [torch.cuda.Stream(device=cuda) for _ in range(STREAMS)]
        counts = [torch.empty(1, dtype=torch.int64, device=cuda) for _ in range(STREAMS)]
        for rnd in range(ROUNDS):
            torch.cuda.synchronize()
            outs = [t.probe_gather(pk, attached=True, capacity=N_PROBE, stream=s, sync=False, d_count=dc)
                    for pk, s, dc in zip(probes, streams, counts)]
            torch.cuda.synchronize()
            for q, (out, dc) in enumerate(zip(outs, counts)):
                c = int(dc.item())
                assert c == alone[q][0], f"round {rnd}, stream {q}: {c} matches, {alone[q][0]} alone"
                for a, b in zip(_rows(out, c), alone[q][1]):
                    assert np.array_equal(a, b), f"round {rnd}, stream {q}: rows differ from the probe alone"
