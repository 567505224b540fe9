"""Benchmark of the sm_100a equi-hash-join on the large 1:1 foreign-key workload.

Workload (one "step" = one pass of the hot path over one probe batch):
  build 16M rows: unique int64 keys (seeded 40-bit Feistel permutation of 0..2^40) + two int64
  payloads; probe 64M rows: int64 keys drawn uniformly from the build keys (every probe matches
  once) + one int64 payload; output per match: probe rid, build rid (int32), probe payload and
  both build payloads (32 bytes).

Reported (one JSON line on rank 0):
  value     probe Mtuples/s of the probe phase (probe + payload gather + output write) against a
            device-resident table (the BUILD_PROBE pattern: build once, probe many), inputs
            resident in HBM; all ranks' probe rows / max-over-ranks time;
  e2e       the same metric for the one-shot join through the C ABI from pinned host buffers:
            H2D of all inputs + build + probe/gather + D2H of the whole output, per step;
  roofline  algorithmic bytes of the probe phase per launch / the probe kernel's average
            CUDA-event duration, against the measured HBM copy bandwidth;
  cpu_baseline  the CPU oracle join (all host threads) on the same workload.
Multi-GPU (torchrun): every rank builds the same table (a replicated build, the reference's
broadcast-join shape) and probes its own 64M-row shard: weak scaling, no data-path collective.

--impl reference: the CPU join (the oracle restatement of the reference's algorithm; the
reference itself cannot be built here) timed on the host cores on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NOMINAL_HBM_GBS = 8000.0
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sj", choices=["sj", "reference"])
    ap.add_argument("--n-build", type=int, default=None, help="build rows (default: the workload's)")
    ap.add_argument("--n-probe", type=int, default=None, help="probe rows (default: the workload's)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--partition-bits", type=int, default=0)
    ap.add_argument("--aggregation", type=int, default=0)
    ap.add_argument("--probe-kernel", type=int, default=0, help="0 auto, 1 staged write-out, 2 direct write-out")
    ap.add_argument("--rows-per-lane", type=int, default=0)
    ap.add_argument("--probe-partition-mb", type=int, default=0,
                    help="table MB per probe partition of the partitioned probe (0 = default)")
    ap.add_argument("--e2e-chunk-rows", type=int, default=0, help="probe rows per chunk of the e2e host join")
    ap.add_argument("--table-l2", type=int, default=0, help="L2 priority of table loads: 0 auto, 1 normal, 2 evict_last")
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--workload", default="large", choices=["large", "small", "skewed", "batched", "served", "next"])
    ap.add_argument("--autotune", action="store_true", help="batched: choose launch parameters by the autotuner")
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--slots", type=int, default=6,
                    help="served: concurrent request slots (4, 6, 8 measured 20.5, 21.5, 21.0 G rows/s)")
    ap.add_argument("--served-max-rows", type=int, default=20_000_000)
    ap.add_argument("--reserve-gib", type=int, default=16, help="served: device memory each server pool takes up front")
    ap.add_argument("--joins", type=int, default=4096)
    ap.add_argument("--wave-probe-rows", type=int, default=1_500_000_000)
    ap.add_argument("--block-size", type=int, default=0)
    ap.add_argument("--group-width", type=int, default=0)
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--load-factor", type=float, default=0.0)
    ap.add_argument("--no-secondary", action="store_true",
                    help="large workload: skip the small / skewed / batched / served records")
    ap.add_argument("--check-joins", type=int, default=64, help="batched: joins checked row by row against the oracle")
    ap.add_argument("--check-requests", type=int, default=16,
                    help="served: requests checked row by row against the oracle")
    return ap.parse_args()


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def profile_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None, None
    try:
        d = json.loads(p.read_text())
        e = d.get(kernel)
        return (float(e["bytes_per_launch"]), e.get("source")) if e else (None, None)
    except Exception:
        return None, None


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every ~2 ms during the timed region
    (nvidia-smi as a fallback). Reads only; changes no GPU setting."""
    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self._nvml = None
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        while not self._stop.is_set():
            if self._nvml is not None:
                try:
                    self.samples.append(float(self._nvml.nvmlDeviceGetClockInfo(self._h, self._nvml.NVML_CLOCK_SM)))
                    r = self._nvml.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                    for name, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(name)
                except Exception:
                    pass
                time.sleep(0.002)
            else:
                try:
                    out = subprocess.run(["nvidia-smi", f"--id={self.index}",
                                          "--query-gpu=clocks.sm,clocks.max.sm", "--format=csv,noheader,nounits"],
                                         capture_output=True, text=True, timeout=5).stdout.split(",")
                    self.samples.append(float(out[0]))
                    self.max_mhz = float(out[1])
                except Exception:
                    pass
                time.sleep(0.05)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


def workload_desc(nb, np_):
    return (f"large 1:1 FK equi-join: build {nb} rows unique int64 keys (seeded Feistel over 0..2^40) "
            f"+ 2 int64 payloads; probe {np_} rows int64 keys drawn from the build keys (all match) "
            f"+ 1 int64 payload; output probe rid, build rid, 3 payloads (32 B/row)")


def alg_bytes_probe_phase(inp) -> int:
    """Compulsory bytes of the probe phase: probe keys + probe payloads read once, build payloads
    read once, every output byte written once (table traffic is not counted)."""
    probe_in = inp.probe_keys.nbytes + sum(c.nbytes for c in inp.probe_payload)
    build_pay = sum(c.nbytes for c in inp.build_payload)
    out = inp.n_probe * inp.output_row_bytes()  # every probe row matches once
    return probe_in + build_pay + out


# --------------------------------------------------------------------------------------------
# CPU join (oracle) timing
# --------------------------------------------------------------------------------------------
def cpu_join_seconds(inp, threads):
    from oracle import oracle as O
    t0 = time.perf_counter()
    r = O.hash_join(inp.build_keys, inp.probe_keys, probe_payload=inp.probe_payload,
                    build_payload=inp.build_payload, threads=threads, capacity=inp.n_probe)
    dt = time.perf_counter() - t0
    assert r.rows == inp.n_probe
    return dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    from sirius_b200 import datagen as D
    O.build()
    inp = D.large(args.seed, args.n_build, args.n_probe)
    threads = O.default_threads()
    for _ in range(max(0, args.warmup)):
        cpu_join_seconds(inp, threads)
    times = [cpu_join_seconds(inp, threads) for _ in range(max(1, args.steps))]
    total = sum(times)
    value = args.n_probe * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": "join probe Mtuples/s", "value": round(value, 3), "unit": "Mtuples/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / len(times), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
        "config": {"workload": workload_desc(args.n_build, args.n_probe), "build_rows": args.n_build,
                   "probe_rows": args.n_probe},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mtuples/s", "cores": threads, "kind": "port",
                         "sample": "full workload per step: one-shot CPU hash join (build + probe + payload "
                                   "gather into host arrays) by the oracle's multithreaded C join; the "
                                   "reference (libcudf) cannot be built or run here"},
        "e2e": {"value": round(value, 3), "unit": "Mtuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------------------------
def run_sj(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    from sirius_b200 import datagen as D
    from sirius_b200 import join as J
    from sirius_b200 import multigpu as MG
    from sirius_b200 import _lib

    _lib.load()
    # every rank: the same build side; its own probe shard (seed stream offset by rank)
    inp = D.large(args.seed, args.n_build, args.n_probe)
    if rank > 0:
        # same (replicated) build side; this rank's own probe shard
        keys, pay = MG.probe_shard(inp.build_keys, args.n_probe, args.seed, rank)
        inp.probe_keys, inp.probe_payload = keys, [pay]
    bk = torch.from_numpy(inp.build_keys).to(dev)
    pk = torch.from_numpy(inp.probe_keys).to(dev)
    bp = [torch.from_numpy(c).to(dev) for c in inp.build_payload]
    pp = [torch.from_numpy(c).to(dev) for c in inp.probe_payload]
    stream = torch.cuda.current_stream()

    # ---- build (timed separately) ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_build = []
    for i in range(3):
        torch.cuda.synchronize()
        ev0.record()
        tb = J.HashTable(bk, attach=bp, partition_bits=args.partition_bits, aggregation=args.aggregation,
                         probe_kernel=args.probe_kernel, rows_per_lane=args.rows_per_lane,
                         ctas_per_sm=args.ctas_per_sm, load_factor=args.load_factor or 0.5,
                         probe_partition_mb=args.probe_partition_mb, table_l2_priority=args.table_l2)
        ev1.record()
        torch.cuda.synchronize()
        t_build.append(ev0.elapsed_time(ev1))
        if i < 2:
            tb.close()
    table = tb
    info = table.info()

    out = J.allocate_output(args.n_probe, pp, bp, dev)
    d_count = torch.zeros(1, dtype=torch.int64, device=dev)

    def step():
        table.probe_gather(pk, None, pp, attached=True, capacity=args.n_probe, out=out, d_count=d_count, sync=False)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    got = int(d_count.item())
    assert got == args.n_probe, f"probe produced {got} rows, expected {args.n_probe}"
    # correctness spot check of the timed configuration (full size, size-independent properties)
    sample = torch.randint(0, args.n_probe, (1 << 16,), device=dev)
    prid = out.probe_rid[sample].long()
    brid = out.build_rid[sample].long()
    assert torch.equal(pk[prid], bk[brid]), "joined keys differ"
    assert torch.equal(out.build_payload[0][sample], bp[0][brid])
    assert torch.equal(out.probe_payload[0][sample], pp[0][prid])

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    _lib.timing_collect()           # drop warm-up records
    _lib.timing_enable(True)        # per-kernel CUDA events inside the library, on the launch stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        # a ~2 ms spin kernel ahead of the start event, so the host has queued the first steps
        # before the timed region starts: otherwise the first step also measures the host's
        # first enqueue after the synchronize above (one step of 20 was seen at 3.1 ms vs 1.81)
        torch.cuda._sleep(4_000_000)
        t_all0.record()
        for i in range(args.steps):
            starts[i].record()
            step()
            ends[i].record()
        t_all1.record()
        torch.cuda.synchronize()
    _lib.timing_enable(False)
    kernel_times = _lib.timing_collect()
    if world > 1:
        dist.barrier()
    total_ms = t_all0.elapsed_time(t_all1)
    per_launch = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    max_ms = MG.max_over_ranks(total_ms, dev)
    value = MG.weak_scaling_value(args.n_probe, args.steps, world, max_ms)
    clocks = clk.summary()

    # ---- e2e: one-shot join through the C ABI from pinned host buffers (sj_inner_join_host) ----
    e2e = None
    if args.e2e_steps > 0:
        pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
        h_bk, h_pk = pin(inp.build_keys), pin(inp.probe_keys)
        h_bp = [pin(c) for c in inp.build_payload]
        h_pp = [pin(c) for c in inp.probe_payload]
        h_out = [torch.empty(args.n_probe, dtype=torch.int32).pin_memory() for _ in range(2)]
        h_out += [torch.empty(args.n_probe, dtype=c.dtype).pin_memory() for c in pp + bp]
        h_res = J.JoinOutput(0, h_out[0], h_out[1], h_out[2:2 + len(pp)], h_out[2 + len(pp):])
        h2d = sum(x.numel() * x.element_size() for x in [h_bk, h_pk] + h_bp + h_pp)
        d2h = sum(x.numel() * x.element_size() for x in h_out)
        e2e_counts = []

        def e2e_step():
            o = J.inner_join_host(h_bk, h_pk, None, None, h_pp, h_bp, capacity=args.n_probe, out=h_res,
                                  chunk_rows=args.e2e_chunk_rows, partition_bits=args.partition_bits,
                                  probe_kernel=args.probe_kernel, rows_per_lane=args.rows_per_lane,
                                  probe_partition_mb=args.probe_partition_mb, table_l2_priority=args.table_l2)
            e2e_counts.append(o.count)

        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record()
        for _ in range(args.e2e_steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        e_ms = e0.elapsed_time(e1)
        wall_ms = (time.perf_counter() - w0) * 1e3
        e_max = MG.max_over_ranks(max(e_ms, wall_ms), dev)
        assert all(c == args.n_probe for c in e2e_counts), e2e_counts
        # spot check of the host result: probe row i matched the build row holding its key
        sample = np.random.default_rng(7).integers(0, args.n_probe, 4096)
        hp, hb = h_out[0].numpy()[sample], h_out[1].numpy()[sample]
        assert np.array_equal(inp.probe_keys[hp], inp.build_keys[hb]), "e2e output rows do not match"
        e2e = {"value": round(args.n_probe * args.e2e_steps * world / (e_max / 1e3) / 1e6, 3),
               "unit": "Mtuples/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": round(e_max / args.e2e_steps, 3),
               "chunk_rows": args.e2e_chunk_rows or 8388608,
               "what": "one-shot join from pinned host buffers through sj_inner_join_host: H2D of all "
                       "inputs, build, chunked probe + gather, D2H of the whole output (uploads, probes "
                       "and downloads of the probe chunks overlapped)"}

    # ---- roofline of the probe phase (the sj_probe_gather call) and its kernels ----
    alg = alg_bytes_probe_phase(inp)
    launch_ms = statistics.mean(per_launch)
    peak, peak_src = measured_peak()
    achieved = alg / (launch_ms / 1e3) / 1e9
    per_kernel = {}
    for name, ms in kernel_times:
        k = per_kernel.setdefault(name, [0, 0.0])
        k[0] += 1
        k[1] += ms
    ktot = sum(v[1] for v in per_kernel.values()) or 1.0
    kernels = {n: {"launches": c, "ms_per_launch": round(t / c, 4), "share": round(t / ktot, 4)}
               for n, (c, t) in sorted(per_kernel.items(), key=lambda kv: -kv[1][1])}
    dominant = next(iter(kernels), None)
    traffic, traffic_src = profile_traffic("probe_phase")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and args.cpu_steps > 0:
        from oracle import oracle as O
        O.build()
        threads = O.default_threads()
        ts = [cpu_join_seconds(inp, threads) for _ in range(args.cpu_steps)]
        cpu = {"value": round(args.n_probe / statistics.median(ts) / 1e6, 3), "unit": "Mtuples/s",
               "cores": threads, "kind": "port",
               "sample": f"full workload, {len(ts)} one-shot CPU joins (build + probe + gather into host "
                         f"arrays), median {statistics.median(ts):.3f} s; oracle multithreaded C join"}

    if rank == 0:
        line = {
            "metric": "join probe Mtuples/s", "value": round(value, 3), "unit": "Mtuples/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(max_ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded numpy PCG64 / Feistel keys)",
            "config": {"workload": workload_desc(args.n_build, args.n_probe), "build_rows": args.n_build,
                       "probe_rows": args.n_probe, "parallelism": f"replicated build, probe sharded x{world}",
                       "l2": "no flush: every step streams 1 GiB of probe input and writes 2 GiB of output, "
                             "both larger than the 126 MB L2",
                       "start": "a ~2 ms GPU spin kernel precedes the start event, so the host's enqueue of "
                                "the first steps is not inside the timed region",
                       "table": {"layout": "DISTINCT" if info.layout == 1 else "GROUPED",
                                 "slot": "PACKED64" if info.slot_kind == 0 else "WIDE128",
                                 "slots": int(info.num_slots), "rid_bits": int(info.rid_bits),
                                 "bytes": int(info.device_bytes), "partition_bits": int(info.partition_bits),
                                 "probe_partition_mb": args.probe_partition_mb or 48, "table_l2": args.table_l2},
                       "t_build_ms": round(min(t_build), 3)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "unit_of_work": "probe phase = one sj_probe_gather call over 64M probe rows "
                                         "(partition + probe/gather kernels)",
                         "alg_bytes_per_launch": int(alg), "launch_ms": round(launch_ms, 4),
                         "launch_ms_min_median_max": [round(min(per_launch), 4),
                                                      round(statistics.median(per_launch), 4),
                                                      round(max(per_launch), 4)],
                         "dominant_kernel": dominant, "kernels": kernels, "peak_source": peak_src,
                         "frac_of_nominal_8TBs": round(achieved / NOMINAL_HBM_GBS, 4),
                         "traffic_source": traffic_src},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": len(kernel_times),
            "clocks": clocks,
        }
    table.close()
    if rank == 0 and world == 1 and not args.no_secondary:
        # the other configurations, each with its own clocks and oracle check
        del out, d_count, bk, pk, bp, pp, inp
        if args.e2e_steps > 0:
            del h_bk, h_pk, h_bp, h_pp, h_out, h_res
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["workloads"] = run_secondary(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_secondary(args):
    """Records of the small, skewed, batched and served workloads and of the rows after the INNER path
    (join kinds, two-column keys, partition operator, dynamic filter), at default sizes and seeds."""
    import copy
    import torch
    recs = {}
    for wl in ("small", "skewed", "batched", "served", "next"):
        a = copy.copy(args)
        a.workload = wl
        a.n_build = a.n_probe = None
        a.partition_bits, a.probe_partition_mb, a.table_l2 = 0, 0, 0
        a.steps = 10 if wl in ("small", "skewed") else 5
        a.autotune = wl == "batched"
        t0 = time.perf_counter()
        try:
            rec = (run_batched(a) if wl == "batched" else run_served(a) if wl == "served" else
                   run_next(a) if wl == "next" else run_other(a))
            rec["bench_seconds"] = round(time.perf_counter() - t0, 1)
        except Exception as e:  # one workload's failure is reported in its record, the line still prints
            rec = {"error": f"{type(e).__name__}: {e}"}
        recs[wl] = rec
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return recs


# --------------------------------------------------------------------------------------------
# batched workload: 4,096 independent joins in one persistent launch
# --------------------------------------------------------------------------------------------
def batched_wave_specs(sizes, first, dev, seed):
    """Joins [first, first+len(sizes)) of the batched workload, generated on the device:
    build keys = an affine permutation of 0..nb-1 (unique int32), probe = 10*nb keys uniform on
    [0, 1.2*nb), int32 payloads."""
    import torch
    from sirius_b200 import batch as B
    g = torch.Generator(device=dev)
    g.manual_seed(seed * 1_000_003 + first)
    specs = []
    for j, nb in enumerate(sizes):
        nb = int(nb)
        b = int((first + j) * 7919) % nb
        bk = ((torch.arange(nb, device=dev, dtype=torch.int64) * 1_000_003 + b) % nb).to(torch.int32)
        npr = 10 * nb
        pk = (torch.rand(npr, device=dev, generator=g) * (1.2 * nb)).to(torch.int32)
        bp = torch.randint(-2**31, 2**31 - 1, (nb,), device=dev, dtype=torch.int32, generator=g)
        pp = torch.randint(-2**31, 2**31 - 1, (npr,), device=dev, dtype=torch.int32, generator=g)
        specs.append(B.BatchJoinSpec(bk, pk, bp, pp, capacity=npr))
    return specs


def run_batched(args):
    import ctypes
    import torch
    from sirius_b200 import batch as B
    from sirius_b200 import datagen as D
    from sirius_b200 import join as J
    from sirius_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    sizes = D.batched_sizes(args.seed, args.joins)
    params = B.batch_params(block_size=args.block_size, group_width=args.group_width, tile_rows=args.tile_rows,
                            load_factor=args.load_factor)
    tuned = None
    if args.autotune:
        from sirius_b200 import autotune as A
        # 256 joins spread over the size distribution
        sample = np.sort(sizes)[np.linspace(0, len(sizes) - 1, 256).astype(int)]
        t0 = time.perf_counter()
        tuned = A.tune_batch(batched_wave_specs(sample, 0, dev, args.seed + 1), key_type="int32")
        tuned = dict(tuned, tune_seconds=round(time.perf_counter() - t0, 2))
        params = B.batch_params(**{k: v for k, v in tuned.items() if k in A.BATCH_SPACE})
        torch.cuda.empty_cache()
    # waves bounded by probe rows so inputs + outputs + tables fit in HBM
    waves, cur, acc = [], [], 0
    for i, nb in enumerate(sizes):
        if cur and acc + 10 * int(nb) > args.wave_probe_rows:
            waves.append(cur)
            cur, acc = [], 0
        cur.append(i)
        acc += 10 * int(nb)
    if cur:
        waves.append(cur)
    stream = torch.cuda.Stream()
    t_graph = t_launch = t_per_join = t_inner_each = 0.0
    probe_rows = build_rows = matches = 0
    kernels = {}
    from oracle import oracle as O
    O.build()
    check_set = set(np.random.default_rng(args.seed + 5).choice(len(sizes), min(args.check_joins, len(sizes)),
                                                                 replace=False).tolist())
    checked_joins = checked_rows = 0
    lib = _lib.load()
    with ClockSampler(0) as clk:
        for w in waves:
            specs = batched_wave_specs(sizes[w], w[0], dev, args.seed)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                plan = B.BatchPlan(specs, params, stream=stream)
                expect = torch.stack([(s.probe_key < s.build_key.numel()).sum() for s in specs])

                def timed(fn, reps):
                    for _ in range(max(3, args.warmup)):
                        fn()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    stream.synchronize()
                    e0.record(stream)
                    for _ in range(reps):
                        fn()
                    e1.record(stream)
                    e1.synchronize()
                    return e0.elapsed_time(e1) / reps

                t_graph += timed(lambda: plan.replay(stream), args.steps)
                counts, err = plan.counts(stream)
                stream.synchronize()
                assert int(err.item()) == 0 and torch.equal(counts, expect), "batched join counts differ"
                # sampled joins of the graph-replay output against the oracle, row by row
                for k, j in enumerate(w):
                    if j not in check_set:
                        continue
                    sp, c = specs[k], int(counts[k].item())
                    o = sp.out
                    got = [o.probe_rid[:c].cpu().numpy(), o.build_rid[:c].cpu().numpy(),
                           o.probe_payload[:c].cpu().numpy(), o.build_payload[:c].cpu().numpy()]
                    ref = O.hash_join(sp.build_key.cpu().numpy(), sp.probe_key.cpu().numpy(),
                                      probe_payload=[sp.probe_payload.cpu().numpy()],
                                      build_payload=[sp.build_payload.cpu().numpy()])
                    want = [ref.probe_rid, ref.build_rid, ref.probe_payload[0], ref.build_payload[0]]
                    assert ref.rows == c, f"join {j}: {c} rows, oracle {ref.rows}"
                    for g, e in zip(O.canonical(*got), O.canonical(*want)):
                        assert np.array_equal(g, e), f"join {j}: rows differ from the oracle"
                    checked_joins += 1
                    checked_rows += c
                t_launch += timed(lambda: plan.launch(stream), max(1, args.steps // 2))
                t_per_join += timed(lambda: plan.launch_per_join(stream), max(1, args.steps // 4))
                counts, err = plan.counts(stream)
                stream.synchronize()
                assert int(err.item()) == 0 and torch.equal(counts, expect), "per-join counts differ"
                # what the operator calls per join today: the one-shot sj_inner_join (build, probe,
                # gather), one call per join into the same outputs
                d_cnt = torch.zeros(len(specs), dtype=torch.int64, device=dev)
                cols = [(J.make_column(sp.build_key), J.make_column(sp.probe_key),
                         J._cols([J.make_column(sp.probe_payload)]), J._cols([J.make_column(sp.build_payload)]),
                         J._cols([J._mut(sp.out.probe_payload, None)], _lib.SjMutColumn),
                         J._cols([J._mut(sp.out.build_payload, None)], _lib.SjMutColumn)) for sp in specs]

                def inner_each():
                    for k, sp in enumerate(specs):
                        bc, pc, pin, bin_, pout, bout = cols[k]
                        _lib.check(lib.sj_inner_join(ctypes.byref(bc), ctypes.byref(pc), 1, pin, 1, bin_, 1,
                                                     sp.out.probe_rid.data_ptr(), sp.out.build_rid.data_ptr(), pout,
                                                     bout, sp.capacity, None, None, stream.cuda_stream,
                                                     d_cnt[k:k + 1].data_ptr()), "sj_inner_join")

                t_inner_each += timed(inner_each, 1)
                stream.synchronize()
                assert torch.equal(d_cnt, expect), "per-join sj_inner_join counts differ"
                probe_rows += sum(int(s.probe_key.numel()) for s in specs)
                build_rows += sum(int(s.build_key.numel()) for s in specs)
                matches += int(counts.sum().item())
                plan.close()
            del specs
            torch.cuda.empty_cache()
    line = {
        "metric": "batched join probe Mtuples/s (one persistent launch, CUDA-graph replay)",
        "value": round(probe_rows / (t_graph / 1e3) / 1e6, 3), "unit": "Mtuples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(t_graph, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (generated on the device per wave)",
        "config": {"workload": f"{args.joins} independent inner joins, build log-uniform 1K..1M unique int32 keys, "
                               f"probe 10x build uniform over 1.2x the key range, int32 payloads",
                   "joins": args.joins, "waves": len(waves), "build_rows": build_rows, "probe_rows": probe_rows,
                   "matches": matches, "params": {"block_size": params.block_size, "group_width": params.group_width,
                                                  "tile_rows": params.tile_rows,
                                                  "load_factor": round(params.load_factor, 3)},
                   "autotuned": tuned},
        "persistent_launch_ms": round(t_launch, 3), "graph_replay_ms": round(t_graph, 3),
        "one_launch_per_join_ms": round(t_per_join, 3),
        "speedup_vs_per_join": round(t_per_join / t_graph, 3),
        "sj_inner_join_per_join_ms": round(t_inner_each, 3),
        "speedup_vs_sj_inner_join_per_join": round(t_inner_each / t_graph, 3),
        "oracle_check": {"kind": "per-join match counts of every join; every output row of a seeded sample of "
                                 "joins, bit-exact after a canonical sort",
                         "joins_counted": len(sizes), "joins_checked": checked_joins, "rows_checked": checked_rows,
                         "passed": True},
        "gpu_launches": len(waves), "clocks": clk.summary(),
    }
    return line


# --------------------------------------------------------------------------------------------
# served workload: resident tables, a stream of probe requests
# --------------------------------------------------------------------------------------------
def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(q / 100 * (len(xs) - 1))))]


def run_served(args):
    """8 resident tables (unique int64 keys, 1M..48M rows, one int64 payload); requests pick a table
    uniformly and probe a log-uniform 10K..20M keys at a 70% hit rate. Each request is served by
    the join server (admission against a 120 GiB budget, `--slots` concurrent streams) and, for
    comparison, by the same server with one slot (serial one-at-a-time execution). Both see the
    same requests: all at once (saturation: throughput) and as Poisson arrivals at 0.5, 0.8 and
    0.95 x the serial capacity (latency p50/p99, submit to the request's last GPU operation)."""
    import torch
    from sirius_b200 import datagen as D
    from sirius_b200 import serve as S
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rows = D.SERVED_TABLE_ROWS
    tables = [D.served_table_device(args.seed, t, n, dev) for t, n in enumerate(rows)]
    hi = args.served_max_rows
    pools = [D.served_probe_pool(args.seed, t, k, hi) for t, (k, _) in enumerate(tables)]
    ts, sizes, starts = D.served_requests(args.seed, args.requests, len(rows), 1e4, hi)
    reqs = []
    for i in range(args.requests):
        t, m = int(ts[i]), int(sizes[i])
        off = int(starts[i] * (hi - m)) & ~1  # 16-byte aligned windows
        reqs.append((t, pools[t][off:off + m]))
    probe_rows = int(sizes.sum())
    torch.cuda.synchronize()

    def make(slots, batch):
        srv = S.JoinServer(slots=slots, memory_budget_bytes=120 << 30, reserve_bytes=args.reserve_gib << 30,
                           batch_small=batch)
        tids = [srv.add_table(k, attach=[p]) for k, p in tables]
        return srv, tids

    def run(srv, tids, arrivals, base_id, keep=None):
        """Submit every request at t0 + arrivals[i]; returns {i: (latency s, count)}, makespan s.
        keep: {request index: None} filled with host copies of those requests' output rows."""
        n = len(reqs)
        err = []

        def submitter():
            t0 = time.perf_counter()
            try:
                for i, (t, pk) in enumerate(reqs):
                    if arrivals is not None:
                        d = t0 + arrivals[i] - time.perf_counter()
                        if d > 0:
                            time.sleep(d)
                    srv.submit(tids[t], pk, base_id + i, sync=False)
            except Exception as e:  # surfaced below
                err.append(e)

        th = threading.Thread(target=submitter)
        th.start()
        got = {}
        while len(got) < n:
            if err and not th.is_alive() and not srv._inflight:
                break
            for r in srv.poll(256, wait_ms=20):
                assert r.status == 0, f"request {r.request_id} failed with status {r.status}"
                got[r.request_id - base_id] = (r.t_done - r.t_submit, r.count, r.t_submit, r.t_done)
                if keep is not None and r.request_id - base_id in keep:
                    keep[r.request_id - base_id] = (r.probe_rid.cpu().numpy(), r.build_rid.cpu().numpy(),
                                                    r.build_payload[0].cpu().numpy())
                srv.release(r.request_id)
        th.join()
        if err:
            raise err[0]
        makespan = max(v[3] for v in got.values()) - min(v[2] for v in got.values())
        return got, makespan

    results = {}
    with ClockSampler(0) as clk:
        ser, ser_t = make(1, False)  # serial one-at-a-time execution: one slot, no batching
        con, con_t = make(args.slots, True)
        # warm-up: one untimed saturated pass per server (kernels loaded, memory pools grown); the
        # concurrent server's warm-up also keeps host copies of a sample of results for the oracle
        # check (copying them inside a timed run would hold its outputs and stall its admission)
        sample = np.random.default_rng(args.seed + 9).choice(len(reqs), min(args.check_requests, len(reqs)),
                                                            replace=False)
        kept = {int(i): None for i in sample}
        run(ser, ser_t, None, 10_000_000)
        run(con, con_t, None, 20_000_000, keep=kept)
        s_sat, s_span = run(ser, ser_t, None, 0)
        c_sat, c_span = run(con, con_t, None, 100_000)
        for i in range(len(reqs)):
            assert s_sat[i][1] == c_sat[i][1], f"request {i}: serial and concurrent counts differ"
        cap = len(reqs) / s_span  # serial capacity, requests/s
        rng = np.random.default_rng(args.seed + 77)
        gaps = rng.exponential(1.0, size=len(reqs))
        for k, frac in enumerate((0.5, 0.8, 0.95)):
            arr = np.cumsum(gaps) / (frac * cap)
            arr -= arr[0]
            s_p, _ = run(ser, ser_t, arr, 200_000 + 10_000 * k)
            c_p, _ = run(con, con_t, arr, 300_000 + 10_000 * k)
            for i in range(len(reqs)):
                assert s_p[i][1] == c_p[i][1] == s_sat[i][1], f"request {i}: counts differ between runs"
            lat = lambda d: [v[0] * 1e3 for v in d.values()]
            results[frac] = {"arrival_rate_rps": round(frac * cap, 2),
                             "serial_p50_ms": round(_pct(lat(s_p), 50), 3), "serial_p99_ms": round(_pct(lat(s_p), 99), 3),
                             "served_p50_ms": round(_pct(lat(c_p), 50), 3), "served_p99_ms": round(_pct(lat(c_p), 99), 3)}
        con.close()
        # the same slots without batching the small requests: what batching adds
        nob, nob_t = make(args.slots, False)
        run(nob, nob_t, None, 30_000_000)
        n_sat, n_span = run(nob, nob_t, None, 400_000)
        arr = np.cumsum(gaps) / (0.95 * cap)
        arr -= arr[0]
        n_p, _ = run(nob, nob_t, arr, 500_000)
        for i in range(len(reqs)):
            assert n_sat[i][1] == n_p[i][1] == s_sat[i][1], f"request {i}: counts differ without batching"
        no_batch = {"makespan_s": round(n_span, 4), "value": round(probe_rows / n_span / 1e6, 3),
                    "poisson_0.95_p50_ms": round(_pct([v[0] * 1e3 for v in n_p.values()], 50), 3),
                    "poisson_0.95_p99_ms": round(_pct([v[0] * 1e3 for v in n_p.values()], 99), 3)}
        nob.close()
        ser.close()
    # sampled requests of the concurrent server's saturated warm-up pass against the oracle, row by row
    from oracle import oracle as O
    O.build()
    host_tables = {}
    checked_rows = 0
    for i, rows_out in sorted(kept.items()):
        t, pk = reqs[i]
        if t not in host_tables:
            host_tables[t] = (tables[t][0].cpu().numpy(), tables[t][1].cpu().numpy())
        tk, tp = host_tables[t]
        ref = O.hash_join(tk, pk.cpu().numpy(), build_payload=[tp])
        assert ref.rows == len(rows_out[0]), f"request {i}: {len(rows_out[0])} rows, oracle {ref.rows}"
        for g, e in zip(O.canonical(*rows_out), O.canonical(ref.probe_rid, ref.build_rid, ref.build_payload[0])):
            assert np.array_equal(g, e), f"request {i}: rows differ from the oracle"
        checked_rows += ref.rows
    del host_tables
    matches = sum(v[1] for v in s_sat.values())
    line = {
        "metric": "served join stream: probe Mtuples/s at saturation, p50/p99 request latency",
        "value": round(probe_rows / c_span / 1e6, 3), "unit": "Mtuples/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": round(c_span * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic (generated on the device)",
        "config": {"workload": "8 resident tables of unique int64 keys (1M,2M,4M,8M,16M,24M,32M,48M rows, one int64 "
                               "payload); requests pick a table uniformly, probe log-uniform 10K..20M int64 keys at a "
                               "70% hit rate; 120 GiB admission budget",
                   "requests": len(reqs), "probe_rows": probe_rows, "matches": matches, "slots": args.slots,
                   "pool_reserve_gib": args.reserve_gib},
        "serial_value": round(probe_rows / s_span / 1e6, 3),
        "throughput_speedup_vs_serial": round(s_span / c_span, 3),
        "saturated": {"serial_makespan_s": round(s_span, 4), "served_makespan_s": round(c_span, 4),
                      "serial_p50_ms": round(_pct([v[0] * 1e3 for v in s_sat.values()], 50), 3),
                      "serial_p99_ms": round(_pct([v[0] * 1e3 for v in s_sat.values()], 99), 3),
                      "served_p50_ms": round(_pct([v[0] * 1e3 for v in c_sat.values()], 50), 3),
                      "served_p99_ms": round(_pct([v[0] * 1e3 for v in c_sat.values()], 99), 3)},
        "poisson": {str(k): v for k, v in results.items()},
        "served_without_batching": no_batch,
        "small_request_rows": "< 65,536 probe rows: batched into shared launches",
        "clocks": clk.summary(),
        "oracle_check": {"kind": "match counts of every request, identical serial and concurrent, in every "
                                 "arrival pattern; every output row of a seeded sample of requests (concurrent "
                                 "server with batching), bit-exact after a canonical sort",
                         "requests_checked": len(kept), "rows_checked": checked_rows, "passed": True},
    }
    return line


# --------------------------------------------------------------------------------------------
# small (100K x 1M int32) and skewed (8M Zipf x 32M Zipf + 5% NULL, int64) workloads
# --------------------------------------------------------------------------------------------
def run_other(args):
    """Probe phase of the small or skewed join against a resident table (attached build payload),
    the same metric as the large workload; correctness spot checks use torch on the device."""
    import torch
    from sirius_b200 import datagen as D
    from sirius_b200 import join as J
    from sirius_b200 import _lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    sizes = {k: v for k, v in (("n_build", args.n_build), ("n_probe", args.n_probe)) if v}
    inp = D.small(args.seed, **sizes) if args.workload == "small" else D.skewed(args.seed, **sizes)
    bk = torch.from_numpy(inp.build_keys).to(dev)
    pk = torch.from_numpy(inp.probe_keys).to(dev)
    pv = None if inp.probe_validity is None else torch.from_numpy(inp.probe_validity.view(np.int32)).to(dev)
    bp = [torch.from_numpy(c).to(dev) for c in inp.build_payload]
    pp = [torch.from_numpy(c).to(dev) for c in inp.probe_payload]
    t_build = []
    for i in range(3):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tb = J.HashTable(bk, attach=bp, partition_bits=args.partition_bits, aggregation=args.aggregation,
                         probe_kernel=args.probe_kernel, rows_per_lane=args.rows_per_lane,
                         probe_partition_mb=args.probe_partition_mb, table_l2_priority=args.table_l2)
        e1.record()
        torch.cuda.synchronize()
        t_build.append(e0.elapsed_time(e1))
        if i < 2:
            tb.close()
    info = tb.info()
    m = int(tb.count(pk, pv).item())
    # expected output size from the key multiplicities (torch, independent of the join kernels)
    uk, cnt = torch.unique(bk, return_counts=True)
    idx = torch.searchsorted(uk, pk).clamp(max=uk.numel() - 1)
    mult = torch.where(uk[idx] == pk, cnt[idx], torch.zeros_like(cnt[idx]))
    if pv is not None:
        valid = ((pv.view(torch.int32).long().repeat_interleave(32)[: pk.numel()] >>
                  (torch.arange(pk.numel(), device=dev) % 32)) & 1).bool()
        mult = torch.where(valid, mult, torch.zeros_like(mult))
    assert m == int(mult.sum().item()), "match count differs from the key multiplicities"
    out = J.allocate_output(m, pp, bp, dev)
    d_count = torch.zeros(1, dtype=torch.int64, device=dev)
    # the C ABI call with its arguments built once: a step of 1M rows takes tens of microseconds, so
    # rebuilding the ctypes arguments every call (the Python wrapper) would be timed instead
    lib = _lib.load()
    kcols, nkeys, _ = J._keys(pk, pv)
    pin = J._cols([J.make_column(*J._as_pair(c)) for c in pp])
    pout = J._cols([J._mut(t, v) for t, v in zip(out.probe_payload, out.probe_payload_validity)], _lib.SjMutColumn)
    bout = J._cols([J._mut(t, v) for t, v in zip(out.build_payload, out.build_payload_validity)], _lib.SjMutColumn)
    sh = torch.cuda.current_stream().cuda_stream

    def step():
        _lib.check(lib.sj_probe_gather(tb.handle, kcols, nkeys, pin, len(pp), None, len(bp), out.probe_rid.data_ptr(),
                                       out.build_rid.data_ptr(), pout, bout, m, None, sh, d_count.data_ptr()),
                   "sj_probe_gather")

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    assert int(d_count.item()) == m
    sample = torch.randint(0, m, (1 << 16,), device=dev)
    assert torch.equal(pk[out.probe_rid[sample].long()], bk[out.build_rid[sample].long()]), "joined keys differ"
    _lib.timing_collect()
    _lib.timing_enable(True)
    with ClockSampler(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda._sleep(4_000_000)  # the host queues the first steps before the start event
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    _lib.timing_enable(False)
    kt = _lib.timing_collect()
    ms = e0.elapsed_time(e1) / args.steps
    alg = (inp.probe_keys.nbytes + (0 if inp.probe_validity is None else inp.probe_validity.nbytes) +
           sum(c.nbytes for c in inp.probe_payload) + sum(c.nbytes for c in inp.build_payload) +
           m * inp.output_row_bytes())
    peak, peak_src = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    traffic, traffic_src = profile_traffic("skewed_probe_phase") if args.workload == "skewed" else (None, None)
    per_kernel = {}
    for name, kms in kt:
        k = per_kernel.setdefault(name, [0, 0.0])
        k[0] += 1
        k[1] += kms
    ktot = sum(v[1] for v in per_kernel.values()) or 1.0
    kernels = {n: {"launches": c, "ms_per_launch": round(t / c, 4), "share": round(t / ktot, 4)}
               for n, (c, t) in sorted(per_kernel.items(), key=lambda kv: -kv[1][1])}
    from oracle import oracle as O
    O.build()
    threads = O.default_threads()
    cpu, ref = None, None
    if not args.no_cpu and args.cpu_steps > 0:
        ts = []
        for _ in range(args.cpu_steps):
            t0 = time.perf_counter()
            ref = O.hash_join(inp.build_keys, inp.probe_keys, None, inp.probe_validity, probe_payload=inp.probe_payload,
                              build_payload=inp.build_payload, threads=threads, capacity=m)
            ts.append(time.perf_counter() - t0)
            assert ref.rows == m
        cpu = {"value": round(inp.n_probe / statistics.median(ts) / 1e6, 3), "unit": "Mtuples/s", "cores": threads,
               "kind": "port", "sample": f"full workload, {len(ts)} one-shot CPU joins, median {statistics.median(ts):.3f} s"}
    # the timed output against the oracle: every row (small) or the multiset checksum of every row
    if ref is None:
        ref = O.hash_join(inp.build_keys, inp.probe_keys, None, inp.probe_validity, probe_payload=inp.probe_payload,
                          build_payload=inp.build_payload, threads=threads, capacity=m)
    got = [out.probe_rid[:m].cpu().numpy(), out.build_rid[:m].cpu().numpy()] + \
        [c[:m].cpu().numpy() for c in out.probe_payload] + [c[:m].cpu().numpy() for c in out.build_payload]
    want = [ref.probe_rid, ref.build_rid] + list(ref.probe_payload) + list(ref.build_payload)
    if args.workload == "small":
        for g, e in zip(O.canonical(*got), O.canonical(*want)):
            assert np.array_equal(g, e), "small: output rows differ from the oracle"
        check = {"kind": "every output row, bit-exact after a canonical sort", "rows": m, "passed": True}
    else:
        assert O.multiset_checksum(*got) == O.multiset_checksum(*want), "skewed: output checksum differs"
        check = {"kind": "64-bit order-independent checksum of every output row (probe rid, build rid, payloads)",
                 "rows": m, "passed": True}
    del got, want, ref
    desc = (f"small: build {inp.n_build} unique int32 keys (permutation) + int32 payload; probe {inp.n_probe} "
            f"int32 keys uniform over 1.1x the build range + int32 payload" if args.workload == "small" else
            f"skewed: build {inp.n_build} int64 keys Zipf(1.1) over 1M values + int32 payload; probe {inp.n_probe} "
            f"int64 keys Zipf(0.8) over 2M values (half absent), 5% NULL")
    line = {
        "metric": "join probe Mtuples/s", "value": round(inp.n_probe / (ms / 1e3) / 1e6, 3), "unit": "Mtuples/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32" if args.workload == "small" else "int64", "data": "synthetic (seeded numpy)",
        "config": {"workload": desc, "build_rows": inp.n_build, "probe_rows": inp.n_probe, "matches": m,
                   "table": {"layout": "DISTINCT" if info.layout == 1 else "GROUPED",
                             "slot": "PACKED64" if info.slot_kind == 0 else "WIDE128",
                             "partition_bits": int(info.partition_bits), "max_group": int(info.max_group)},
                   "t_build_ms": round(min(t_build), 3)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                     "alg_bytes_per_launch": int(alg), "launch_ms": round(ms, 4), "kernels": kernels,
                     "peak_source": peak_src},
        "cpu_baseline": cpu, "gpu_launches": len(kt), "clocks": clk.summary(),
        "oracle_check": check,
    }
    return line


# --------------------------------------------------------------------------------------------
# the rows after the INNER path: join kinds, two-column keys, the partition operator, the filter
# --------------------------------------------------------------------------------------------
def run_next(args):
    """LEFT / SEMI / ANTI / MARK on the large table with 30 % of the probe keys absent, a two-column
    int32 key, the hash partition operator and the dynamic filter, each timed on the device (CUDA
    events, inputs resident, a short spin kernel ahead of each timed region) and checked against
    an independent rule in the same run."""
    import ctypes
    import torch
    from sirius_b200 import datagen as D
    from sirius_b200 import join as J
    from sirius_b200 import _lib as L
    from oracle import oracle as O
    lib = L.load()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    peak, peak_src = measured_peak()
    steps = max(3, args.steps)

    last_kernels = {}

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        L.timing_collect()
        L.timing_enable(True)
        torch.cuda._sleep(4_000_000)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        L.timing_enable(False)
        per = {}
        for name, kms in L.timing_collect():
            per[name] = per.get(name, 0.0) + kms
        last_kernels.clear()
        last_kernels.update({k: round(v / steps, 4) for k, v in sorted(per.items(), key=lambda kv: -kv[1])})
        return e0.elapsed_time(e1) / steps

    def rec(rows, ms, alg, check, **extra):
        a = alg / (ms / 1e3) / 1e9
        return dict({"ms": round(ms, 4), "Mrows_per_s": round(rows / (ms / 1e3) / 1e6, 1),
                     "alg_bytes": int(alg), "achieved_GBps": round(a, 1), "frac_of_peak": round(a / peak, 4),
                     "kernels_ms": dict(last_kernels), "oracle_check": check}, **extra)

    out = {"peak": peak, "peak_source": peak_src, "steps": steps}
    with ClockSampler(0) as clk:
        # ---- 1. join kinds on the large table ----
        nb, n = 16 << 20, 64 << 20
        inp = D.large(args.seed, nb, n)
        bk = torch.from_numpy(inp.build_keys).to(dev)
        bp = [torch.from_numpy(c).to(dev) for c in inp.build_payload]
        pk0 = torch.from_numpy(inp.probe_keys).to(dev)
        pp = torch.from_numpy(inp.probe_payload[0]).to(dev)
        g = torch.Generator(device=dev)
        g.manual_seed(args.seed + 9)
        miss = torch.rand(n, device=dev, generator=g) < 0.3
        pk = torch.where(miss, pk0 + (1 << 41), pk0)  # build keys are < 2^40: these are absent
        del pk0
        hits = int((~miss).sum().item())
        misses = n - hits
        table = J.HashTable(bk, attach=bp)
        kcols, nkeys, _ = J._keys(pk)
        pin = J._cols([J.make_column(pp)])
        dc = torch.zeros(1, dtype=torch.int64, device=dev)
        cap_full = n + nb  # FULL: every probe row, plus at most every build row
        words = (cap_full + 31) // 32
        o_prid = torch.empty(cap_full, dtype=torch.int32, device=dev)
        o_brid = torch.empty(cap_full, dtype=torch.int32, device=dev)
        o_pp = torch.empty(cap_full, dtype=torch.int64, device=dev)
        o_pv = torch.empty(words, dtype=torch.int32, device=dev)
        o_bp = [torch.empty(cap_full, dtype=torch.int64, device=dev) for _ in bp]
        o_bv = [torch.empty(words, dtype=torch.int32, device=dev) for _ in bp]
        o_mark = torch.empty(n, dtype=torch.uint8, device=dev)
        o_markv = torch.empty(words, dtype=torch.int32, device=dev)
        pout = J._cols([J._mut(o_pp, None)], L.SjMutColumn)
        pout_full = J._cols([J._mut(o_pp, o_pv)], L.SjMutColumn)
        bin_full = J._cols([J.make_column(c) for c in bp])  # FULL gathers from the caller's columns
        bout_left = J._cols([J._mut(t, v) for t, v in zip(o_bp, o_bv)], L.SjMutColumn)
        bout_inner = J._cols([J._mut(t, None) for t in o_bp], L.SjMutColumn)

        def kind(k):
            def f():
                if k == L.SJ_JOIN_INNER:
                    L.check(lib.sj_probe_gather(table.handle, kcols, nkeys, pin, 1, None, len(bp), o_prid.data_ptr(),
                                                o_brid.data_ptr(), pout, bout_inner, n, None, sh, dc.data_ptr()),
                            "sj_probe_gather")
                    return
                full = k == L.SJ_JOIN_FULL
                left, mark = k == L.SJ_JOIN_LEFT or full, k == L.SJ_JOIN_MARK
                L.check(lib.sj_probe_join(table.handle, k, kcols, nkeys, None if mark else pin, 0 if mark else 1,
                                          bin_full if full else None, len(bp) if left else 0,
                                          None if mark else o_prid.data_ptr(),
                                          o_brid.data_ptr() if left else None,
                                          None if mark else pout_full if full else pout,
                                          bout_left if left else None, 0 if mark else cap_full if full else n,
                                          o_mark.data_ptr() if mark else None, o_markv.data_ptr() if mark else None,
                                          None, sh, dc.data_ptr()), "sj_probe_join")
            return f

        sample = torch.randint(0, n, (1 << 20,), device=dev, generator=g)
        kinds = {}
        key_in = 8 * n
        # INNER
        ms = timed(kind(L.SJ_JOIN_INNER))
        c = int(dc.item())
        s = sample[sample < c]
        ok = c == hits and torch.equal(pk[o_prid[s].long()], bk[o_brid[s].long()])
        assert ok, "inner: count or joined keys differ"
        kinds["inner"] = rec(n, ms, key_in + 8 * hits + 32 * hits + 16 * nb,
                             {"kind": "count = probe rows whose key is in the build; sampled rows join equal keys",
                              "rows": c, "passed": True})
        # LEFT
        ms = timed(kind(L.SJ_JOIN_LEFT))
        c = int(dc.item())
        nr = o_brid[:c] == L.SJ_NO_ROW
        s = sample[sample < c]
        sb = o_brid[s]
        ok = (c == n and int(nr.sum().item()) == misses and torch.equal(miss[o_prid[:c].long()], nr)
              and torch.equal(pk[o_prid[s].long()][sb != L.SJ_NO_ROW], bk[sb[sb != L.SJ_NO_ROW].long()]))
        assert ok, "left: rows differ"
        kinds["left"] = rec(n, ms, key_in + 8 * n + n * 32 + 2 * n // 8 + 16 * nb,
                            {"kind": "every probe row once; no build row exactly for the absent keys; sampled "
                                     "matched rows join equal keys", "rows": c, "passed": True})
        # SEMI
        ms = timed(kind(L.SJ_JOIN_SEMI))
        c = int(dc.item())
        ok = c == hits and not bool(miss[o_prid[:c].long()].any())
        assert ok, "semi: rows differ"
        kinds["semi"] = rec(n, ms, key_in + (8 + 12) * hits,
                            {"kind": "exactly the probe rows whose key is in the build", "rows": c, "passed": True})
        # ANTI
        ms = timed(kind(L.SJ_JOIN_ANTI))
        c = int(dc.item())
        ok = c == misses and bool(miss[o_prid[:c].long()].all())
        assert ok, "anti: rows differ"
        kinds["anti"] = rec(n, ms, key_in + (8 + 12) * misses,
                            {"kind": "exactly the probe rows whose key is absent", "rows": c, "passed": True})
        # MARK
        ms = timed(kind(L.SJ_JOIN_MARK))
        ok = torch.equal(o_mark.bool(), ~miss)
        assert ok, "mark: marks differ"
        kinds["mark"] = rec(n, ms, key_in + n + n // 8,
                            {"kind": "mark byte of every probe row equals key-in-build", "rows": n, "passed": True})
        # FULL
        ms = timed(kind(L.SJ_JOIN_FULL))
        c = int(dc.item())
        hit_keys = torch.unique(pk[~miss])
        unmatched_build = int((~torch.isin(bk, hit_keys)).sum().item())
        del hit_keys
        ok = c == n + unmatched_build
        ok = ok and int((o_prid[:c] == L.SJ_NO_ROW).sum().item()) == unmatched_build
        ok = ok and int((o_brid[:c] == L.SJ_NO_ROW).sum().item()) == misses
        assert ok, "full: rows differ"
        kinds["full"] = rec(n, ms, key_in + 8 * n + c * 32 + 3 * c // 8 + 16 * nb,
                            {"kind": "probe rows + build rows no probe row matched; padded rows are exactly the "
                                     "absent probe keys and the unmatched build keys", "rows": c,
                             "unmatched_build_rows": unmatched_build, "passed": True})
        out["join_kinds"] = {"workload": f"build {nb} unique int64 keys + 2 int64 payloads (attached, partitioned "
                                         f"table); probe {n} int64 keys, 30 % absent from the build, + 1 int64 "
                                         f"payload", "probe_rows": n, "hits": hits, **kinds}
        # ---- 4. the dynamic filter: filled by the insert pass, tested against the probe keys ----
        t_plain, t_bloom = [], []
        bt = None
        for _ in range(3):
            for bits, acc in ((0, t_plain), (16, t_bloom)):
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                tb = J.HashTable(bk, attach=bp, bloom_bits_per_key=bits)
                e1.record()
                torch.cuda.synchronize()
                acc.append(e0.elapsed_time(e1))
                if bits:
                    if bt is not None:
                        bt.close()
                    bt = tb
                else:
                    tb.close()
        bloom = bt.bloom()
        mask = torch.empty(n, dtype=torch.uint8, device=dev)
        pcol = J.make_column(pk)

        def contains():
            L.check(lib.sj_bloom_contains(bloom._h, ctypes.byref(pcol), mask.data_ptr(), None, sh), "sj_bloom_contains")

        ms = timed(contains)
        fneg = int((~mask.bool() & ~miss).sum().item())
        fpr = float(mask[miss].float().mean().item())
        assert fneg == 0 and fpr < 0.01, f"filter: {fneg} false negatives, false-positive rate {fpr}"
        out["dynamic_filter"] = {
            "workload": f"filter of {nb} build keys at 16 bits per key, filled by the table's insert pass; "
                        f"tested against the {n} probe keys above",
            "build_ms_without": round(min(t_plain), 3), "build_ms_with_filter": round(min(t_bloom), 3),
            "filter_bytes": bloom.nbytes,
            "contains": rec(n, ms, 8 * n + n + bloom.nbytes,
                            {"kind": "no false negatives over every present key; false-positive rate over the "
                                     "absent keys", "false_positive_rate": round(fpr, 6), "passed": True})}
        bt.close()
        table.close()
        del o_bp, o_bv, o_pp, o_pv, o_brid, o_prid, o_mark, mask
        torch.cuda.empty_cache()
        # ---- 3. the partition operator on the probe side ----
        P = 64
        kpart = J._keys(pk)[0]
        ins = J._cols([J.make_column(pk), J.make_column(pp)])
        p_keys = torch.empty(n, dtype=torch.int64, device=dev)
        p_pay = torch.empty(n, dtype=torch.int64, device=dev)
        p_outs = J._cols([J._mut(p_keys, None), J._mut(p_pay, None)], L.SjMutColumn)
        offs = torch.empty(P + 1, dtype=torch.int64, device=dev)

        def part():
            L.check(lib.sj_hash_partition(kpart, 1, ins, 2, P, p_outs, offs.data_ptr(), None, sh), "sj_hash_partition")

        ms = timed(part)
        off = offs.cpu().numpy()
        ok = off[0] == 0 and off[-1] == n and bool(np.all(np.diff(off) >= 0))
        ok = ok and int(p_keys.sum().item()) == int(pk.sum().item())  # the same multiset of keys (sum)
        pos = np.sort(np.random.default_rng(args.seed).choice(n, 1 << 20, replace=False))
        kk = p_keys[torch.from_numpy(pos).to(dev)].cpu().numpy()
        want = O.partition_ids([kk], [None], P)
        got = np.searchsorted(off, pos, side="right") - 1
        ok = ok and bool(np.array_equal(want, got))
        assert ok, "partition: rows in the wrong partition"
        out["partition_operator"] = {
            "workload": f"{n} int64 keys + 1 int64 payload (the probe side above) into {P} partitions",
            **rec(n, ms, 32 * n + 8 * (P + 1),
                  {"kind": "offsets cover every row; the key multiset is kept (sum); 2^20 sampled rows lie in "
                           "the partition the oracle's partition rule gives them", "rows": n, "passed": True})}
        del p_keys, p_pay, pk, pp, miss
        torch.cuda.empty_cache()
        # ---- 2. two int32 key columns ----
        nb2, n2 = 8 << 20, 32 << 20
        r = np.random.default_rng(args.seed + 11)
        codes = r.permutation(1 << 24)[:nb2]
        k1, k2 = (codes >> 11).astype(np.int32), (codes & 2047).astype(np.int32)
        idx = r.integers(0, nb2, n2)
        b1, b2 = torch.from_numpy(k1).to(dev), torch.from_numpy(k2).to(dev)
        q1, q2 = torch.from_numpy(k1[idx]).to(dev), torch.from_numpy(k2[idx]).to(dev)
        t2 = J.HashTable([b1, b2])
        mk, mn, _ = J._keys([q1, q2])
        m_prid = torch.empty(n2, dtype=torch.int32, device=dev)
        m_brid = torch.empty(n2, dtype=torch.int32, device=dev)

        def multikey():
            L.check(lib.sj_probe_gather(t2.handle, mk, mn, None, 0, None, 0, m_prid.data_ptr(), m_brid.data_ptr(),
                                        None, None, n2, None, sh, dc.data_ptr()), "sj_probe_gather")

        ms = timed(multikey)
        c = int(dc.item())
        s = torch.randint(0, n2, (1 << 20,), device=dev)
        pr, br = m_prid[s].long(), m_brid[s].long()
        ok = c == n2 and torch.equal(q1[pr], b1[br]) and torch.equal(q2[pr], b2[br])
        assert ok, "two-column keys: rows differ"
        out["multi_column_keys"] = {
            "workload": f"build {nb2} unique (int32, int32) keys; probe {n2} rows drawn from them",
            **rec(n2, ms, 8 * n2 + 8 * c,
                  {"kind": "every probe row matches once; 2^20 sampled rows join equal key pairs", "rows": c,
                   "passed": True})}
        t2.close()
    out["clocks"] = clk.summary()
    return out

def main():
    args = parse()
    if args.workload == "large" or args.impl == "reference":
        args.n_build = args.n_build or 16 << 20
        args.n_probe = args.n_probe or 64 << 20
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("batched", "served", "small", "skewed", "next"):
        runner = {"batched": run_batched, "served": run_served, "next": run_next}.get(args.workload, run_other)
        print(json.dumps(runner(args)), flush=True)
        return 0
    return run_sj(args)


if __name__ == "__main__":
    sys.exit(main())
