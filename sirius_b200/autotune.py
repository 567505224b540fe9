"""Autotuner for the join's launch parameters.

Two searches, both coordinate descent (start from the defaults, sweep one knob at a time keeping
the best value, repeat while anything improves), each candidate timed with CUDA events on a
sample of the real workload after warm-up:

* batched launches: block size, probe group width, load factor, rows per work item
  (``sj_batch_params``), on a sample of the batch's joins;
* single joins: radix partition bits ("partition fan-out"), output reservation (per warp or per
  CTA), probe CTAs per SM and load factor (``sj_join_params``), on the table and a probe sample.

Results are cached per (GPU name, SM count, search, key type, size class) in a JSON file
(``$SJ_AUTOTUNE_CACHE`` or ``~/.cache/sirius_b200/autotune.json``) so a size class is tuned once
per GPU model.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path
from typing import Callable, Dict, List, Optional

from . import _lib as L

BATCH_SPACE = {
    "block_size": [128, 256, 512],
    "group_width": [1, 2, 4, 8],
    "load_factor": [0.35, 0.5, 0.7],
    "tile_rows": [1024, 4096, 16384],
}
BATCH_DEFAULT = {"block_size": 256, "group_width": 1, "load_factor": 0.5, "tile_rows": 4096}

JOIN_SPACE = {
    "partition_bits": [-1, 0, 3, 4, 5, 6, 7],
    "aggregation": [L.SJ_AGG_WARP, L.SJ_AGG_CTA],
    "ctas_per_sm": [2, 3, 4, 6, 8],
    "load_factor": [0.35, 0.5, 0.7],
}
JOIN_DEFAULT = {"partition_bits": 0, "aggregation": L.SJ_AGG_AUTO, "ctas_per_sm": 4, "load_factor": 0.5}


def cache_path() -> Path:
    p = os.environ.get("SJ_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "sirius_b200" / "autotune.json"


def _load_cache() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store_cache(c: dict):
    p = cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass


def size_class(rows: int) -> int:
    """log2 bucket of a row count (tables of similar size tune alike)."""
    return int(math.log2(max(rows, 1)))


def gpu_key(device=None) -> str:
    import torch
    d = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    props = torch.cuda.get_device_properties(d)
    return f"{props.name}|sm{props.multi_processor_count}"


def coordinate_descent(space: Dict[str, list], start: Dict, measure: Callable[[Dict], float],
                       rounds: int = 2, log: Optional[List] = None) -> Dict:
    """Minimise measure(config) one knob at a time; returns the best config (with its time in
    ``_ms``). A candidate must beat the incumbent by 2% to count (timer noise)."""
    best = dict(start)
    best_t = measure(best)
    if log is not None:
        log.append((dict(best), best_t))
    for _ in range(rounds):
        improved = False
        for knob, values in space.items():
            for v in values:
                if v == best.get(knob):
                    continue
                cand = dict(best, **{knob: v})
                t = measure(cand)
                if log is not None:
                    log.append((dict(cand), t))
                if t < best_t * 0.98:
                    best, best_t, improved = cand, t, True
        if not improved:
            break
    best["_ms"] = best_t
    return best


def _time(fn: Callable[[], None], stream, reps: int = 5, warmup: int = 2) -> float:
    import torch
    for _ in range(warmup):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _public(cfg: Dict) -> Dict:
    return {k: v for k, v in cfg.items() if not k.startswith("_")}


def tune_batch(specs, *, key_type: str = "int32", use_cache: bool = True, rounds: int = 2,
               log: Optional[List] = None) -> Dict:
    """Best sj_batch_params (as a dict) for a batch; `specs` is a representative sample of
    batch.BatchJoinSpec."""
    import torch
    from . import batch as B
    total = sum(int(s.build_key.numel()) for s in specs)
    key = f"{gpu_key()}|batch|{key_type}|{size_class(total // max(1, len(specs)))}"
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    stream = torch.cuda.Stream()

    def measure(cfg):
        with torch.cuda.stream(stream):
            plan = B.BatchPlan(specs, B.batch_params(**_public(cfg)), stream=stream)
            try:
                return _time(lambda: plan.launch(stream), stream)
            finally:
                plan.close(stream)

    best = coordinate_descent(BATCH_SPACE, BATCH_DEFAULT, measure, rounds, log)
    if use_cache:
        cache[key] = best
        _store_cache(cache)
    return best


def tune_join(build_keys, probe_keys, attach=(), probe_payload=(), *, use_cache: bool = True, rounds: int = 1,
              log: Optional[List] = None) -> Dict:
    """Best single-join parameters for a build table and a probe sample (INNER, attached payloads)."""
    import torch
    from . import join as J
    key = f"{gpu_key()}|join|{str(build_keys.dtype)}|{size_class(build_keys.numel())}|{len(attach)}"
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return cache[key]
    stream = torch.cuda.Stream()
    n = probe_keys.numel()
    d = torch.zeros(1, dtype=torch.int64, device=probe_keys.device)

    def measure(cfg):
        with torch.cuda.stream(stream):
            t = J.HashTable(build_keys, attach=attach, stream=stream, **_public(cfg))
            try:
                out = J.allocate_output(n, probe_payload, attach, probe_keys.device)
                return _time(lambda: t.probe_gather(probe_keys, None, probe_payload, attached=bool(attach),
                                                    capacity=n, out=out, d_count=d, stream=stream, sync=False),
                             stream)
            finally:
                t.close(stream)

    best = coordinate_descent(JOIN_SPACE, JOIN_DEFAULT, measure, rounds, log)
    if use_cache:
        cache[key] = best
        _store_cache(cache)
    return best
