"""Seeded synthetic inputs for the join workloads (numpy PCG64; identical on every machine).

The reference ships no dataset for this path; these generators produce the shapes, sizes and
value distributions of the five workloads the join is measured on:

* ``small``    100k build rows (int32 key = permutation of 0..99,999, int32 payload) x 1M probe
               rows (int32 key uniform on 0..109,999 -> ~9% misses, int32 payload);
* ``large``    16M build rows (unique int64 keys, a seeded 40-bit Feistel permutation of a sparse
               range 0..2^40, two int64 payloads) x 64M probe rows (keys drawn uniformly from the
               build keys, every probe matches once, one int64 payload);
* ``skewed``   8M build rows with Zipf(1.1) keys over 1M values (int32 payload) x 32M probe rows
               with Zipf(0.8) keys over 2M values, half of them absent from the build, 5% NULL
               keys via a validity bitmask;
* ``batched``  4,096 joins, build sizes log-uniform 1K..1M of unique int32 keys, probe = 10x
               build with keys uniform over 1.2x the build key range, int32 payloads;
* ``served``   8 resident tables of unique full-range int64 keys (1, 2, 4, 8, 16, 24, 32, 48 M
               rows, one int64 payload) and probe requests of log-uniform 10K..20M keys with a 70%
               hit rate.

Every function takes a seed and optional size overrides so tests can run scaled-down copies.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLD = np.uint64(0x9E3779B97F4A7C15)


def mix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer, vectorised (a bijection on uint64)."""
    x = np.asarray(x, np.uint64)
    with np.errstate(over="ignore"):
        x = x ^ (x >> np.uint64(30))
        x = x * _M1
        x = x ^ (x >> np.uint64(27))
        x = x * _M2
        return x ^ (x >> np.uint64(31))


def feistel40(idx: np.ndarray, seed: int, rounds: int = 4) -> np.ndarray:
    """Seeded bijection on [0, 2^40) (balanced 20/20-bit Feistel network); idx -> int64 keys."""
    x = np.asarray(idx, np.uint64)
    mask = np.uint64((1 << 20) - 1)
    left = x >> np.uint64(20)
    right = x & mask
    with np.errstate(over="ignore"):
        for r in range(rounds):
            k = mix64(np.uint64(seed) * _GOLD + np.uint64(r + 1))
            f = mix64(right ^ k) & mask
            left, right = right, left ^ f
    return ((left << np.uint64(20)) | right).astype(np.int64)


def pack_validity(valid: np.ndarray) -> np.ndarray:
    valid = np.asarray(valid, bool)
    n = len(valid)
    padded = np.zeros(((n + 31) // 32) * 32, bool)
    padded[:n] = valid
    return np.packbits(padded, bitorder="little").view(np.uint32).copy()


def _rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, stream])))


def _u(rng, n, dtype):
    info = np.iinfo(dtype)
    return rng.integers(info.min, info.max, size=n, dtype=dtype, endpoint=True)


@dataclass
class JoinInput:
    """One join: build side (keys + payloads) and probe side (keys + payloads), host arrays."""
    name: str
    build_keys: np.ndarray
    probe_keys: np.ndarray
    build_payload: list = field(default_factory=list)
    probe_payload: list = field(default_factory=list)
    build_validity: Optional[np.ndarray] = None  # uint32 bitmask words
    probe_validity: Optional[np.ndarray] = None
    expected_rows: Optional[int] = None  # exact output rows when known by construction

    @property
    def n_build(self) -> int:
        return len(self.build_keys)

    @property
    def n_probe(self) -> int:
        return len(self.probe_keys)

    def input_bytes(self) -> int:
        b = self.build_keys.nbytes + self.probe_keys.nbytes
        b += sum(c.nbytes for c in self.build_payload) + sum(c.nbytes for c in self.probe_payload)
        for v in (self.build_validity, self.probe_validity):
            if v is not None:
                b += v.nbytes
        return b

    def output_row_bytes(self) -> int:
        """Bytes of one output row: probe rid, build rid and the gathered payloads."""
        return 8 + sum(c.itemsize for c in self.probe_payload) + sum(c.itemsize for c in self.build_payload)


def small(seed: int = 1, n_build: int = 100_000, n_probe: int = 1_000_000) -> JoinInput:
    r = _rng(seed, 1)
    bk = r.permutation(n_build).astype(np.int32)
    pk = r.integers(0, int(n_build * 1.1), size=n_probe, dtype=np.int32)
    return JoinInput("small", bk, pk, [_u(r, n_build, np.int32)], [_u(r, n_probe, np.int32)])


def large(seed: int = 1, n_build: int = 16 << 20, n_probe: int = 64 << 20) -> JoinInput:
    r = _rng(seed, 2)
    bk = feistel40(np.arange(n_build, dtype=np.uint64), seed)
    idx = r.integers(0, n_build, size=n_probe, dtype=np.int64)
    pk = bk[idx]
    return JoinInput("large", bk, pk, [_u(r, n_build, np.int64), _u(r, n_build, np.int64)],
                     [_u(r, n_probe, np.int64)], expected_rows=n_probe)


def _zipf_ranks(r: np.random.Generator, n: int, domain: int, s: float) -> np.ndarray:
    """n ranks in [0, domain) with P(rank k) proportional to (k+1)^-s (inverse CDF)."""
    w = np.arange(1, domain + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    u = r.random(n) * cdf[-1]
    return np.minimum(np.searchsorted(cdf, u, side="right"), domain - 1)


def skewed(seed: int = 1, n_build: int = 8 << 20, n_probe: int = 32 << 20, build_values: int = 1 << 20,
           probe_values: int = 2 << 20, s_build: float = 1.1, s_probe: float = 0.8,
           null_frac: float = 0.05) -> JoinInput:
    r = _rng(seed, 3)
    n_absent = probe_values - probe_values // 2
    values = feistel40(np.arange(build_values + n_absent, dtype=np.uint64), seed + 7)
    # values[:build_values] is the build domain; the probe maps half of its ranks onto it and the
    # other half onto values[build_values:] (absent from the build).
    perm_b = r.permutation(build_values)
    bk = values[perm_b[_zipf_ranks(r, n_build, build_values, s_build)]]
    present = r.permutation(build_values)[: probe_values // 2]
    absent = build_values + r.permutation(n_absent)
    pmap = r.permutation(np.concatenate([present, absent]))
    pk = values[pmap[_zipf_ranks(r, n_probe, probe_values, s_probe)]]
    pvalid = r.random(n_probe) >= null_frac
    return JoinInput("skewed", bk, pk, [_u(r, n_build, np.int32)], [], None, pack_validity(pvalid))


def batched_sizes(seed: int = 1, n_joins: int = 4096, lo: float = 1e3, hi: float = 1e6) -> np.ndarray:
    r = _rng(seed, 4)
    return np.floor(np.exp(r.uniform(np.log(lo), np.log(hi), size=n_joins))).astype(np.int64)


def batched_join(seed: int, j: int, n_build: int, probe_factor: int = 10) -> JoinInput:
    r = _rng(seed, 1000 + j)
    bk = r.permutation(n_build).astype(np.int32)
    pk = r.integers(0, int(1.2 * n_build), size=probe_factor * n_build, dtype=np.int32)
    return JoinInput(f"batched[{j}]", bk, pk, [_u(r, n_build, np.int32)], [_u(r, len(pk), np.int32)])


SERVED_TABLE_ROWS = [1 << 20, 2 << 20, 4 << 20, 8 << 20, 16 << 20, 24 << 20, 32 << 20, 48 << 20]


def served_table(seed: int, t: int, n_rows: int):
    """Resident table t: unique full-range int64 keys (mix64 of a disjoint index range), payload."""
    base = np.uint64((t + 1) << 40)
    keys = mix64(np.arange(n_rows, dtype=np.uint64) + base + np.uint64(seed) * np.uint64(1 << 56)).view(np.int64)
    payload = _u(_rng(seed, 5000 + t), n_rows, np.int64)
    return keys, payload


def served_request(seed: int, i: int, table_keys: np.ndarray, t: int, n_probe: int, hit_rate: float = 0.7):
    """Probe keys: hit_rate of them drawn from the table, the rest absent (outside its index range)."""
    r = _rng(seed, 100000 + i)
    n_hit = int(round(n_probe * hit_rate))
    hits = table_keys[r.integers(0, len(table_keys), size=n_hit)]
    base = np.uint64((t + 1) << 40) + np.uint64(seed) * np.uint64(1 << 56)
    miss_idx = np.uint64(len(table_keys)) + r.integers(0, 1 << 30, size=n_probe - n_hit, dtype=np.uint64)
    misses = mix64(miss_idx + base).view(np.int64)
    keys = np.concatenate([hits, misses])
    r.shuffle(keys)
    return keys, n_hit


# ---- the served workload generated on the device (same key functions as above) ----

def _srl(x, s: int):
    """Logical right shift of int64 tensor bits."""
    return (x >> s) & ((1 << (64 - s)) - 1)


def mix64_torch(x):
    """mix64 on an int64 torch tensor (bit pattern as uint64; multiplication wraps)."""
    m1 = int(_M1) - (1 << 64)
    m2 = int(_M2) - (1 << 64)
    x = x ^ _srl(x, 30)
    x = x * m1
    x = x ^ _srl(x, 27)
    x = x * m2
    return x ^ _srl(x, 31)


def _served_base(seed: int, t: int) -> int:
    b = ((t + 1) << 40) + (seed % 256) * (1 << 56)
    return b - (1 << 64) if b >= 1 << 63 else b


def served_table_device(seed: int, t: int, n_rows: int, device):
    """served_table(seed, t, n_rows) generated on `device` (identical keys; payload from torch's
    generator)."""
    import torch
    idx = torch.arange(n_rows, dtype=torch.int64, device=device) + _served_base(seed, t)
    g = torch.Generator(device=device)
    g.manual_seed(seed * 7919 + t)
    payload = torch.randint(-2**62, 2**62, (n_rows,), dtype=torch.int64, device=device, generator=g)
    return mix64_torch(idx), payload


def served_probe_pool(seed: int, t: int, table_keys, n_pool: int, hit_rate: float = 0.7):
    """A shuffled pool of probe keys for table t: hit_rate of them drawn from the table's keys, the
    rest absent from it (mix64 of indices past the table's range). A request of n rows probes a
    random window of the pool."""
    import torch
    dev = table_keys.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed * 104729 + t)
    n_hit = int(round(n_pool * hit_rate))
    hits = table_keys[torch.randint(0, table_keys.numel(), (n_hit,), device=dev, generator=g)]
    miss_idx = table_keys.numel() + torch.randint(0, 1 << 30, (n_pool - n_hit,), device=dev, generator=g)
    misses = mix64_torch(miss_idx + _served_base(seed, t))
    keys = torch.cat([hits, misses])
    return keys[torch.randperm(n_pool, device=dev, generator=g)]


def served_requests(seed: int, n_requests: int, n_tables: int = 8, lo: float = 1e4, hi: float = 2e7):
    """(table, probe rows, window seed) per request: table uniform, size log-uniform [lo, hi]."""
    r = _rng(seed, 6000)
    tables = r.integers(0, n_tables, size=n_requests)
    sizes = np.floor(np.exp(r.uniform(np.log(lo), np.log(hi), size=n_requests))).astype(np.int64)
    starts = r.random(n_requests)
    return tables, sizes, starts
