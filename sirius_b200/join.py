"""Host-side API of the join over torch device tensors, calling the C ABI (``libsj.so``).

``HashTable`` mirrors how Sirius's hash-join operator uses a built table
(``src/op/sirius_physical_hash_join.cpp``): build once per partition (``:1593-1624``), then
probe it many times, each probe followed by the payload gather (``gather_join_output``,
``:1299-1359``). ``inner_join`` is the one-shot STANDARD-mode join (``cudf::inner_join`` at
``:1872``). Output columns come in the operator's order: probe payloads, then build payloads.

torch is used only for device memory and streams; every join step runs in ``libsj.so``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import torch

from . import _lib as L

_TYPES = {
    torch.int8: L.SJ_INT8, torch.int16: L.SJ_INT16, torch.int32: L.SJ_INT32, torch.int64: L.SJ_INT64,
    torch.float32: L.SJ_FLOAT32, torch.float64: L.SJ_FLOAT64, torch.bool: L.SJ_BOOL8,
    torch.uint32: L.SJ_UINT32, torch.uint64: L.SJ_UINT64,
}


def sj_type(dtype: torch.dtype) -> int:
    try:
        return _TYPES[dtype]
    except KeyError:
        raise TypeError(f"unsupported column dtype {dtype}") from None


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _as_pair(c):
    """A payload/key argument is a tensor or a (tensor, validity-words-or-None) pair."""
    if isinstance(c, (tuple, list)):
        return c[0], (c[1] if len(c) > 1 else None)
    return c, None


def make_column(data: torch.Tensor, validity: Optional[torch.Tensor] = None, validity_offset: int = 0) -> L.SjColumn:
    if data.dim() != 1 or not data.is_contiguous():
        raise ValueError("columns must be contiguous 1-D tensors")
    if not data.is_cuda:
        raise ValueError("columns must live on the GPU")
    if validity is not None and (not validity.is_cuda or validity.dtype not in (torch.int32, torch.uint32)):
        raise ValueError("validity must be a CUDA int32/uint32 tensor of bitmask words")
    col = L.SjColumn()
    col.data = data.data_ptr() if data.numel() else None
    col.validity = validity.data_ptr() if validity is not None else None
    col.validity_offset = validity_offset
    col.num_rows = data.numel()
    col.type = sj_type(data.dtype)
    return col


def _keys(keys, validity=None):
    """Key argument -> (ctypes column array, number of columns, first tensor). `keys` is a tensor (with
    `validity`) or a list of tensors / (tensor, validity) pairs: a composite key of 2..4 columns."""
    if isinstance(keys, (list, tuple)):
        if validity is not None:
            raise ValueError("pass (tensor, validity) pairs for composite keys")
        pairs = [_as_pair(k) for k in keys]
        cols = [make_column(t, v) for t, v in pairs]
        return _cols(cols), len(cols), pairs[0][0]
    return _cols([make_column(keys, validity)]), 1, keys


def _cols(cols: Sequence[L.SjColumn], cls=L.SjColumn):
    arr = (cls * max(1, len(cols)))()
    for i, c in enumerate(cols):
        arr[i] = c
    return arr


@dataclass
class JoinOutput:
    """Result of an INNER probe + gather: ``count`` rows (the tensors may be longer)."""
    count: int
    probe_rid: Optional[torch.Tensor]
    build_rid: Optional[torch.Tensor]
    probe_payload: list = field(default_factory=list)
    build_payload: list = field(default_factory=list)
    probe_payload_validity: list = field(default_factory=list)
    build_payload_validity: list = field(default_factory=list)
    mark: Optional[torch.Tensor] = None           # MARK: one uint8 per probe row
    mark_validity: Optional[torch.Tensor] = None  # MARK: bitmask words

    def trimmed(self) -> "JoinOutput":
        n = self.count

        def cut(t):
            return None if t is None else t[:n]

        def cutv(v):
            return None if v is None else v[: (n + 31) // 32]
        return JoinOutput(n, cut(self.probe_rid), cut(self.build_rid),
                          [cut(t) for t in self.probe_payload], [cut(t) for t in self.build_payload],
                          [cutv(v) for v in self.probe_payload_validity],
                          [cutv(v) for v in self.build_payload_validity])


def allocate_output(capacity: int, probe_payload=(), build_payload=(), device=None, rids=True) -> JoinOutput:
    """Pre-allocate output buffers for ``capacity`` rows (payload dtypes/validity follow the inputs)."""
    dev = device or torch.device("cuda")
    words = (capacity + 31) // 32

    def outs(cols):
        data, val = [], []
        for c in cols:
            t, v = _as_pair(c)
            data.append(torch.empty(capacity, dtype=t.dtype, device=dev))
            val.append(torch.empty(words, dtype=torch.int32, device=dev) if v is not None else None)
        return data, val
    pd, pv = outs(probe_payload)
    bd, bv = outs(build_payload)
    prid = torch.empty(capacity, dtype=torch.int32, device=dev) if rids else None
    brid = torch.empty(capacity, dtype=torch.int32, device=dev) if rids else None
    return JoinOutput(0, prid, brid, pd, bd, pv, bv)


def _mut(t: torch.Tensor, v: Optional[torch.Tensor]) -> L.SjMutColumn:
    m = L.SjMutColumn()
    m.data = t.data_ptr() if t.numel() else None
    m.validity = v.data_ptr() if v is not None else None
    m.type = sj_type(t.dtype)
    return m


class HashTable:
    """A built table resident on the device (one partition slot of the BUILD_PROBE mode)."""

    def __init__(self, keys: torch.Tensor, validity: Optional[torch.Tensor] = None, *,
                 attach=(), layout: int = L.SJ_LAYOUT_AUTO, null_equality: int = L.SJ_NULLS_UNEQUAL,
                 load_factor: float = 0.5, partition_bits: int = 0, force_wide: bool = False,
                 ctas_per_sm: int = 0, aggregation: int = L.SJ_AGG_AUTO,
                 probe_kernel: int = L.SJ_PROBE_KERNEL_AUTO, rows_per_lane: int = 0,
                 probe_partition_mb: int = 0, table_l2_priority: int = L.SJ_L2_AUTO,
                 bloom_bits_per_key: int = 0, stream: Optional[torch.cuda.Stream] = None):
        """Build the table. ``attach``: build payload columns (tensor or (tensor, validity)) the
        table copies in its own position order (sj_build_ex); gather them with
        ``probe_gather(..., attached=True)``. ``partition_bits``: 0 = automatic, -1 = never.
        ``bloom_bits_per_key`` > 0: the insert pass also fills the join's dynamic filter
        (``bloom()``)."""
        self._lib = L.load()
        self._handle = ctypes.c_void_p()
        self.keys = keys
        self.params = L.default_params(layout=layout, null_equality=null_equality, load_factor=load_factor,
                                       partition_bits=partition_bits, force_wide=int(force_wide),
                                       aggregation=aggregation, probe_kernel=probe_kernel,
                                       rows_per_lane=rows_per_lane, probe_partition_mb=probe_partition_mb,
                                       table_l2_priority=table_l2_priority,
                                       bloom_bits_per_key=bloom_bits_per_key)
        if ctas_per_sm:
            self.params.ctas_per_sm = ctas_per_sm
        col, nkeys, first = _keys(keys, validity)
        self.attached = [_as_pair(c) for c in attach]
        if self.attached:
            pay = [make_column(t, v) for t, v in self.attached]
            st = self._lib.sj_build_ex(col, nkeys, _cols(pay), len(pay), ctypes.byref(self.params), None,
                                       _stream_handle(stream), ctypes.byref(self._handle))
            L.check(st, "sj_build_ex")
        else:
            st = self._lib.sj_build(col, nkeys, ctypes.byref(self.params), None,
                                    _stream_handle(stream), ctypes.byref(self._handle))
            L.check(st, "sj_build")
        self.build_rows = first.numel()

    @property
    def handle(self):
        if not self._handle:
            raise RuntimeError("table is closed")
        return self._handle

    def bloom(self) -> Optional["BloomFilter"]:
        """The dynamic filter the build filled (``bloom_bits_per_key`` > 0), owned by the table."""
        h = self._lib.sj_table_bloom(self.handle)
        return BloomFilter.view(h, self) if h else None

    def info(self) -> L.SjTableInfo:
        inf = L.SjTableInfo()
        L.check(self._lib.sj_table_get_info(self.handle, ctypes.byref(inf)), "sj_table_get_info")
        return inf

    def count(self, probe_keys: torch.Tensor, probe_validity: Optional[torch.Tensor] = None,
              stream: Optional[torch.cuda.Stream] = None, d_count: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Device int64[1] holding the number of INNER matches (stream-ordered)."""
        col, nkeys, first = _keys(probe_keys, probe_validity)
        dc = d_count if d_count is not None else torch.empty(1, dtype=torch.int64, device=first.device)
        L.check(self._lib.sj_probe_count(self.handle, col, nkeys, None, _stream_handle(stream),
                                         dc.data_ptr()), "sj_probe_count")
        return dc

    def probe_gather(self, probe_keys: torch.Tensor, probe_validity: Optional[torch.Tensor] = None,
                     probe_payload=(), build_payload=(), *, attached: bool = False, capacity: Optional[int] = None,
                     out: Optional[JoinOutput] = None, d_count: Optional[torch.Tensor] = None,
                     stream: Optional[torch.cuda.Stream] = None, sync: bool = True) -> JoinOutput:
        """INNER probe fused with the payload gather.

        ``capacity`` defaults to the exact count (one count pass + a sync) unless the table is
        DISTINCT, where the probe row count is an upper bound. With ``sync=False`` the returned
        ``count`` is -1 and the device count stays in ``d_count``.
        """
        kcols, nkeys, first = _keys(probe_keys, probe_validity)
        dev = first.device
        if capacity is None:
            if out is not None:
                capacity = out.probe_rid.numel() if out.probe_rid is not None else out.probe_payload[0].numel()
            elif self.info().layout == L.SJ_LAYOUT_DISTINCT:
                capacity = first.numel()
            else:
                capacity = int(self.count(probe_keys, probe_validity, stream).item())
        if attached:
            if build_payload:
                raise ValueError("attached=True gathers the attached build columns; pass no build_payload")
            build_payload = self.attached
        if out is None:
            out = allocate_output(capacity, probe_payload, build_payload, dev)
        pin = [make_column(*_as_pair(c)) for c in probe_payload]
        bin_ = [] if attached else [make_column(*_as_pair(c)) for c in build_payload]
        n_bin = len(build_payload)
        pout = [_mut(t, v) for t, v in zip(out.probe_payload, out.probe_payload_validity)]
        bout = [_mut(t, v) for t, v in zip(out.build_payload, out.build_payload_validity)]
        dc = d_count if d_count is not None else torch.empty(1, dtype=torch.int64, device=dev)
        st = self._lib.sj_probe_gather(
            self.handle, kcols, nkeys, _cols(pin), len(pin), None if attached else _cols(bin_), n_bin,
            out.probe_rid.data_ptr() if out.probe_rid is not None else None,
            out.build_rid.data_ptr() if out.build_rid is not None else None,
            _cols(pout, L.SjMutColumn), _cols(bout, L.SjMutColumn), capacity, None, _stream_handle(stream),
            dc.data_ptr())
        L.check(st, "sj_probe_gather")
        if not sync:
            out.count = -1
            return out
        out.count = int(dc.item())
        if out.count < 0:
            raise L.SjError(L.SJ_ERR_TIMEOUT, "sj_probe_gather", "a bounded device wait ran out")
        if out.count > capacity:
            raise L.SjError(L.SJ_ERR_CAPACITY, "sj_probe_gather", f"{out.count} matches > capacity {capacity}")
        return out

    def probe_join(self, kind: int, probe_keys: torch.Tensor, probe_validity: Optional[torch.Tensor] = None,
                   probe_payload=(), build_payload=(), *, attached: bool = False, capacity: Optional[int] = None,
                   stream: Optional[torch.cuda.Stream] = None) -> JoinOutput:
        """LEFT / SEMI / ANTI / MARK / FULL (``sj_probe_join``; INNER is ``probe_gather``).

        Outer rows carry ``SJ_NO_ROW`` as the missing side's row id and NULL payloads; LEFT/FULL
        outputs get validity buffers for every padded payload column. Synchronizes."""
        kcols, nkeys, first = _keys(probe_keys, probe_validity)
        dev = first.device
        n = first.numel()
        if kind == L.SJ_JOIN_INNER:
            return self.probe_gather(probe_keys, probe_validity, probe_payload, build_payload, attached=attached,
                                     capacity=capacity, stream=stream)
        if attached:
            if build_payload:
                raise ValueError("attached=True gathers the attached build columns; pass no build_payload")
            build_payload = self.attached
        out = JoinOutput(0, None, None)
        if kind == L.SJ_JOIN_MARK:
            out.mark = torch.empty(n, dtype=torch.uint8, device=dev)
            out.mark_validity = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
            capacity = 0
        else:
            if capacity is None:
                capacity = n
                if kind in (L.SJ_JOIN_LEFT, L.SJ_JOIN_FULL):
                    capacity += int(self.count(probe_keys, probe_validity, stream).item())
                if kind == L.SJ_JOIN_FULL:
                    capacity += self.build_rows
            pad_probe = kind == L.SJ_JOIN_FULL
            pad_build = kind in (L.SJ_JOIN_LEFT, L.SJ_JOIN_FULL)
            words = (capacity + 31) // 32
            out.probe_rid = torch.empty(capacity, dtype=torch.int32, device=dev)
            out.build_rid = torch.empty(capacity, dtype=torch.int32, device=dev) if pad_build else None
            for c in probe_payload:
                t, v = _as_pair(c)
                out.probe_payload.append(torch.empty(capacity, dtype=t.dtype, device=dev))
                out.probe_payload_validity.append(
                    torch.empty(words, dtype=torch.int32, device=dev) if (v is not None or pad_probe) else None)
            if pad_build:
                for c in build_payload:
                    t, _ = _as_pair(c)
                    out.build_payload.append(torch.empty(capacity, dtype=t.dtype, device=dev))
                    out.build_payload_validity.append(torch.empty(words, dtype=torch.int32, device=dev))
        pin = [make_column(*_as_pair(c)) for c in probe_payload]
        use_build = kind in (L.SJ_JOIN_LEFT, L.SJ_JOIN_FULL)
        bin_ = [] if (attached or not use_build) else [make_column(*_as_pair(c)) for c in build_payload]
        n_bin = len(build_payload) if use_build else 0
        pout = [_mut(t, v) for t, v in zip(out.probe_payload, out.probe_payload_validity)]
        bout = [_mut(t, v) for t, v in zip(out.build_payload, out.build_payload_validity)]
        dc = torch.empty(1, dtype=torch.int64, device=dev)
        st = self._lib.sj_probe_join(
            self.handle, kind, kcols, nkeys, _cols(pin), len(pin), None if attached else _cols(bin_), n_bin,
            out.probe_rid.data_ptr() if out.probe_rid is not None else None,
            out.build_rid.data_ptr() if out.build_rid is not None else None,
            _cols(pout, L.SjMutColumn), _cols(bout, L.SjMutColumn), capacity,
            out.mark.data_ptr() if out.mark is not None else None,
            out.mark_validity.data_ptr() if out.mark_validity is not None else None, None, _stream_handle(stream),
            dc.data_ptr())
        L.check(st, "sj_probe_join")
        out.count = int(dc.item())
        if kind != L.SJ_JOIN_MARK and out.count > capacity:
            raise L.SjError(L.SJ_ERR_CAPACITY, "sj_probe_join", f"{out.count} rows > capacity {capacity}")
        return out

    def close(self, stream: Optional[torch.cuda.Stream] = None):
        if self._handle:
            self._lib.sj_table_destroy(self._handle, _stream_handle(stream))
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def inner_join(build_keys, probe_keys, build_validity=None, probe_validity=None, probe_payload=(),
               build_payload=(), *, capacity: Optional[int] = None, **table_kwargs) -> JoinOutput:
    """One-shot INNER join (build, probe, gather, free): STANDARD mode."""
    stream = table_kwargs.pop("stream", None)
    with HashTable(build_keys, build_validity, stream=stream, **table_kwargs) as t:
        return t.probe_gather(probe_keys, probe_validity, probe_payload, build_payload, capacity=capacity,
                              stream=stream).trimmed()


# The RIGHT family of STANDARD mode (src/op/sirius_physical_hash_join.cpp:1879-1895), which the
# reference runs with the sides swapped: RIGHT = cudf::left_join(right_keys, left_keys); RIGHT_SEMI /
# RIGHT_ANTI = a filtered join built on the left keys and probed by the right ones.
JOIN_RIGHT, JOIN_RIGHT_SEMI, JOIN_RIGHT_ANTI = "right", "right_semi", "right_anti"


def right_join(kind: str, left_keys, right_keys, left_validity=None, right_validity=None, left_payload=(),
               right_payload=(), **table_kwargs) -> JoinOutput:
    """RIGHT / RIGHT_SEMI / RIGHT_ANTI: a table built on the LEFT keys, probed by the RIGHT keys.

    The result is the swapped join's: ``probe_rid`` / ``probe_payload`` are right-side rows and
    columns; for RIGHT, ``build_rid`` is the left row (``SJ_NO_ROW`` where the right row has no
    match) and ``build_payload`` the left columns, NULL where unmatched. RIGHT_SEMI / RIGHT_ANTI
    return the right rows with / without a match (a NULL right key has none). Synchronizes."""
    inner = {JOIN_RIGHT: L.SJ_JOIN_LEFT, JOIN_RIGHT_SEMI: L.SJ_JOIN_SEMI, JOIN_RIGHT_ANTI: L.SJ_JOIN_ANTI}
    if kind not in inner:
        raise ValueError(f"unknown RIGHT-family join {kind!r}")
    stream = table_kwargs.pop("stream", None)
    with HashTable(left_keys, left_validity, stream=stream, **table_kwargs) as t:
        return t.probe_join(inner[kind], right_keys, right_validity, right_payload,
                            left_payload if kind == JOIN_RIGHT else (), stream=stream)


def _host_column(data: torch.Tensor, validity: Optional[torch.Tensor] = None) -> L.SjColumn:
    """A column in host memory for sj_inner_join_host (pinned memory lets its copies overlap)."""
    if data.dim() != 1 or not data.is_contiguous() or data.is_cuda:
        raise ValueError("host columns must be contiguous 1-D CPU tensors")
    if validity is not None and (validity.is_cuda or validity.dtype not in (torch.int32, torch.uint32)):
        raise ValueError("host validity must be a CPU int32/uint32 tensor of bitmask words")
    col = L.SjColumn()
    col.data = data.data_ptr() if data.numel() else None
    col.validity = validity.data_ptr() if validity is not None else None
    col.validity_offset = 0
    col.num_rows = data.numel()
    col.type = sj_type(data.dtype)
    return col


def inner_join_host(build_keys, probe_keys, build_validity=None, probe_validity=None, probe_payload=(),
                    build_payload=(), *, capacity: Optional[int] = None, out: Optional[JoinOutput] = None,
                    chunk_rows: int = 0, stream: Optional[torch.cuda.Stream] = None, **table_kwargs) -> JoinOutput:
    """One-shot INNER join of host (CPU) tensors into host tensors (sj_inner_join_host).

    The build side is copied in and built. The probe side streams through in chunks of
    ``chunk_rows`` rows, with uploads, probes and downloads overlapped. Keys are a tensor (with
    ``*_validity``) or a list of tensors / (tensor, validity) pairs. Payloads carry no NULLs.
    ``capacity`` defaults to the probe row count, and ``out`` to pinned host buffers of that size.
    More matches than ``capacity`` raise SJ_ERR_CAPACITY, which reports the count."""
    def keys_of(k, v):
        if isinstance(k, (list, tuple)):
            if v is not None:
                raise ValueError("pass (tensor, validity) pairs for composite keys")
            pairs = [_as_pair(x) for x in k]
        else:
            pairs = [(k, v)]
        return _cols([_host_column(t, vv) for t, vv in pairs]), len(pairs), pairs[0][0]
    bcols, nkeys, _ = keys_of(build_keys, build_validity)
    pcols, pk_n, first = keys_of(probe_keys, probe_validity)
    if pk_n != nkeys:
        raise ValueError("build and probe have different numbers of key columns")
    pp = [_as_pair(c)[0] for c in probe_payload]
    bp = [_as_pair(c)[0] for c in build_payload]
    if capacity is None:
        capacity = out.probe_rid.numel() if out is not None else first.numel()
    if out is None:
        def host(n, dt):
            return torch.empty(n, dtype=dt).pin_memory()
        out = JoinOutput(0, host(capacity, torch.int32), host(capacity, torch.int32),
                         [host(capacity, t.dtype) for t in pp], [host(capacity, t.dtype) for t in bp])
    params = L.default_params(**{k: v for k, v in table_kwargs.items()})
    cnt = ctypes.c_int64(0)
    lib = L.load()
    st = lib.sj_inner_join_host(
        bcols, pcols, nkeys, _cols([_host_column(t) for t in pp]), len(pp), _cols([_host_column(t) for t in bp]),
        len(bp), out.probe_rid.data_ptr() if out.probe_rid is not None else None,
        out.build_rid.data_ptr() if out.build_rid is not None else None,
        _cols([_mut(t, None) for t in out.probe_payload], L.SjMutColumn),
        _cols([_mut(t, None) for t in out.build_payload], L.SjMutColumn), capacity, chunk_rows,
        ctypes.byref(params), None, _stream_handle(stream), ctypes.byref(cnt))
    L.check(st, "sj_inner_join_host")
    out.count = cnt.value
    if out.count > capacity:
        raise L.SjError(L.SJ_ERR_CAPACITY, "sj_inner_join_host", f"{out.count} matches > capacity {capacity}")
    return out


def hash_partition(keys, columns, num_partitions: int, stream: Optional[torch.cuda.Stream] = None):
    """Reorder `columns` (tensors or (tensor, validity) pairs) by the hash partition of `keys` (a
    tensor, or a list of 1..4 key columns / pairs). Returns (partitioned columns, partitioned validity
    words or None per column, offsets: int64 tensor of num_partitions + 1)."""
    lib = L.load()
    kcols, nkeys, first = _keys(keys)
    dev = first.device
    n = first.numel()
    pairs = [_as_pair(c) for c in columns]
    ins = [make_column(t, v) for t, v in pairs]
    outs = [torch.empty(n, dtype=t.dtype, device=dev) for t, _ in pairs]
    vouts = [torch.empty((n + 31) // 32, dtype=torch.int32, device=dev) if v is not None else None for _, v in pairs]
    offsets = torch.empty(num_partitions + 1, dtype=torch.int64, device=dev)
    st = lib.sj_hash_partition(kcols, nkeys, _cols(ins), len(ins), num_partitions,
                               _cols([_mut(t, v) for t, v in zip(outs, vouts)], L.SjMutColumn), offsets.data_ptr(),
                               None, _stream_handle(stream))
    L.check(st, "sj_hash_partition")
    return outs, vouts, offsets


class BloomFilter:
    """Dynamic filter from build keys (``sj_bloom_build``); ``contains`` gives the per-row mask."""

    def __init__(self, keys: torch.Tensor, validity: Optional[torch.Tensor] = None, bits_per_key: int = 16,
                 stream: Optional[torch.cuda.Stream] = None):
        self._lib = L.load()
        self._h = ctypes.c_void_p()
        self._owner = None
        col = make_column(keys, validity)
        L.check(self._lib.sj_bloom_build(ctypes.byref(col), bits_per_key, None, _stream_handle(stream),
                                         ctypes.byref(self._h)), "sj_bloom_build")

    @classmethod
    def view(cls, handle: int, owner) -> "BloomFilter":
        """A filter owned by `owner` (a HashTable's build-time filter): never destroyed here."""
        b = cls.__new__(cls)
        b._lib = L.load()
        b._h = ctypes.c_void_p(handle)
        b._owner = owner
        return b

    @property
    def nbytes(self) -> int:
        return int(self._lib.sj_bloom_bytes(self._h))

    def contains(self, probe_keys: torch.Tensor, probe_validity: Optional[torch.Tensor] = None,
                 stream: Optional[torch.cuda.Stream] = None):
        """(uint8 mask per row, validity words or None)."""
        n = probe_keys.numel()
        mask = torch.empty(n, dtype=torch.uint8, device=probe_keys.device)
        valid = torch.empty((n + 31) // 32, dtype=torch.int32, device=probe_keys.device) if probe_validity is not None else None
        col = make_column(probe_keys, probe_validity)
        L.check(self._lib.sj_bloom_contains(self._h, ctypes.byref(col), mask.data_ptr() if n else None,
                                            valid.data_ptr() if valid is not None else None,
                                            _stream_handle(stream)), "sj_bloom_contains")
        return mask, valid

    def close(self):
        if self._h and self._owner is None:
            self._lib.sj_bloom_destroy(self._h, None)
        self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
