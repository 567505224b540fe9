"""Host-side API of the join server (``sj_server_*`` in the C ABI): device-resident tables probed
by a stream of requests that a worker thread admits under a device-memory budget and runs
concurrently on several CUDA streams.

Tables and probe keys are torch device tensors. A request's probe key must be complete on the
device when it is submitted (``submit(..., sync=True)`` synchronizes the current stream first) and
stay alive until the request is polled. Results expose the server-owned output buffers as torch
tensors without a copy; they stay valid until ``release``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import torch

from . import _lib as L
from .join import _as_pair, _cols, make_column, sj_type

_DTYPES = {L.SJ_INT8: torch.int8, L.SJ_INT16: torch.int16, L.SJ_INT32: torch.int32, L.SJ_INT64: torch.int64,
           L.SJ_FLOAT32: torch.float32, L.SJ_FLOAT64: torch.float64, L.SJ_BOOL8: torch.bool,
           L.SJ_UINT32: torch.uint32, L.SJ_UINT64: torch.uint64}
_TYPESTR = {torch.int8: "|i1", torch.int16: "<i2", torch.int32: "<i4", torch.int64: "<i8",
            torch.float32: "<f4", torch.float64: "<f8", torch.bool: "|b1", torch.uint32: "<u4",
            torch.uint64: "<u8"}


class _DeviceBuffer:
    """A device pointer seen through ``__cuda_array_interface__`` (for torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, dtype: torch.dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": _TYPESTR[dtype], "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


def _view(ptr: Optional[int], n: int, dtype: torch.dtype, device) -> torch.Tensor:
    if not ptr or n == 0:
        return torch.empty(0, dtype=dtype, device=device)
    with torch.cuda.device(device):
        return torch.as_tensor(_DeviceBuffer(ptr, n, dtype), device=device)


@dataclass
class RequestResult:
    request_id: int
    status: int
    table_id: int
    count: int
    probe_rows: int
    probe_rid: torch.Tensor
    build_rid: torch.Tensor
    build_payload: List[torch.Tensor]
    build_validity: List[Optional[torch.Tensor]]
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class JoinServer:
    """Resident tables + continuous batching of probe requests (``sj_server_create``)."""

    def __init__(self, slots: int = 4, max_skip: int = 8, memory_budget_bytes: int = 120 << 30,
                 reserve_bytes: int = 0, batch_small: bool = True, device=None):
        """``batch_small``: run queued small requests (fewer than 65,536 rows) together as one kernel
        launch on the server's batch stream; False runs every request alone on a slot stream."""
        self._lib = L.load()
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        cfg = L.SjServerConfig()
        cfg.slots, cfg.max_skip, cfg.memory_budget_bytes = slots, max_skip, memory_budget_bytes
        cfg.reserve_bytes = reserve_bytes
        cfg.batch_small = 0 if batch_small else -1
        self._h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            L.check(self._lib.sj_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "sj_server_create")
        self._tables: Dict[int, tuple] = {}
        self._inflight: Dict[int, torch.Tensor] = {}

    def add_table(self, keys: torch.Tensor, attach: Sequence = (), load_factor: float = 0.5,
                  partition_bits: int = 0) -> int:
        """Build a resident table of unique keys with attached payload columns; returns its id."""
        torch.cuda.current_stream(self.device).synchronize()
        pay = [_as_pair(c) for c in attach]
        cols = [make_column(t, v) for t, v in pay]
        params = L.default_params(load_factor=load_factor, partition_bits=partition_bits)
        tid = ctypes.c_int32()
        key = make_column(keys)
        L.check(self._lib.sj_server_add_table(self._h, ctypes.byref(key), _cols(cols), len(cols),
                                              ctypes.byref(params), ctypes.byref(tid)), "sj_server_add_table")
        self._tables[tid.value] = (keys, [t for t, _ in pay], [sj_type(t.dtype) for t, _ in pay],
                                   [v is not None for _, v in pay])
        return tid.value

    def submit(self, table_id: int, probe_keys: torch.Tensor, request_id: int, sync: bool = True):
        if sync:
            torch.cuda.current_stream(self.device).synchronize()
        col = make_column(probe_keys)
        L.check(self._lib.sj_server_submit(self._h, table_id, ctypes.byref(col), request_id), "sj_server_submit")
        self._inflight[request_id] = probe_keys

    def poll(self, capacity: int = 64, wait_ms: int = 0) -> List[RequestResult]:
        buf = (L.SjRequestResult * capacity)()
        n = self._lib.sj_server_poll(self._h, buf, capacity, wait_ms)
        if n < 0:
            L.check(-n, "sj_server_poll")
        out = []
        for i in range(n):
            r = buf[i]
            self._inflight.pop(r.request_id, None)
            _, _, types, has_valid = self._tables[r.table_id]
            cnt = r.count if r.status == L.SJ_OK else 0
            pay = [_view(r.build_payload[c], cnt, _DTYPES[types[c]], self.device) for c in range(len(types))]
            val = [_view(r.build_validity[c], (cnt + 31) // 32, torch.int32, self.device) if has_valid[c] else None
                   for c in range(len(types))]
            out.append(RequestResult(r.request_id, r.status, r.table_id, r.count, r.probe_rows,
                                     _view(r.probe_rid, cnt, torch.int32, self.device),
                                     _view(r.build_rid, cnt, torch.int32, self.device), pay, val,
                                     r.t_submit, r.t_admit, r.t_done))
        return out

    def release(self, request_id: int):
        L.check(self._lib.sj_server_release(self._h, request_id), "sj_server_release")

    def close(self):
        if self._h:
            with torch.cuda.device(self.device):
                L.check(self._lib.sj_server_destroy(self._h), "sj_server_destroy")
            self._h = ctypes.c_void_p()
            self._tables.clear()
            self._inflight.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
