"""Batched INNER joins (many independent small joins in one persistent launch) over torch tensors.

Mirrors the operator's many partition-pair joins (src/op/sirius_physical_hash_join.cpp, one
build + probe per (probe batch, build batch) pair in STANDARD mode, :1825-1943) executed as one
work queue on the GPU. Every join writes into its own caller-provided output buffers.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import torch

from . import _lib as L
from .join import _as_pair, _mut, make_column, _stream_handle


@dataclass
class BatchJoinOutput:
    probe_rid: torch.Tensor
    build_rid: torch.Tensor
    probe_payload: Optional[torch.Tensor] = None
    build_payload: Optional[torch.Tensor] = None


@dataclass
class BatchJoinSpec:
    build_key: torch.Tensor
    probe_key: torch.Tensor
    build_payload: Optional[torch.Tensor] = None
    probe_payload: Optional[torch.Tensor] = None
    build_validity: Optional[torch.Tensor] = None
    probe_validity: Optional[torch.Tensor] = None
    capacity: int = -1  # -1: probe rows (unique build keys)
    out: Optional[BatchJoinOutput] = field(default=None)


def batch_params(block_size=0, group_width=0, load_factor=0.0, tile_rows=0, ctas_per_sm=0) -> L.SjBatchParams:
    p = L.SjBatchParams()
    p.block_size, p.group_width, p.load_factor = block_size, group_width, load_factor
    p.tile_rows, p.ctas_per_sm = tile_rows, ctas_per_sm
    return p


class BatchPlan:
    """A planned batch; launch() runs every join in one persistent kernel."""

    def __init__(self, specs: List[BatchJoinSpec], params: Optional[L.SjBatchParams] = None,
                 stream: Optional[torch.cuda.Stream] = None, allocate_outputs: bool = True):
        self._lib = L.load()
        self.specs = specs
        arr = (L.SjBatchJoin * max(1, len(specs)))()
        for i, s in enumerate(specs):
            cap = s.capacity if s.capacity >= 0 else s.probe_key.numel()
            s.capacity = cap
            dev = s.probe_key.device
            if s.out is None and allocate_outputs:
                s.out = BatchJoinOutput(
                    torch.empty(cap, dtype=torch.int32, device=dev), torch.empty(cap, dtype=torch.int32, device=dev),
                    torch.empty(cap, dtype=s.probe_payload.dtype, device=dev) if s.probe_payload is not None else None,
                    torch.empty(cap, dtype=s.build_payload.dtype, device=dev) if s.build_payload is not None else None)
            j = arr[i]
            j.build_key = make_column(s.build_key, s.build_validity)
            j.probe_key = make_column(s.probe_key, s.probe_validity)
            if s.build_payload is not None:
                j.build_payload = make_column(s.build_payload)
                j.out_build_payload = _mut(s.out.build_payload, None)
            if s.probe_payload is not None:
                j.probe_payload = make_column(s.probe_payload)
                j.out_probe_payload = _mut(s.out.probe_payload, None)
            j.out_probe_rid = s.out.probe_rid.data_ptr() if cap else None
            j.out_build_rid = s.out.build_rid.data_ptr() if cap else None
            j.capacity = cap
        self.params = params if params is not None else batch_params()
        self._handle = ctypes.c_void_p()
        L.check(self._lib.sj_batch_plan_create(arr, len(specs), ctypes.byref(self.params), None,
                                               _stream_handle(stream), ctypes.byref(self._handle)),
                "sj_batch_plan_create")

    def launch(self, stream=None):
        L.check(self._lib.sj_batch_plan_launch(self._handle, _stream_handle(stream)), "sj_batch_plan_launch")

    def replay(self, stream: torch.cuda.Stream):
        L.check(self._lib.sj_batch_plan_replay(self._handle, _stream_handle(stream)), "sj_batch_plan_replay")

    def launch_per_join(self, stream=None):
        L.check(self._lib.sj_batch_plan_launch_per_join(self._handle, _stream_handle(stream)),
                "sj_batch_plan_launch_per_join")

    def counts(self, stream=None):
        """(device int64[num_joins] match counts, device int32[1] error word)."""
        dev = self.specs[0].probe_key.device if self.specs else torch.device("cuda")
        c = torch.zeros(max(1, len(self.specs)), dtype=torch.int64, device=dev)
        e = torch.zeros(1, dtype=torch.int32, device=dev)
        L.check(self._lib.sj_batch_plan_counts(self._handle, c.data_ptr(), e.data_ptr(), _stream_handle(stream)),
                "sj_batch_plan_counts")
        return c[:len(self.specs)], e

    def close(self, stream=None):
        if self._handle:
            self._lib.sj_batch_plan_destroy(self._handle, _stream_handle(stream))
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
