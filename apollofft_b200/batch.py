"""Uneven batches: many 1D transforms of different lengths in one call.

Lanes are packed back to back (offset = prefix sum of lengths).  mode 0 runs
the whole batch as one CUDA graph (captured on first use for a buffer pair),
mode 1 issues one plain launch per distinct length.  No reference counterpart
(apollo-fft callers loop over FftPlan1D per lane).
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib as L
from .plan import require_device


class BatchPlan:
    def __init__(self, lengths: Sequence[int], precision: str = "f32", device: int = 0):
        self.lengths = np.ascontiguousarray(np.asarray(lengths, dtype=np.int64))
        self.precision = precision
        self.device = int(device)
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths)[:-1]]).astype(np.int64)
        self.total = int(self.lengths.sum())
        self._h = ctypes.c_void_p()
        prec = L.PREC_F64 if precision == "f64" else L.PREC_F32
        arr = self.lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        L.check(L.lib().afc_batch_plan_create(ctypes.byref(self._h), arr, len(self.lengths), prec, int(device)),
                "batch plan")

    def execute(self, x, out=None, inverse: bool = False, mode: int = 0, stream=None):
        import torch
        want = torch.complex128 if self.precision == "f64" else torch.complex64
        if x.dtype != want or not x.is_contiguous() or x.numel() != self.total or not x.is_cuda:
            raise ValueError(f"expected a contiguous {want} tensor of {self.total} elements")
        require_device(x, self.device, "input")
        if out is None:
            out = torch.empty_like(x)
        if out.dtype != want or not out.is_contiguous() or out.numel() != self.total or not out.is_cuda:
            raise ValueError("output buffer does not match the plan")
        require_device(out, self.device, "output")
        st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        L.check(L.lib().afc_batch_execute(self._h, x.data_ptr(), out.data_ptr(), int(inverse), int(mode), st),
                "batch execute")
        return out

    def close(self):
        if self._h:
            L.lib().afc_batch_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
