"""Analytic signal / Hilbert transform on the device (apollo-hilbert's HilbertPlan).

`HilbertPlan(n, precision="f64")` mirrors crates/apollo-hilbert/src/application/
execution/plan/hilbert.rs: `analytic_signal(x)` returns x + i H{x} for real
lanes of length n (forward FFT, the analytic mask, normalized inverse FFT, one
fused launch of this library per call); `transform(x)` is the quadrature H{x}
(the imaginary part), `envelope(x)` its magnitude and `phase(x)` its wrapped
angle, as the reference derives them from the analytic signal.  Input: a
contiguous real tensor (float64 for "f64", float32 for "f32") whose last
dimension is n; leading dimensions are lanes.
"""
from __future__ import annotations

import ctypes

from . import _lib as L
from .plan import require_device

_PREC = {"f32": L.PREC_F32, "f64": L.PREC_F64}


class HilbertPlan:
    def __init__(self, n: int, precision: str = "f64", device: int = 0):
        if precision not in _PREC:
            raise ValueError(f"unsupported precision `{precision}`; expected f32 or f64")
        self.n, self.precision, self.device = int(n), precision, int(device)
        self._h = ctypes.c_void_p()
        L.check(L.lib().afc_hilbert_plan_create(ctypes.byref(self._h), self.n, _PREC[precision], self.device),
                "hilbert plan")

    def __len__(self):
        return self.n

    def analytic_signal(self, x, out=None, stream=None):
        import torch
        rt = torch.float64 if self.precision == "f64" else torch.float32
        ct = torch.complex128 if self.precision == "f64" else torch.complex64
        if x.dtype != rt or not x.is_contiguous() or x.dim() < 1 or x.shape[-1] != self.n or not x.is_cuda:
            raise ValueError(f"signal: expected a contiguous {rt} tensor whose last dimension is {self.n}")
        require_device(x, self.device, "signal")
        lanes = x.numel() // self.n
        if out is None:
            out = torch.empty(x.shape, dtype=ct, device=x.device)
        if out.dtype != ct or not out.is_contiguous() or out.numel() != x.numel() or not out.is_cuda:
            raise ValueError("output buffer does not match the signal")
        require_device(out, self.device, "output")
        if lanes == 0:
            return out
        st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        L.check(L.lib().afc_hilbert_analytic(self._h, x.data_ptr(), out.data_ptr(), lanes, st), "analytic signal")
        return out

    def transform(self, x):
        return self.analytic_signal(x).imag.contiguous()

    def envelope(self, x):
        return self.analytic_signal(x).abs()

    def phase(self, x):
        return self.analytic_signal(x).angle()

    def close(self):
        if self._h:
            L.lib().afc_hilbert_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
