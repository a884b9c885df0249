"""Chirp z-transform on the device (apollo-czt's CztPlan).

`CztPlan(n, m, a, w)` mirrors apollo-czt's plan
(crates/apollo-czt/src/application/execution/plan/czt/dimension_1d.rs:60-120):
X_k = sum_j x_j a^-j w^(j k) for k < m, evaluated with Bluestein's identity over
a convolution of length next_pow2(n + m - 1).  The premultiply, both FFTs, the
kernel product and the postmultiply run in one kernel launch on device data
when the convolution fits one CTA, else around the multi-pass plan.
`inverse(X)` is the reference's exact inverse of a square plan (CztPlan::inverse:
Björck-Pereyra solve on the nodes W^k), one CTA per lane in FP64.
"""
from __future__ import annotations

import ctypes

from . import _lib as L
from .plan import require_device


class CztError(ValueError):
    """Invalid CZT parameters (the reference's CztError variants)."""


class CztPlan:
    def __init__(self, n: int, m: int, a: complex = 1.0, w: complex = None, precision: str = "f64", device: int = 0):
        import cmath
        if w is None:
            w = cmath.exp(-2j * cmath.pi / max(int(m), 1))
        a, w = complex(a), complex(w)
        if n <= 0 or m <= 0:
            raise CztError("CZT lengths must be positive")
        if not (cmath.isfinite(a) and cmath.isfinite(w)) or a == 0 or w == 0:
            raise CztError("CZT parameters must be finite and non-zero")
        if precision not in ("f64", "f32"):
            raise CztError(f"unsupported precision `{precision}`; expected f64 or f32")
        self.n, self.m, self.a, self.w = int(n), int(m), a, w
        self.precision = precision
        self.device = int(device)
        self._h = ctypes.c_void_p()
        prec = L.PREC_F64 if precision == "f64" else L.PREC_F32
        L.check(L.lib().afc_czt_plan_create(ctypes.byref(self._h), self.n, self.m, a.real, a.imag, w.real, w.imag,
                                            prec, self.device), "czt plan")

    def input_len(self) -> int:
        return self.n

    def output_len(self) -> int:
        return self.m

    def convolution_len(self) -> int:
        v = ctypes.c_int64()
        L.check(L.lib().afc_czt_conv_len(self._h, ctypes.byref(v)), "czt conv len")
        return v.value

    def forward(self, x, out=None, stream=None):
        """x: complex torch tensor on the device with last dimension n (any
        leading batch); returns the (..., m) transform."""
        import torch
        cdt = torch.complex128 if self.precision == "f64" else torch.complex64
        if x.dtype != cdt or not x.is_contiguous() or x.shape[-1] != self.n or not x.is_cuda:
            raise ValueError(f"expected a contiguous {cdt} tensor with last dimension {self.n}")
        require_device(x, self.device, "input")
        batch = x.numel() // self.n
        if out is None:
            out = torch.empty(tuple(x.shape[:-1]) + (self.m,), dtype=cdt, device=x.device)
        if out.dtype != cdt or not out.is_contiguous() or out.numel() != batch * self.m or not out.is_cuda:
            raise ValueError("output buffer does not match the plan")
        require_device(out, self.device, "output")
        st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        L.check(L.lib().afc_czt_execute(self._h, x.data_ptr(), out.data_ptr(), batch, st), "czt execute")
        return out

    def inverse(self, X, out=None, stream=None):
        """X: complex torch tensor on the device with last dimension n (= m);
        returns the signal whose forward transform is X."""
        import torch
        cdt = torch.complex128 if self.precision == "f64" else torch.complex64
        if X.dtype != cdt or not X.is_contiguous() or X.shape[-1] != self.m or not X.is_cuda:
            raise ValueError(f"expected a contiguous {cdt} tensor with last dimension {self.m}")
        require_device(X, self.device, "spectrum")
        batch = X.numel() // self.m
        if out is None:
            out = torch.empty(tuple(X.shape[:-1]) + (self.n,), dtype=cdt, device=X.device)
        if out.dtype != cdt or not out.is_contiguous() or out.numel() != batch * self.n or not out.is_cuda:
            raise ValueError("output buffer does not match the plan")
        require_device(out, self.device, "output")
        st = stream if stream is not None else torch.cuda.current_stream(X.device).cuda_stream
        status = L.lib().afc_czt_inverse(self._h, X.data_ptr(), out.data_ptr(), batch, st)
        if status == L.AFC_ERR_VALIDATION:
            raise CztError(L.last_error())
        L.check(status, "czt inverse")
        return out

    def close(self):
        if self._h:
            L.lib().afc_czt_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
