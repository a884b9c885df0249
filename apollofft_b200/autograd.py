"""torch.autograd Functions whose backward is the library's adjoint kernel.

The forward calls afc_execute; the backward calls afc_execute_adjoint, which
runs the conjugate transform with the exact scaling (and, for half spectra,
the Hermitian weights).  With torch's convention for complex gradients
(grad = dL/d(Re z) + i dL/d(Im z)) the adjoint of a C-linear map A is A^H, of an
R->C map Re(A^H .), of a C->R map A^H applied to the real cotangent.
The reference has no autograd; this is the capability that makes spectral
losses and NUFFT/STFT pipelines built on the plans trainable.
"""
from __future__ import annotations

import torch

from .plan import CudaPlan

_PREC = {torch.float32: "f32", torch.complex64: "f32", torch.float64: "f64", torch.complex128: "f64"}


class _PlanFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan: CudaPlan, inverse: bool, out_shape):
        ctx.plan = plan
        ctx.inverse = inverse
        ctx.in_shape = x.shape
        y = plan.execute(x.contiguous(), inverse=inverse)
        return y.reshape(out_shape)

    @staticmethod
    def backward(ctx, g):
        gx = ctx.plan.adjoint(g.contiguous(), inverse=ctx.inverse)
        return gx.reshape(ctx.in_shape), None, None, None


def _split(x, ndim):
    if x.dim() < ndim:
        raise ValueError(f"expected at least {ndim} dimensions, got {x.dim()}")
    dims = list(x.shape[x.dim() - ndim:])
    batch = 1
    for d in x.shape[: x.dim() - ndim]:
        batch *= d
    return dims, batch, tuple(x.shape[: x.dim() - ndim])


def fftn(x: torch.Tensor, ndim: int = 1, inverse: bool = False) -> torch.Tensor:
    """Complex-to-complex transform over the last `ndim` dims (leading dims batch)."""
    if not x.is_complex():
        raise ValueError("fftn expects a complex tensor")
    dims, batch, lead = _split(x, ndim)
    plan = CudaPlan(dims, precision=_PREC[x.dtype], kind="c2c", batch=batch, device=x.device.index or 0)
    return _PlanFn.apply(x, plan, inverse, lead + tuple(dims))


def rfftn(x: torch.Tensor, ndim: int = 1, half: bool = False) -> torch.Tensor:
    """Real-to-complex transform over the last `ndim` dims.  half=False: the
    reference's full spectrum (same shape); half=True: last dim n -> n/2+1."""
    if x.is_complex():
        raise ValueError("rfftn expects a real tensor")
    dims, batch, lead = _split(x, ndim)
    plan = CudaPlan(dims, precision=_PREC[x.dtype], kind="r2c_half" if half else "r2c_full", batch=batch,
                    device=x.device.index or 0)
    out_dims = list(dims)
    if half:
        out_dims[-1] = dims[-1] // 2 + 1
    return _PlanFn.apply(x, plan, False, lead + tuple(out_dims))


def irfftn(X: torch.Tensor, n_last: int, ndim: int = 1, half: bool = False) -> torch.Tensor:
    """Complex-to-real inverse over the last `ndim` dims (scaled by 1/N)."""
    if not X.is_complex():
        raise ValueError("irfftn expects a complex tensor")
    dims, batch, lead = _split(X, ndim)
    full = list(dims)
    full[-1] = n_last
    expect = n_last // 2 + 1 if half else n_last
    if dims[-1] != expect:
        raise ValueError(f"inconsistent spectrum length {dims[-1]} for n_last={n_last} (expected {expect})")
    plan = CudaPlan(full, precision=_PREC[X.dtype], kind="r2c_half" if half else "r2c_full", batch=batch,
                    device=X.device.index or 0)
    return _PlanFn.apply(X, plan, True, lead + tuple(full))


def rfft2(x: torch.Tensor, half: bool = False) -> torch.Tensor:
    return rfftn(x, 2, half)


def irfft2(X: torch.Tensor, n_last: int, half: bool = False) -> torch.Tensor:
    return irfftn(X, n_last, 2, half)
