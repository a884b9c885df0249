"""1D and 3D non-uniform FFTs on the device (apollo-nufft's NufftPlan1D and
NufftPlan3D).

`NufftPlan1D(n, dx, sigma=2, kernel_width=6)` mirrors the reference plan
(crates/apollo-nufft/src/application/execution/transform/dimension_1d.rs):
n uniform bins on the periodic domain [0, n dx), an oversampled grid of
sigma n points, the Kaiser-Bessel kernel of half width kernel_width.
`type1(positions, values)` -> n bins ~ sum_j c_j exp(-2 pi i k x_j / L);
`type2(coeffs, positions)` -> values ~ sum_k f_k exp(+2 pi i k x_j / L)
(k signed, L = n dx).  Positions float64, values complex128, torch tensors on
the plan's device.

`NufftPlan3D((nx, ny, nz), (dx, dy, dz), sigma=2, kernel_width=6)` mirrors
transform/dimension_3d.rs: per axis an oversampled grid of
next_pow2(max(sigma n, 2 kernel_width + 1)) points.  `type1(positions,
values)` takes positions of shape (npts, 3) and returns (nx, ny, nz) modes;
`type2(modes, positions)` returns npts values carrying the reference's
1 / (mx my mz) from its normalized inverse axis passes.
"""
from __future__ import annotations

import ctypes

from . import _lib as L
from .plan import require_device

DEFAULT_NUFFT_KERNEL_WIDTH = 6
DEFAULT_NUFFT_OVERSAMPLING = 2


class NufftPlan1D:
    def __init__(self, n: int, dx: float, sigma: int = DEFAULT_NUFFT_OVERSAMPLING,
                 kernel_width: int = DEFAULT_NUFFT_KERNEL_WIDTH, device: int = 0):
        self.n, self.dx, self.sigma, self.kernel_width = int(n), float(dx), int(sigma), int(kernel_width)
        self.m = self.sigma * self.n
        self.device = int(device)
        self._h = ctypes.c_void_p()
        L.check(L.lib().afc_nufft1d_plan_create(ctypes.byref(self._h), self.n, self.dx, self.sigma,
                                                self.kernel_width, self.device), "nufft plan")

    def _check(self, t, dtype, what):
        if t.dtype != dtype or not t.is_contiguous() or t.dim() != 1 or not t.is_cuda:
            raise ValueError(f"{what}: expected a contiguous 1D {dtype} tensor")
        require_device(t, self.device, what)

    def type1(self, positions, values, out=None, stream=None):
        import torch
        self._check(positions, torch.float64, "positions")
        self._check(values, torch.complex128, "values")
        if positions.numel() != values.numel():
            raise ValueError("positions/value length mismatch")
        if out is None:
            out = torch.empty(self.n, dtype=torch.complex128, device=values.device)
        self._check(out, torch.complex128, "output")
        if out.numel() != self.n:
            raise ValueError("output length mismatch")
        st = stream if stream is not None else torch.cuda.current_stream(values.device).cuda_stream
        L.check(L.lib().afc_nufft1d_type1(self._h, positions.data_ptr(), values.data_ptr(), positions.numel(),
                                          out.data_ptr(), st), "nufft type1")
        return out

    def type2(self, coeffs, positions, out=None, stream=None):
        import torch
        self._check(positions, torch.float64, "positions")
        self._check(coeffs, torch.complex128, "fourier_coeffs")
        if coeffs.numel() != self.n:
            raise ValueError("fourier_coeffs length mismatch")
        if out is None:
            out = torch.empty(positions.numel(), dtype=torch.complex128, device=coeffs.device)
        self._check(out, torch.complex128, "output")
        if out.numel() != positions.numel():
            raise ValueError("output length mismatch")
        st = stream if stream is not None else torch.cuda.current_stream(coeffs.device).cuda_stream
        L.check(L.lib().afc_nufft1d_type2(self._h, coeffs.data_ptr(), positions.data_ptr(), positions.numel(),
                                          out.data_ptr(), st), "nufft type2")
        return out

    def close(self):
        if self._h:
            L.lib().afc_nufft_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NufftPlan3D:
    def __init__(self, shape, spacing, sigma: int = DEFAULT_NUFFT_OVERSAMPLING,
                 kernel_width: int = DEFAULT_NUFFT_KERNEL_WIDTH, device: int = 0):
        self.shape = tuple(int(v) for v in shape)
        self.spacing = tuple(float(v) for v in spacing)
        if len(self.shape) != 3 or len(self.spacing) != 3:
            raise ValueError("shape and spacing must have three entries")
        self.sigma, self.kernel_width, self.device = int(sigma), int(kernel_width), int(device)
        self._h = ctypes.c_void_p()
        L.check(L.lib().afc_nufft3d_plan_create(ctypes.byref(self._h), *self.shape, *self.spacing, self.sigma,
                                                self.kernel_width, self.device), "nufft3d plan")
        m = (ctypes.c_int64 * 3)()
        L.check(L.lib().afc_nufft3d_grid_dims(self._h, m), "nufft3d grid dims")
        self.oversampled = tuple(int(v) for v in m)

    def _check(self, t, dtype, what, shape=None):
        if t.dtype != dtype or not t.is_contiguous() or not t.is_cuda:
            raise ValueError(f"{what}: expected a contiguous {dtype} tensor")
        require_device(t, self.device, what)
        if shape is not None and tuple(t.shape) != tuple(shape):
            raise ValueError(f"{what}: expected shape {tuple(shape)}, got {tuple(t.shape)}")

    def type1(self, positions, values, out=None, stream=None):
        import torch
        npts = values.numel()
        self._check(positions, torch.float64, "positions", (npts, 3))
        self._check(values, torch.complex128, "values")
        if out is None:
            out = torch.empty(self.shape, dtype=torch.complex128, device=values.device)
        self._check(out, torch.complex128, "output", self.shape)
        st = stream if stream is not None else torch.cuda.current_stream(values.device).cuda_stream
        L.check(L.lib().afc_nufft3d_type1(self._h, positions.data_ptr(), values.data_ptr(), npts, out.data_ptr(), st),
                "nufft3d type1")
        return out

    def type2(self, modes, positions, out=None, stream=None):
        import torch
        self._check(modes, torch.complex128, "modes", self.shape)
        if positions.dim() != 2 or positions.shape[1] != 3:
            raise ValueError("positions: expected shape (npts, 3)")
        npts = positions.shape[0]
        self._check(positions, torch.float64, "positions")
        if out is None:
            out = torch.empty(npts, dtype=torch.complex128, device=modes.device)
        self._check(out, torch.complex128, "output", (npts,))
        st = stream if stream is not None else torch.cuda.current_stream(modes.device).cuda_stream
        L.check(L.lib().afc_nufft3d_type2(self._h, modes.data_ptr(), positions.data_ptr(), npts, out.data_ptr(), st),
                "nufft3d type2")
        return out

    def close(self):
        if self._h:
            L.lib().afc_nufft3d_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
