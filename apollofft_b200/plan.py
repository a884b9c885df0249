"""Device plans over the C ABI (torch tensors in HBM, host numpy buffers).

`CudaPlan` mirrors FftPlan1D/2D/3D (crates/apollo-fft/src/application/execution/
plan/fft/dimension_{1,2,3}d.rs): forward unnormalized, inverse scaled by 1/N,
C-order data.  Plans come from the library's process-wide cache
(afc_plan_get_cached, the counterpart of orchestration/cache/plans.rs).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

_PREC = {"f32": L.PREC_F32, "f64": L.PREC_F64, "tc_bf16": L.PREC_TC_BF16, "tc_fp16": L.PREC_TC_FP16}
_KIND = {"c2c": L.KIND_C2C, "r2c_full": L.KIND_R2C_FULL, "r2c_half": L.KIND_R2C_HALF}


class CudaPlan:
    """A (batched) rank-1..3 transform plan resident on one CUDA device."""

    def __init__(self, dims: Sequence[int], precision: str = "f64", kind: str = "c2c", batch: int = 1,
                 device: int = 0, cached: bool = True):
        dims = [int(d) for d in dims]
        if precision not in _PREC:
            raise ValueError(f"unsupported precision `{precision}`; expected f32, f64, tc_bf16 or tc_fp16")
        if kind not in _KIND:
            raise ValueError(f"unsupported kind `{kind}`; expected c2c, r2c_full or r2c_half")
        self.dims = tuple(dims)
        self.rank = len(dims)
        self.precision = precision
        self.kind = kind
        self.batch = int(batch)
        self.device = int(device)
        self._h = ctypes.c_void_p()
        self._exec = L.lib().afc_execute
        arr = (ctypes.c_int64 * max(self.rank, 1))(*dims)
        fn = L.lib().afc_plan_get_cached if cached else L.lib().afc_plan_create
        L.check(fn(ctypes.byref(self._h), self.rank, arr, _PREC[precision], _KIND[kind], self.batch, self.device),
                "plan")

    # ── sizes ──
    @property
    def n(self) -> int:
        return int(np.prod(self.dims))

    def io_elems(self, inverse: bool = False):
        inverse = bool(inverse)
        cache = self.__dict__.setdefault("_io_cache", {})
        if inverse not in cache:  # fixed per plan: one library call per direction
            a, b = ctypes.c_int64(), ctypes.c_int64()
            L.check(L.lib().afc_plan_io_elems(self._h, int(inverse), ctypes.byref(a), ctypes.byref(b)), "io_elems")
            cache[inverse] = (a.value, b.value)
        return cache[inverse]

    def workspace_size(self) -> int:
        s = ctypes.c_size_t()
        L.check(L.lib().afc_workspace_size(self._h, ctypes.byref(s)), "workspace_size")
        return s.value

    def describe(self, axis: int = 0) -> dict:
        info = L.LengthInfo()
        L.check(L.lib().afc_plan_describe(self._h, axis, ctypes.byref(info)), "describe")
        return L._info_dict(info)

    # ── dtypes ──
    def _real_dtype(self):
        return np.float64 if self.precision == "f64" else np.float32

    def _cplx_dtype(self):
        return np.complex128 if self.precision == "f64" else np.complex64  # tensor-core plans use complex64

    def in_dtype(self, inverse: bool):
        if self.kind == "c2c" or inverse:
            return self._cplx_dtype()
        return self._real_dtype()

    def out_dtype(self, inverse: bool):
        if self.kind == "c2c" or not inverse:
            return self._cplx_dtype()
        return self._real_dtype()

    def out_shape(self, inverse: bool):
        lead = (self.batch,) if self.batch > 1 else ()
        dims = list(self.dims)
        if self.kind == "r2c_half" and not inverse:
            dims[-1] = dims[-1] // 2 + 1
        return lead + tuple(dims)

    def _io(self, inverse: bool):
        """(input dtype, output dtype, input elements, output elements), cached per direction."""
        inverse = bool(inverse)
        cache = self.__dict__.setdefault("_io_full", {})
        if inverse not in cache:
            ie, oe = self.io_elems(inverse)
            cache[inverse] = (_TORCH_DTYPES[np.dtype(self.in_dtype(inverse))],
                              _TORCH_DTYPES[np.dtype(self.out_dtype(inverse))], ie, oe)
        return cache[inverse]

    # ── device execution (torch tensors) ──
    def execute(self, x, out=None, inverse: bool = False, scale: Optional[float] = None, stream=None):
        """Runs on torch CUDA tensors; returns `out` (allocated if None)."""
        io = self.__dict__.get("_io_inv" if inverse else "_io_fwd")
        if io is None:  # fixed per plan and direction: looked up once
            io = self._io(inverse)
            self.__dict__["_io_inv" if inverse else "_io_fwd"] = io
        t_in, t_out, ie, oe = io
        if x.dtype != t_in:
            raise ValueError(f"expected {t_in} input, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError("input must be C-contiguous")
        if x.numel() != ie:
            raise ValueError(f"shape mismatch: expected {ie} elements, got {x.numel()}")
        if not x.is_cuda:
            raise ValueError("input must be a CUDA tensor (use execute_host for host arrays)")
        if x.get_device() != self.device:
            require_device(x, self.device, "input")
        if out is None:
            import torch
            out = torch.empty(self.out_shape(inverse) if oe == int(np.prod(self.out_shape(inverse))) else (oe,),
                              dtype=t_out, device=x.device)
        if out.numel() != oe or out.dtype != t_out or not out.is_contiguous() or not out.is_cuda:
            raise ValueError("output buffer does not match the plan")
        if out.get_device() != self.device:
            require_device(out, self.device, "output")
        st = stream if stream is not None else _stream_of(x)
        if scale is None:
            status = self._exec(self._h, x.data_ptr(), out.data_ptr(), 1 if inverse else 0, st)
        else:
            status = L.lib().afc_execute_scaled(self._h, x.data_ptr(), out.data_ptr(), int(inverse), float(scale), st)
        if status:
            L.check(status, "execute")
        return out

    def adjoint(self, g, inverse: bool = False, stream=None):
        """Adjoint of `execute(., inverse)` applied to g (the autograd backward)."""
        import torch
        # the adjoint of the forward map consumes the forward's output type and
        # produces its input type
        t_in = _TORCH_DTYPES[np.dtype(self.out_dtype(inverse))]
        t_out = _TORCH_DTYPES[np.dtype(self.in_dtype(inverse))]
        ie, oe = self.io_elems(inverse)
        g = g.to(t_in).contiguous()
        require_device(g, self.device, "gradient")
        if g.numel() != oe:
            raise ValueError(f"shape mismatch: expected {oe} elements, got {g.numel()}")
        out = torch.empty((ie,), dtype=t_out, device=g.device)
        st = stream if stream is not None else torch.cuda.current_stream(g.device).cuda_stream
        L.check(L.lib().afc_execute_adjoint(self._h, g.data_ptr(), out.data_ptr(), int(inverse), st), "adjoint")
        return out

    # ── host execution (numpy arrays; copies inside the C ABI) ──
    def execute_host(self, x: np.ndarray, inverse: bool = False) -> np.ndarray:
        ie, oe = self.io_elems(inverse)
        x = np.asarray(x)
        if x.dtype != np.dtype(self.in_dtype(inverse)):
            raise ValueError(f"expected {np.dtype(self.in_dtype(inverse))} input, got {x.dtype}")
        if not x.flags.c_contiguous:
            raise ValueError("input must be C-contiguous")
        if x.size != ie:
            raise ValueError(f"shape mismatch: expected {ie} elements, got {x.size}")
        out = np.empty(oe, dtype=self.out_dtype(inverse))
        L.check(L.lib().afc_execute_host(self._h, x.ctypes.data, out.ctypes.data, int(inverse)), "execute_host")
        return out

    def close(self):
        if self._h:
            L.lib().afc_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def require_device(t, device: int, what: str) -> None:
    """Raises ValueError unless torch tensor `t` lives on CUDA device `device`
    (the plan's): the kernels run on the plan's device, so a pointer into host
    memory or into another GPU's memory must never reach them."""
    d = t.get_device()
    if d != device:
        where = "host memory" if d < 0 else f"cuda:{d}"
        raise ValueError(f"{what} is in {where}; the plan is on cuda:{device}")


_RAW_STREAM = None


def _stream_of(x):
    """Raw handle of the current CUDA stream of tensor x's device (torch's
    fast accessor, looked up once)."""
    global _RAW_STREAM
    if _RAW_STREAM is None:
        import torch
        _RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None) or \
            (lambda idx: torch.cuda.current_stream(idx).cuda_stream)
    return _RAW_STREAM(x.get_device())


def _torch_dtypes():
    try:
        import torch
    except ImportError:  # pragma: no cover
        return {}
    return {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
            np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128}


_TORCH_DTYPES = _torch_dtypes()
