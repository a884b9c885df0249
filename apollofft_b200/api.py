"""`pyapollofft`-compatible functions executed by the CUDA library.

Same names, argument meaning and error behaviour as the reference's Python
module (crates/apollo-python/src/lib.rs:66-752,1005-1076 and
python/pyapollofft/__init__.py): numpy arrays in, numpy arrays out, precision
strings `high_accuracy` (f64), `low_precision` (f32) and `mixed_precision`
(f16 storage computed in f32), C-contiguity and dtype checks raising
ValueError with the reference's messages.  `fft1/2/3` take real input and
return the full complex spectrum (RealFftData contract, real_storage.rs:186-303);
`ifft1/2/3` return the real part of the normalized inverse; `rfft3` is the
full-spectrum transform and `irfft3` rejects half spectra, as the reference does.
All arithmetic runs on the GPU through include/apollofft_cuda.h.

Inputs may also be torch tensors or any DLPack producer (CuPy, JAX ...): a
CUDA tensor is transformed where it lives, without a copy, and the result is a
torch tensor on the same device; a torch CPU tensor goes the host route and
comes back as a torch CPU tensor.  The NUFFT names (`nufft_type1_1d`,
`nufft_type2_1d`, `nufft_type1_3d` and their `_fast` forms) follow
apollo-python's bindings (lib.rs:753-960): the plain forms are the exact
direct sums, the `_fast` forms the Kaiser-Bessel plans (oversampling 2).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .plan import CudaPlan

_PRECISIONS = ("high_accuracy", "low_precision", "mixed_precision")


def _parse_precision(precision):
    p = precision or "high_accuracy"
    if p not in _PRECISIONS:
        raise ValueError(f"unsupported precision `{p}`; expected `high_accuracy`, `low_precision`, or `mixed_precision`")
    return p


def _require_contiguous(x: np.ndarray, name: str):
    if not x.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")


def _require_f64(profile, name):
    if profile != "high_accuracy":
        raise ValueError(f"{name} received float64/complex128 input but precision `{profile}` expects float32/complex64 storage")


def _require_f32(profile, name):
    if profile == "high_accuracy":
        raise ValueError(f"{name} received float32/complex64 input but precision `{profile}` expects float64/complex128 storage")


def _to_f16_storage(a: np.ndarray) -> np.ndarray:
    """Round to binary16 storage (mixed_precision keeps f16 data, f32 compute)."""
    if np.iscomplexobj(a):
        return (a.real.astype(np.float16).astype(np.float32) + 1j * a.imag.astype(np.float16).astype(np.float32)).astype(np.complex64)
    return a.astype(np.float16).astype(np.float32)


def _plan(shape, prec, kind, device=0):
    return CudaPlan(list(shape), precision="f64" if prec == "f64" else "f32", kind=kind, device=device)


# ── input kinds: numpy arrays, torch tensors (CUDA or CPU), DLPack producers ──

def _torch():
    import torch
    return torch


def _as_device_tensor(x):
    """A CUDA torch tensor for x (zero copy) when x lives on a CUDA device,
    else None.  torch tensors are used as they are; other objects exposing
    __dlpack__ on a CUDA device go through torch.from_dlpack."""
    if isinstance(x, np.ndarray):
        return None
    mod = type(x).__module__.split(".")[0]
    if mod == "torch":
        return x if x.is_cuda else None
    dl = getattr(x, "__dlpack_device__", None)
    if dl is not None:
        try:
            dev_type = int(dl()[0])
        except Exception:  # not a DLPack producer after all
            return None
        if dev_type == 2:  # kDLCUDA
            return _torch().from_dlpack(x)
    return None


def _is_cpu_tensor(x):
    return type(x).__module__.split(".")[0] == "torch" and not x.is_cuda


def _host_array(x):
    return x.numpy() if _is_cpu_tensor(x) else np.asarray(x)


def _wrap_host(result, like):
    return _torch().from_numpy(np.ascontiguousarray(result)) if _is_cpu_tensor(like) else result


def _require_contiguous_t(t, name: str):
    if not t.is_contiguous():
        raise ValueError(f"{name} must be C-contiguous")


def _f16_storage_t(t):
    """binary16 storage of a float32 / complex64 tensor, back in float32 storage."""
    torch = _torch()
    if t.is_complex():
        return torch.complex(t.real.to(torch.float16).to(torch.float32), t.imag.to(torch.float16).to(torch.float32))
    return t.to(torch.float16).to(torch.float32)


def _real_forward_dev(t, ndim: int, name: str, profile):
    torch = _torch()
    if t.dim() != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional array, got {t.dim()} dimensions")
    dev = t.device.index or 0
    if t.dtype == torch.float64:
        _require_contiguous_t(t, f"{name} input")
        _require_f64(profile, name)
        return _plan(t.shape, "f64", "r2c_full", dev).execute(t).reshape(t.shape)
    if t.dtype != torch.float32:
        raise ValueError(f"{name} expects float64 or float32 input, got {t.dtype}")
    _require_contiguous_t(t, f"{name} input")
    if profile == "mixed_precision":
        y = _plan(t.shape, "f32", "r2c_full", dev).execute(_f16_storage_t(t).contiguous())
        return _f16_storage_t(y).reshape(t.shape)
    _require_f32(profile, name)
    return _plan(t.shape, "f32", "r2c_full", dev).execute(t).reshape(t.shape)


def _real_inverse_dev(t, ndim: int, name: str, profile):
    torch = _torch()
    if t.dim() != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional array, got {t.dim()} dimensions")
    dev = t.device.index or 0
    if t.dtype == torch.complex128:
        _require_contiguous_t(t, f"{name} input")
        _require_f64(profile, name)
        return _plan(t.shape, "f64", "r2c_full", dev).execute(t, inverse=True).reshape(t.shape)
    if t.dtype != torch.complex64:
        raise ValueError(f"{name} expects complex128 or complex64 input, got {t.dtype}")
    _require_contiguous_t(t, f"{name} input")
    if profile == "mixed_precision":
        y = _plan(t.shape, "f32", "r2c_full", dev).execute(_f16_storage_t(t).contiguous(), inverse=True)
        return _f16_storage_t(y).reshape(t.shape)
    _require_f32(profile, name)
    return _plan(t.shape, "f32", "r2c_full", dev).execute(t, inverse=True).reshape(t.shape)


def _real_forward(x, ndim: int, name: str, precision):
    profile = _parse_precision(precision)
    t = _as_device_tensor(x)
    if t is not None:
        return _real_forward_dev(t, ndim, name, profile)
    if _is_cpu_tensor(x):
        return _wrap_host(_real_forward(x.numpy(), ndim, name, profile), x)
    x = np.asarray(x)
    if x.ndim != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional array, got {x.ndim} dimensions")
    if x.dtype == np.float64:
        _require_contiguous(x, f"{name} input")
        _require_f64(profile, name)
        p = _plan(x.shape, "f64", "r2c_full")
        return p.execute_host(x).reshape(x.shape)
    if x.dtype != np.float32:
        raise ValueError(f"{name} expects float64 or float32 input, got {x.dtype}")
    _require_contiguous(x, f"{name} input")
    if profile == "mixed_precision":
        p = _plan(x.shape, "f32", "r2c_full")
        return _to_f16_storage(p.execute_host(_to_f16_storage(x)).reshape(x.shape))
    _require_f32(profile, name)
    p = _plan(x.shape, "f32", "r2c_full")
    return p.execute_host(x).reshape(x.shape)


def _real_inverse(X, ndim: int, name: str, precision):
    profile = _parse_precision(precision)
    t = _as_device_tensor(X)
    if t is not None:
        return _real_inverse_dev(t, ndim, name, profile)
    if _is_cpu_tensor(X):
        return _wrap_host(_real_inverse(X.numpy(), ndim, name, profile), X)
    X = np.asarray(X)
    if X.ndim != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional array, got {X.ndim} dimensions")
    if X.dtype == np.complex128:
        _require_contiguous(X, f"{name} input")
        _require_f64(profile, name)
        p = _plan(X.shape, "f64", "r2c_full")
        return p.execute_host(X, inverse=True).reshape(X.shape)
    if X.dtype != np.complex64:
        raise ValueError(f"{name} expects complex128 or complex64 input, got {X.dtype}")
    _require_contiguous(X, f"{name} input")
    if profile == "mixed_precision":
        p = _plan(X.shape, "f32", "r2c_full")
        return _to_f16_storage(p.execute_host(_to_f16_storage(X), inverse=True).reshape(X.shape))
    _require_f32(profile, name)
    p = _plan(X.shape, "f32", "r2c_full")
    return p.execute_host(X, inverse=True).reshape(X.shape)


def fft1(input, precision=None):
    """Forward 1D FFT of a real signal (full complex spectrum)."""
    return _real_forward(input, 1, "fft1", precision)


def ifft1(input, precision=None):
    """Inverse 1D FFT of a complex spectrum; returns the real part."""
    return _real_inverse(input, 1, "ifft1", precision)


def fft2(input, precision=None):
    return _real_forward(input, 2, "fft2", precision)


def ifft2(input, precision=None):
    return _real_inverse(input, 2, "ifft2", precision)


def fft3(input, precision=None):
    return _real_forward(input, 3, "fft3", precision)


def ifft3(input, precision=None):
    return _real_inverse(input, 3, "ifft3", precision)


def rfft3(input):
    """Reference contract: the full complex spectrum of the same shape (f64)."""
    t = _as_device_tensor(input)
    if t is not None:
        return _real_forward(t.to(_torch().float64).contiguous(), 3, "rfft3", None)
    if _is_cpu_tensor(input):
        return _wrap_host(rfft3(input.numpy()), input)
    x = np.asarray(input, dtype=np.float64) if np.asarray(input).dtype != np.float64 else np.asarray(input)
    return _real_forward(x, 3, "rfft3", None)


def irfft3(input, n):
    """Inverse of rfft3; rejects half-spectrum input (apollo-python/src/lib.rs:740-746)."""
    t = _as_device_tensor(input)
    X = t if t is not None else _host_array(input)
    if X.ndim != 3 or X.shape[-1] != n:
        raise ValueError(f"inconsistent spectrum shape {tuple(X.shape)} for last-axis length {n}: expected the full spectrum")
    if t is not None:
        return _real_inverse(t.to(_torch().complex128).contiguous(), 3, "irfft3", None)
    return _wrap_host(_real_inverse(X.astype(np.complex128, copy=False), 3, "irfft3", None), input)


def _complex(x, ndim: int, name: str, inverse: bool):
    t = _as_device_tensor(x)
    if t is not None:
        if t.dtype != _torch().complex128 or t.dim() != ndim:
            raise ValueError(f"{name} expects a {ndim}-dimensional complex128 array")
        _require_contiguous_t(t, f"{name} input")
        return _plan(t.shape, "f64", "c2c", t.device.index or 0).execute(t, inverse=inverse).reshape(t.shape)
    xa = _host_array(x)
    if xa.dtype != np.complex128 or xa.ndim != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional complex128 array")
    _require_contiguous(xa, f"{name} input")
    p = _plan(xa.shape, "f64", "c2c")
    return _wrap_host(p.execute_host(xa, inverse=inverse).reshape(xa.shape), x)


def fft_complex1(input):
    return _complex(input, 1, "fft_complex1", False)


def ifft_complex1(input):
    return _complex(input, 1, "ifft_complex1", True)


def fft_complex2(input):
    return _complex(input, 2, "fft_complex2", False)


def ifft_complex2(input):
    return _complex(input, 2, "ifft_complex2", True)


def fft_complex3(input):
    return _complex(input, 3, "fft_complex3", False)


def ifft_complex3(input):
    return _complex(input, 3, "ifft_complex3", True)


class _PlanBase:
    _rank = 1

    def __init__(self, *dims, precision=None):
        if len(dims) != self._rank:
            raise ValueError(f"expected {self._rank} dimensions")
        for name, d in zip(("nx", "ny", "nz") if self._rank > 1 else ("n",), dims):
            if int(d) <= 0:
                raise ValueError(f"validation failed for `{name}`: `{d}` violates `must be > 0`")
        self.shape = tuple(int(d) for d in dims)
        self.profile = _parse_precision(precision)

    def _check_shape(self, x):
        shape = tuple(x.shape) if hasattr(x, "shape") else np.asarray(x).shape
        if shape != self.shape:
            raise ValueError(f"shape mismatch: expected {self.shape}, got {shape}")

    def fft(self, input):
        self._check_shape(input)
        return _real_forward(input, self._rank, "fft", self.profile)

    def ifft(self, input):
        self._check_shape(input)
        return _real_inverse(input, self._rank, "ifft", self.profile)

    def fft_complex(self, input):
        return _complex(input, self._rank, "fft_complex", False)

    def ifft_complex(self, input):
        return _complex(input, self._rank, "ifft_complex", True)


class FftPlan1D(_PlanBase):
    _rank = 1


class FftPlan2D(_PlanBase):
    _rank = 2


class FftPlan3D(_PlanBase):
    _rank = 3

    def rfft(self, input):
        return rfft3(input)

    def irfft(self, input):
        return irfft3(input, self.shape[-1])


def available_backends():
    return ["cuda"]


def backend_capabilities():
    c = L.capabilities()
    entry = {
        "available": c["device_count"] > 0,
        "supports_1d": bool(c["supports_1d"]), "supports_2d": bool(c["supports_2d"]),
        "supports_3d": bool(c["supports_3d"]), "supports_real_to_complex": bool(c["supports_real_to_complex"]),
        "supports_mixed_precision": bool(c["supports_mixed_precision"]),
        "default_precision": "high_accuracy",
        "supported_precisions": list(_PRECISIONS),
        "device_count": c["device_count"], "sm_count": c["sm_count"],
        "compute_capability": f"{c['cc_major']}.{c['cc_minor']}",
    }
    return {"cuda": entry, "cpu": {"available": False, "note": "no CPU path in this backend"},
            "wgpu": {"available": False, "note": "graphics API unavailable"}}


def fftfreq(n, d=1.0):
    """Sample frequencies (utilities/freq.rs:26)."""
    return np.fft.fftfreq(n, d)


def rfftfreq(n, d=1.0):
    return np.fft.rfftfreq(n, d)


def fftshift(x):
    return np.fft.fftshift(x)


def ifftshift(x):
    return np.fft.ifftshift(x)


# ── NUFFT (apollo-python lib.rs:753-960) ─────────────────────────────────────

DEFAULT_NUFFT_KERNEL_WIDTH = 6


def _nufft_inputs(name, **arrays):
    """Each argument as a contiguous CUDA tensor of its required dtype (the
    device of the first CUDA tensor given, else cuda:0).  Returns (tensors,
    host) with host True when every input came from host memory."""
    torch = _torch()
    want = {"positions": torch.float64, "values": torch.complex128, "fourier_coeffs": torch.complex128}
    dev = None
    for v in arrays.values():
        t = _as_device_tensor(v)
        if t is not None:
            dev = t.device
            break
    host = dev is None
    dev = dev or torch.device("cuda", 0)
    out = {}
    for key, v in arrays.items():
        t = _as_device_tensor(v)
        if t is None:
            a = _host_array(v)
            if not a.flags.c_contiguous:
                raise ValueError(f"{name} {key} must be C-contiguous")
            if a.dtype != np.dtype(np.float64 if key == "positions" else np.complex128):
                raise TypeError(f"{name} {key} must be {'float64' if key == 'positions' else 'complex128'}")
            t = torch.from_numpy(a).to(dev)
        else:
            if not t.is_contiguous():
                raise ValueError(f"{name} {key} must be C-contiguous")
            if t.dtype != want[key]:
                raise TypeError(f"{name} {key} must be {'float64' if key == 'positions' else 'complex128'}")
            if t.device != dev:
                raise ValueError(f"{name} {key} is on {t.device}, other inputs on {dev}")
        out[key] = t
    return out, host


def _nufft_out(t, host, like):
    if not host:
        return t
    a = t.cpu().numpy()
    return _torch().from_numpy(a) if _is_cpu_tensor(like) else a


def _positions3(name, pos, values):
    if pos.dim() != 2 or pos.shape[1] != 3:
        raise ValueError(f"{name} positions must have shape (n_samples, 3)")
    if pos.shape[0] != values.numel():
        raise ValueError(f"{name} positions/value length mismatch")


def nufft_type1_1d(positions, values, dx, n_out=None):
    """Exact direct 1D type-1 NUFFT: out[k] = sum_j v_j exp(-2 pi i k_s x_j / (n dx))."""
    t, host = _nufft_inputs("nufft_type1_1d", positions=positions, values=values)
    p, v = t["positions"], t["values"]
    if p.numel() != v.numel():
        raise ValueError("positions/value length mismatch")
    n = int(n_out) if n_out is not None else v.numel()
    out = _torch().empty(max(n, 0), dtype=_torch().complex128, device=v.device)
    st = _torch().cuda.current_stream(v.device).cuda_stream
    L.check(L.lib().afc_nudft1d_type1(p.data_ptr(), v.data_ptr(), p.numel(), n, float(dx), out.data_ptr(),
                                      v.device.index or 0, st), "nufft_type1_1d")
    return _nufft_out(out, host, values)


def nufft_type2_1d(fourier_coeffs, positions, dx):
    """Exact direct 1D type-2 NUFFT: out[j] = sum_k c_k exp(+2 pi i k_s x_j / (n dx))."""
    t, host = _nufft_inputs("nufft_type2_1d", fourier_coeffs=fourier_coeffs, positions=positions)
    c, p = t["fourier_coeffs"], t["positions"]
    out = _torch().empty(p.numel(), dtype=_torch().complex128, device=c.device)
    st = _torch().cuda.current_stream(c.device).cuda_stream
    L.check(L.lib().afc_nudft1d_type2(c.data_ptr(), c.numel(), p.data_ptr(), p.numel(), float(dx), out.data_ptr(),
                                      c.device.index or 0, st), "nufft_type2_1d")
    return _nufft_out(out, host, positions)


def nufft_type1_3d(positions, values, nx, ny, nz, dx, dy, dz):
    """Exact direct 3D type-1 NUFFT on an (nx, ny, nz) grid."""
    t, host = _nufft_inputs("nufft_type1_3d", positions=positions, values=values)
    p, v = t["positions"], t["values"]
    _positions3("nufft_type1_3d", p, v)
    out = _torch().empty((int(nx), int(ny), int(nz)), dtype=_torch().complex128, device=v.device)
    st = _torch().cuda.current_stream(v.device).cuda_stream
    L.check(L.lib().afc_nudft3d_type1(p.data_ptr(), v.data_ptr(), v.numel(), int(nx), int(ny), int(nz), float(dx),
                                      float(dy), float(dz), out.data_ptr(), v.device.index or 0, st),
            "nufft_type1_3d")
    return _nufft_out(out, host, values)


def nufft_type1_1d_fast(positions, values, dx, n_out=None, kernel_width=DEFAULT_NUFFT_KERNEL_WIDTH):
    """Fast 1D type-1 NUFFT (Kaiser-Bessel spreading, oversampling 2)."""
    from .nufft import NufftPlan1D
    t, host = _nufft_inputs("nufft_type1_1d_fast", positions=positions, values=values)
    p, v = t["positions"], t["values"]
    if p.numel() != v.numel():
        raise ValueError("positions/value length mismatch")
    n = int(n_out) if n_out is not None else v.numel()
    plan = NufftPlan1D(n, float(dx), 2, int(kernel_width), device=v.device.index or 0)
    return _nufft_out(plan.type1(p, v), host, values)


def nufft_type2_1d_fast(fourier_coeffs, positions, dx, kernel_width=DEFAULT_NUFFT_KERNEL_WIDTH):
    """Fast 1D type-2 NUFFT (Kaiser-Bessel interpolation, oversampling 2)."""
    from .nufft import NufftPlan1D
    t, host = _nufft_inputs("nufft_type2_1d_fast", fourier_coeffs=fourier_coeffs, positions=positions)
    c, p = t["fourier_coeffs"], t["positions"]
    plan = NufftPlan1D(c.numel(), float(dx), 2, int(kernel_width), device=c.device.index or 0)
    return _nufft_out(plan.type2(c, p), host, positions)


def nufft_type1_3d_fast(positions, values, nx, ny, nz, dx, dy, dz, kernel_width=DEFAULT_NUFFT_KERNEL_WIDTH):
    """Fast 3D type-1 NUFFT (Kaiser-Bessel spreading, oversampling 2)."""
    from .nufft import NufftPlan3D
    t, host = _nufft_inputs("nufft_type1_3d_fast", positions=positions, values=values)
    p, v = t["positions"], t["values"]
    _positions3("nufft_type1_3d_fast", p, v)
    plan = NufftPlan3D((int(nx), int(ny), int(nz)), (float(dx), float(dy), float(dz)), 2, int(kernel_width),
                       device=v.device.index or 0)
    return _nufft_out(plan.type1(p, v), host, values)
