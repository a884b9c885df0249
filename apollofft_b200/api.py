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


def _plan(shape, prec, kind):
    return CudaPlan(shape, precision="f64" if prec == "f64" else "f32", kind=kind)


def _real_forward(x, ndim: int, name: str, precision):
    profile = _parse_precision(precision)
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
    """Reference contract: the full complex spectrum of the same shape."""
    x = np.asarray(input, dtype=np.float64) if np.asarray(input).dtype != np.float64 else np.asarray(input)
    return _real_forward(x, 3, "rfft3", None)


def irfft3(input, n):
    """Inverse of rfft3; rejects half-spectrum input (apollo-python/src/lib.rs:740-746)."""
    X = np.asarray(input)
    if X.ndim != 3 or X.shape[-1] != n:
        raise ValueError(f"inconsistent spectrum shape {tuple(X.shape)} for last-axis length {n}: expected the full spectrum")
    return _real_inverse(X.astype(np.complex128, copy=False), 3, "irfft3", None)


def _complex(x, ndim: int, name: str, inverse: bool):
    x = np.asarray(x)
    if x.dtype != np.complex128 or x.ndim != ndim:
        raise ValueError(f"{name} expects a {ndim}-dimensional complex128 array")
    _require_contiguous(x, f"{name} input")
    p = _plan(x.shape, "f64", "c2c")
    return p.execute_host(x, inverse=inverse).reshape(x.shape)


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

    def fft(self, input):
        x = np.asarray(input)
        if x.shape != self.shape:
            raise ValueError(f"shape mismatch: expected {self.shape}, got {x.shape}")
        return _real_forward(x, self._rank, "fft", self.profile)

    def ifft(self, input):
        X = np.asarray(input)
        if X.shape != self.shape:
            raise ValueError(f"shape mismatch: expected {self.shape}, got {X.shape}")
        return _real_inverse(X, self._rank, "ifft", self.profile)

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
