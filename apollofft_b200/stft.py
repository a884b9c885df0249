"""Short-time Fourier transform frames on the device (apollo-stft's StftPlan).

`StftPlan(frame_len, hop_len)` mirrors apollo-stft's plan
(crates/apollo-stft/src/application/execution/plan/stft/dimension_1d.rs):
validation (`frame_len > 0`, `0 < hop_len <= frame_len`), the symmetric Hann
analysis window of kernel/hann.rs:10-16, frames centred at m * hop_len, and
`frame_count(signal_len) = 1 + ceil(signal_len / hop_len)` (0 for a signal
shorter than a frame).  `forward` gathers and windows every frame inside the
FFT kernel's load (`afc_stft_forward`) instead of copying each frame to a host
slice and transforming it alone.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib as L
from .plan import CudaPlan, require_device


class StftError(ValueError):
    """Invalid STFT parameters (the reference's StftError variants)."""


def hann_window(n: int) -> np.ndarray:
    """Symmetric Hann window 0.5 - 0.5 cos(2 pi i / (n - 1)); [1] for n = 1."""
    if n == 1:
        return np.ones(1)
    i = np.arange(n, dtype=np.float64)
    return 0.5 - 0.5 * np.cos(2.0 * math.pi * i / (n - 1))


class StftPlan:
    """Reusable STFT analysis plan on one CUDA device (f64 or f32)."""

    def __init__(self, frame_len: int, hop_len: int, precision: str = "f64", device: int = 0):
        if frame_len <= 0:
            raise StftError("frame length must be positive")
        if hop_len <= 0:
            raise StftError("hop size must be positive")
        if hop_len > frame_len:
            raise StftError("hop size exceeds frame length")
        if precision not in ("f64", "f32"):
            raise StftError(f"unsupported precision `{precision}`; expected f64 or f32")
        self.frame_len = int(frame_len)
        self.hop_len = int(hop_len)
        self.precision = precision
        self.device = int(device)
        self.plan = CudaPlan([self.frame_len], precision=precision, device=self.device)
        self.window = hann_window(self.frame_len)
        self._win_dev = None

    def spectrum_len(self) -> int:
        return self.frame_len

    def frame_count(self, signal_len: int) -> int:
        n = ctypes.c_int64()
        L.check(L.lib().afc_stft_frame_count(self.frame_len, self.hop_len, int(signal_len), ctypes.byref(n)),
                "stft frame count")
        return n.value

    def _real_dtype(self):
        import torch
        return torch.float64 if self.precision == "f64" else torch.float32

    def forward(self, signal, window=None, out=None, stream=None):
        """signal: 1D real torch tensor on the plan's device.  Returns a
        (frames, frame_len) complex tensor (the reference's flat
        frames x spectrum_len array, reshaped)."""
        import torch
        rdt = self._real_dtype()
        if signal.dtype != rdt or signal.dim() != 1 or not signal.is_contiguous() or not signal.is_cuda:
            raise ValueError(f"expected a contiguous 1D {rdt} signal")
        require_device(signal, self.device, "signal")
        if signal.numel() < self.frame_len:
            raise StftError("input signal shorter than frame length")
        if window is None:
            if self._win_dev is None:
                self._win_dev = torch.from_numpy(self.window).to(device=signal.device, dtype=rdt)
            win = self._win_dev
        else:
            win = torch.as_tensor(window, dtype=rdt, device=signal.device).contiguous()
            if win.numel() != self.frame_len:
                raise StftError("window length does not match frame length")
        frames = self.frame_count(signal.numel())
        cdt = torch.complex128 if rdt == torch.float64 else torch.complex64
        if out is None:
            out = torch.empty((frames, self.frame_len), dtype=cdt, device=signal.device)
        if out.dtype != cdt or not out.is_contiguous() or not out.is_cuda:
            raise ValueError("output buffer does not match the plan")
        require_device(out, self.device, "output")
        st = stream if stream is not None else torch.cuda.current_stream(signal.device).cuda_stream
        L.check(L.lib().afc_stft_forward(self.plan._h, signal.data_ptr(), signal.numel(), win.data_ptr(),
                                         self.hop_len, out.data_ptr(), out.numel(), st), "stft forward")
        return out

    def inverse(self, spectrum, signal_len: int, window=None, out=None, stream=None):
        """Weighted overlap-add inverse (the reference's StftPlan::inverse):
        spectrum (frames, frame_len) complex -> signal_len reals."""
        import torch
        rdt = self._real_dtype()
        cdt = torch.complex128 if rdt == torch.float64 else torch.complex64
        if spectrum.dtype != cdt or not spectrum.is_contiguous() or not spectrum.is_cuda:
            raise ValueError(f"expected a contiguous {cdt} spectrum")
        require_device(spectrum, self.device, "spectrum")
        if signal_len < self.frame_len:
            raise StftError("input signal shorter than frame length")
        frames = self.frame_count(signal_len)
        if spectrum.numel() != frames * self.frame_len:
            raise StftError("spectrum length does not match the frame count")
        if window is None:
            if self._win_dev is None:
                self._win_dev = torch.from_numpy(self.window).to(device=spectrum.device, dtype=rdt)
            win = self._win_dev
        else:
            win = torch.as_tensor(window, dtype=rdt, device=spectrum.device).contiguous()
            if win.numel() != self.frame_len:
                raise StftError("window length does not match frame length")
        nbytes = ctypes.c_size_t()
        L.check(L.lib().afc_stft_inverse_workspace(self.plan._h, self.hop_len, int(signal_len), ctypes.byref(nbytes)),
                "stft inverse workspace")
        ws = torch.empty(max(nbytes.value // (8 if rdt == torch.float64 else 4), 1), dtype=rdt, device=spectrum.device)
        if out is None:
            out = torch.empty(int(signal_len), dtype=rdt, device=spectrum.device)
        if out.dtype != rdt or not out.is_contiguous() or out.numel() != int(signal_len) or not out.is_cuda:
            raise ValueError("output buffer does not match the signal length")
        require_device(out, self.device, "output")
        st = stream if stream is not None else torch.cuda.current_stream(spectrum.device).cuda_stream
        L.check(L.lib().afc_stft_inverse(self.plan._h, spectrum.data_ptr(), spectrum.numel(), win.data_ptr(),
                                         self.hop_len, out.data_ptr(), int(signal_len), ws.data_ptr(),
                                         nbytes.value, st), "stft inverse")
        return out
