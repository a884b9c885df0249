"""apollofft_b200 -- B200 (sm_100a) backend for apollo-fft's dense FFT plans.

The transforms run in hand-written CUDA kernels behind the C ABI declared in
include/apollofft_cuda.h (libapollofft_cuda.so, built in-tree by
`python -m apollofft_b200.build`).  Python exposes:

* `CudaPlan` -- device plans on torch tensors / host numpy buffers;
* the `pyapollofft` function names (fft1/2/3, ifft1/2/3, rfft3, irfft3,
  fft_complex1/2/3, FftPlan1D/2D/3D, nufft_type1/2_1d[_fast],
  nufft_type1_3d[_fast], backend_capabilities ...) on numpy arrays, torch
  tensors and DLPack producers;
* `autograd` -- torch.autograd Functions with the adjoint-kernel backward.
"""
from . import _lib
from ._lib import AfcError, capabilities, kernel_launch_count, length_info, pfa_perm, rader_maps
from .api import (
    FftPlan1D, FftPlan2D, FftPlan3D, available_backends, backend_capabilities, fft1, fft2, fft3,
    fft_complex1, fft_complex2, fft_complex3, fftfreq, fftshift, ifft1, ifft2, ifft3, ifft_complex1,
    ifft_complex2, ifft_complex3, ifftshift, irfft3, nufft_type1_1d, nufft_type1_1d_fast, nufft_type1_3d,
    nufft_type1_3d_fast, nufft_type2_1d, nufft_type2_1d_fast, rfft3, rfftfreq,
)
from .batch import BatchPlan
from .plan import CudaPlan

__all__ = [
    "AfcError", "BatchPlan", "CudaPlan", "FftPlan1D", "FftPlan2D", "FftPlan3D", "available_backends",
    "backend_capabilities", "capabilities", "fft1", "fft2", "fft3", "fft_complex1", "fft_complex2",
    "fft_complex3", "fftfreq", "fftshift", "ifft1", "ifft2", "ifft3", "ifft_complex1", "ifft_complex2",
    "ifft_complex3", "ifftshift", "irfft3", "kernel_launch_count", "length_info", "nufft_type1_1d",
    "nufft_type1_1d_fast", "nufft_type1_3d", "nufft_type1_3d_fast", "nufft_type2_1d", "nufft_type2_1d_fast",
    "pfa_perm", "rader_maps", "rfft3", "rfftfreq",
]

# Every entry point loads libapollofft_cuda.so through _lib.lib(), which raises
# ImportError when it has not been built: there is no CPU fallback.
