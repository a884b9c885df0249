"""The pyapollofft surface on the device: FftPlan1D/2D/3D, numpy arrays, torch
tensors (CUDA and CPU) and DLPack producers, and the NUFFT names.

Same names, argument meaning and error behaviour as apollo-python
(crates/apollo-python/src/lib.rs:108-452 plan classes, 453-752 functions,
753-960 NUFFT).  Results against the oracle's f64 plans (FftPlan1D/2D/3D
restated) at 1e-12, f32 at 1e-5; the exact NUFFT sums against numpy direct
sums at 1e-11 (the phase is evaluated in a different order); the fast NUFFT
forms against the CPU restatement of apollo-nufft's plans at 1e-12.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


class DLPackOnly:
    """A DLPack producer that is neither numpy nor torch (stands in for CuPy)."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None):
        return self._t.__dlpack__()

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


@pytest.mark.parametrize("rank,shape", [(1, (60,)), (2, (12, 20)), (3, (6, 8, 10))])
def test_plan_classes_match_the_oracle(afc, oracle, cuda, rank, shape):
    rng = np.random.default_rng(rank)
    cls = {1: afc.FftPlan1D, 2: afc.FftPlan2D, 3: afc.FftPlan3D}[rank]
    plan = cls(*shape)
    x = rng.standard_normal(shape)
    ref = oracle.fft3d(x.reshape((1,) * (3 - rank) + shape).astype(np.complex128)).reshape(shape)
    y = plan.fft(x)
    assert y.dtype == np.complex128 and y.shape == shape
    assert rel_l2(y, ref) < 1e-12
    assert rel_l2(plan.ifft(y), x) < 1e-12
    z = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    zref = oracle.fft3d(z.reshape((1,) * (3 - rank) + shape)).reshape(shape)
    assert rel_l2(plan.fft_complex(z), zref) < 1e-12
    assert rel_l2(plan.ifft_complex(zref), z) < 1e-12
    if rank == 3:
        assert rel_l2(plan.rfft(x), ref) < 1e-12
        assert rel_l2(plan.irfft(ref), x) < 1e-12
    # low precision plans take float32 / complex64 storage
    p32 = cls(*shape, precision="low_precision")
    y32 = p32.fft(x.astype(np.float32))
    assert y32.dtype == np.complex64 and rel_l2(y32, ref) < 1e-5
    # the reference's validation
    with pytest.raises(ValueError, match="shape mismatch"):
        plan.fft(np.zeros(tuple(d + 1 for d in shape)))
    with pytest.raises(ValueError, match="precision `high_accuracy` expects float64"):
        plan.fft(x.astype(np.float32))
    with pytest.raises(ValueError, match="precision `low_precision` expects float32"):
        p32.fft(x)
    with pytest.raises(ValueError, match="unsupported precision"):
        cls(*shape, precision="quad")
    with pytest.raises(ValueError, match="must be > 0"):
        cls(*((0,) + shape[1:]))


def test_functions_on_cuda_tensors(afc, oracle, cuda):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((6, 8, 10))
    ref = oracle.fft3d(x.astype(np.complex128))
    xt = torch.from_numpy(x).to(cuda)
    y = afc.fft3(xt)
    assert isinstance(y, torch.Tensor) and y.is_cuda and y.dtype == torch.complex128
    assert rel_l2(y.cpu().numpy(), ref) < 1e-12
    back = afc.ifft3(y)
    assert back.is_cuda and back.dtype == torch.float64 and rel_l2(back.cpu().numpy(), x) < 1e-12
    assert rel_l2(afc.rfft3(xt).cpu().numpy(), ref) < 1e-12
    assert rel_l2(afc.irfft3(y, 10).cpu().numpy(), x) < 1e-12
    z = torch.from_numpy(ref).to(cuda)
    assert rel_l2(afc.ifft_complex3(z).cpu().numpy(), x.astype(np.complex128)) < 1e-12
    s = torch.linspace(0.0, 1.0, 16, dtype=torch.float32, device=cuda)
    sp = afc.fft1(s, precision="low_precision")
    assert sp.dtype == torch.complex64 and sp.is_cuda
    assert rel_l2(afc.ifft1(sp, precision="low_precision").cpu().numpy(), s.cpu().numpy()) < 1e-6
    m = afc.fft2(torch.ones((4, 4), dtype=torch.float32, device=cuda), precision="mixed_precision")
    assert m.dtype == torch.complex64 and abs(m[0, 0].item() - 16) < 1e-2
    with pytest.raises(ValueError, match="C-contiguous"):
        afc.fft2(torch.zeros((8, 8), dtype=torch.float64, device=cuda)[:, ::2])
    with pytest.raises(ValueError, match="expects a 3-dimensional"):
        afc.fft3(torch.zeros((4, 4), dtype=torch.float64, device=cuda))


def test_cpu_tensors_and_dlpack_producers(afc, oracle, cuda):
    rng = np.random.default_rng(6)
    x = rng.standard_normal((5, 7))
    ref = oracle.fft2d(x.astype(np.complex128))
    y = afc.fft2(torch.from_numpy(x))
    assert isinstance(y, torch.Tensor) and not y.is_cuda
    assert rel_l2(y.numpy(), ref) < 1e-12
    d = afc.fft2(DLPackOnly(torch.from_numpy(x).to(cuda)))
    assert isinstance(d, torch.Tensor) and d.is_cuda
    assert rel_l2(d.cpu().numpy(), ref) < 1e-12
    z = afc.fft_complex2(DLPackOnly(torch.from_numpy(ref).to(cuda)))
    assert rel_l2(z.cpu().numpy(), oracle.fft2d(ref)) < 1e-12


def test_nufft_exact_names(afc, cuda):
    from oracle import nufft as N
    rng = np.random.default_rng(7)
    n, dx, m = 48, 0.125, 300
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, m)
    val = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y1 = afc.nufft_type1_1d(pos, val, dx)
    assert isinstance(y1, np.ndarray) and y1.shape == (m,)  # n_out defaults to len(values)
    assert rel_l2(y1, N.exact1_1d(pos, val, m, m * dx)) < 1e-11
    y1n = afc.nufft_type1_1d(pos, val, dx, n_out=n)
    assert rel_l2(y1n, N.exact1_1d(pos, val, n, L)) < 1e-11
    y2 = afc.nufft_type2_1d(coeffs, pos, dx)
    assert rel_l2(y2, N.exact2_1d(coeffs, pos, n, L)) < 1e-11
    shape, sp = (6, 5, 4), (0.25, 0.5, 0.2)
    pos3 = np.stack([rng.uniform(0, s * k, 200) for s, k in zip(sp, shape)], -1)
    val3 = rng.standard_normal(200) + 1j * rng.standard_normal(200)
    y3 = afc.nufft_type1_3d(pos3, val3, *shape, *sp)
    assert y3.shape == shape
    assert rel_l2(y3, N.exact1_3d(pos3, val3, shape, [a * b for a, b in zip(shape, sp)])) < 1e-11
    # torch CUDA inputs stay on the device
    yt = afc.nufft_type2_1d(torch.from_numpy(coeffs).to(cuda), torch.from_numpy(pos).to(cuda), dx)
    assert yt.is_cuda and rel_l2(yt.cpu().numpy(), y2) < 1e-14
    # the reference's validation
    with pytest.raises(ValueError, match=r"positions must have shape \(n_samples, 3\)"):
        afc.nufft_type1_3d(pos3[:, :2].copy(), val3, *shape, *sp)
    with pytest.raises(ValueError, match="positions/value length mismatch"):
        afc.nufft_type1_3d(pos3, val3[:10], *shape, *sp)
    with pytest.raises(ValueError, match="must be C-contiguous"):
        afc.nufft_type1_1d(np.zeros(8)[::2], val[:4], dx)
    with pytest.raises(ValueError, match="must be finite and > 0"):
        afc.nufft_type2_1d(coeffs, pos, -1.0)


def test_nufft_fast_names(afc, oracle, cuda):
    from oracle import nufft as N
    rng = np.random.default_rng(8)
    n, dx, m = 32, 0.25, 120
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, m)
    val = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = N.RefPlan(n, dx, 2, 6)
    assert rel_l2(afc.nufft_type1_1d_fast(pos, val, dx, n_out=n), ref.type1(pos, val, oracle)) < 1e-12
    assert rel_l2(afc.nufft_type2_1d_fast(coeffs, pos, dx), ref.type2(coeffs, pos, oracle)) < 1e-12
    shape, sp = (8, 6, 5), (0.25, 0.5, 0.2)
    pos3 = np.stack([rng.uniform(0, s * k, 60) for s, k in zip(sp, shape)], -1)
    val3 = rng.standard_normal(60) + 1j * rng.standard_normal(60)
    ref3 = N.RefPlan3(shape, sp, 2, 6)
    assert rel_l2(afc.nufft_type1_3d_fast(pos3, val3, *shape, *sp), ref3.type1(pos3, val3, oracle)) < 1e-12
    # and close to the exact sums (the Kaiser-Bessel error of width 6)
    assert rel_l2(afc.nufft_type1_1d_fast(pos, val, dx, n_out=n), afc.nufft_type1_1d(pos, val, dx, n_out=n)) < 1e-6
