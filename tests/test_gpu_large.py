"""Size-independent properties at the measured workload sizes (the oracle
would take too long there): round trips, linearity, Parseval, and agreement
with the f64 path for f32 at 256^3 and 243x250x343."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


@pytest.mark.parametrize("shape", [(256, 256, 256), (243, 250, 343)])
def test_3d_full_size_properties(afc, cuda, shape):
    g = torch.Generator(device="cuda").manual_seed(2)
    x = torch.randn(shape, dtype=torch.complex128, device=cuda, generator=g)
    p = afc.CudaPlan(list(shape), precision="f64")
    y = p.execute(x)
    # Parseval: sum |X|^2 = N sum |x|^2
    n = x.numel()
    e_x = torch.sum(x.abs() ** 2).item()
    e_y = torch.sum(y.abs() ** 2).item()
    assert abs(e_y / (n * e_x) - 1) < 1e-12
    # round trip
    xb = p.execute(y, inverse=True)
    assert rel(xb, x) < 1e-12
    # against torch.fft (cuFFT) in f64 as an independent check
    assert rel(y, torch.fft.fftn(x)) < 1e-12
    # f32 path vs the f64 result
    p32 = afc.CudaPlan(list(shape), precision="f32")
    y32 = p32.execute(x.to(torch.complex64))
    assert rel(y32.to(torch.complex128), y) < 1e-5
    del y, xb, y32
    torch.cuda.empty_cache()


def test_linearity_4096_batch64(afc, cuda):
    g = torch.Generator(device="cuda").manual_seed(1)
    a = torch.randn(64, 4096, dtype=torch.complex128, device=cuda, generator=g)
    b = torch.randn(64, 4096, dtype=torch.complex128, device=cuda, generator=g)
    p = afc.CudaPlan([4096], precision="f64", batch=64)
    lhs = p.execute(2.5 * a - 1j * b)
    rhs = 2.5 * p.execute(a) - 1j * p.execute(b)
    assert rel(lhs, rhs) < 1e-13
