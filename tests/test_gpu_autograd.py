"""Adjoint kernels and the torch.autograd Functions.

* dot-product identity <A x, y> = <x, A^H y> (real inner product) for every
  plan kind and direction, f64, relative 1e-12;
* torch.autograd.gradcheck on small shapes;
* the spectral loss sum_k |w(k) X(k)|^2 on 2D real images: gradient against the
  reference gradient 2 Re(F^H (|w|^2 X)) built from the f64 oracle plans, and
  against f64 central finite differences on 64 seeded pixels (the loss is
  quadratic, so central differences carry no truncation error; the step keeps
  f64 rounding, about eps * L / h, below 1e-6 of the gradient's scale max|g|).
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def rdot(a, b):
    a = a.reshape(-1)
    b = b.reshape(-1)
    if a.is_complex() or b.is_complex():
        return torch.sum((torch.conj(a.to(torch.complex128)) * b.to(torch.complex128)).real).item()
    return torch.sum(a.double() * b.double()).item()


@pytest.mark.parametrize("kind", ["c2c", "r2c_full", "r2c_half"])
@pytest.mark.parametrize("dims", [[30], [16, 12], [6, 10, 8], [1031], [5, 7, 9]])
@pytest.mark.parametrize("inverse", [False, True])
def test_adjoint_dot_product(afc, cuda, kind, dims, inverse):
    if kind == "r2c_half" and dims[-1] == 1031:
        pytest.skip("half-spectrum plans need a smooth last dimension")
    p = afc.CudaPlan(dims, precision="f64", kind=kind, batch=2)
    ie, oe = p.io_elems(inverse)
    g = torch.Generator(device="cuda").manual_seed(7)

    def rand(n, complex_):
        if complex_:
            return torch.randn(n, dtype=torch.complex128, device=cuda, generator=g)
        return torch.randn(n, dtype=torch.float64, device=cuda, generator=g)

    in_c = kind == "c2c" or inverse
    out_c = kind == "c2c" or not inverse
    x = rand(ie, in_c)
    y = rand(oe, out_c)
    if kind == "r2c_half" and inverse:
        # a C2R input must be a valid half spectrum for the map to be the one
        # whose adjoint we test: make DC / Nyquist bins real
        n = dims[-1]
        h = n // 2 + 1
        xv = x.view(-1, h)
        xv[:, 0] = xv[:, 0].real
        if n % 2 == 0:
            xv[:, -1] = xv[:, -1].real
    ax = p.execute(x, inverse=inverse).reshape(-1)
    aty = p.adjoint(y, inverse=inverse)
    lhs = rdot(y, ax)
    rhs = rdot(aty, x)
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs) + 1e-30), (lhs, rhs)


def test_gradcheck_small(afc, cuda):
    from apollofft_b200 import autograd as AG
    x = torch.randn(2, 6, 10, dtype=torch.float64, device=cuda, requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: AG.rfftn(t, 2, half=False), (x,))
    assert torch.autograd.gradcheck(lambda t: AG.rfftn(t, 2, half=True), (x,))
    z = torch.randn(3, 12, dtype=torch.complex128, device=cuda, requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: AG.fftn(t, 1), (z,))
    assert torch.autograd.gradcheck(lambda t: AG.fftn(t, 1, inverse=True), (z,))
    X = torch.randn(2, 6, 6, dtype=torch.complex128, device=cuda)
    X[..., 0] = X[..., 0].real
    X[..., -1] = X[..., -1].real
    X.requires_grad_(True)
    assert torch.autograd.gradcheck(lambda t: AG.irfftn(t, 10, 2, half=True), (X,))


def radial_weight(n, seed=5):
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n)
    r = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
    a, b = rng.uniform(0.5, 2.0, 2)
    return (a * np.exp(-b * r * 8) + 0.1).astype(np.float64)


def spectral_loss(X, w):
    return torch.sum(torch.abs(w * X) ** 2)


@pytest.mark.parametrize("n,batch,tol", [(64, 2, 1e-5), (2048, 8, 1e-5)])
def test_spectral_loss_gradient_vs_oracle(afc, oracle, cuda, n, batch, tol):
    from apollofft_b200 import autograd as AG
    rng = np.random.default_rng(5)
    img = rng.standard_normal((batch, n, n)).astype(np.float32)
    w = radial_weight(n)
    x = torch.from_numpy(img).to(cuda).requires_grad_(True)
    wt = torch.from_numpy(w).to(cuda).to(torch.float32)
    X = AG.rfft2(x)
    loss = spectral_loss(X, wt)
    loss.backward()
    g = x.grad.double().cpu().numpy()
    # reference gradient from the f64 CPU plans: 2 Re(F^H (|w|^2 X)), F^H = N * inverse
    Xo = oracle.fft2d(img.astype(np.complex128))
    ref = 2.0 * (n * n) * oracle.fft2d((w ** 2) * Xo, inverse=True).real
    assert rel_l2(g, ref) < tol


@pytest.mark.parametrize("n,h", [(64, 1e-6), (2048, 1e-2)])
def test_spectral_loss_finite_differences(afc, cuda, n, h):
    from apollofft_b200 import autograd as AG
    rng = np.random.default_rng(5)
    img = rng.standard_normal((8 if n == 2048 else 2, n, n))
    w = torch.from_numpy(radial_weight(n)).to(cuda)
    x = torch.from_numpy(img).to(cuda).requires_grad_(True)
    loss = spectral_loss(AG.rfft2(x), w)
    loss.backward()
    g = x.grad
    gmax = g.abs().max().item()
    pix = np.random.default_rng(64).integers(0, img.size, 64)
    xd = torch.from_numpy(img).to(cuda).reshape(-1)
    with torch.no_grad():
        for idx in pix:
            old = xd[idx].item()
            xd[idx] = old + h
            lp = spectral_loss(AG.rfft2(xd.reshape(img.shape)), w).item()
            xd[idx] = old - h
            lm = spectral_loss(AG.rfft2(xd.reshape(img.shape)), w).item()
            xd[idx] = old
            fd = (lp - lm) / (2 * h)
            gi = g.reshape(-1)[idx].item()
            assert abs(fd - gi) <= 1e-6 * gmax, (idx, fd, gi)
