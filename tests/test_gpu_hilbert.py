"""Device analytic signal (afc_hilbert_*, HilbertPlan) against apollo-hilbert's
algorithm restated on the oracle (infrastructure/kernel/direct.rs:85-143:
forward FFT, the analytic mask, normalized inverse FFT, real part reset to
the input) and against the quadrature of known signals."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def analytic_mask(n):  # apply_analytic_mask (direct.rs:130-143)
    k = np.arange(n)
    m = np.where(k < (n + 1) // 2, 2.0, 0.0)
    m[0] = 1.0
    if n % 2 == 0:
        m[n // 2] = 1.0
    return m


def ref_analytic(x, oracle):
    """analytic_signal_into per lane: oracle forward, mask, oracle inverse, re = x."""
    z = oracle.fft1d(x.astype(np.complex128))
    z = oracle.fft1d(z * analytic_mask(x.shape[-1]), inverse=True)
    return x + 1j * z.imag, z


@pytest.mark.parametrize("n,batch", [(2, 3), (3, 5), (8, 1), (1000, 4), (1001, 2), (1024, 64), (2187, 3), (4096, 16)])
def test_analytic_signal_f64_vs_reference(afc, oracle, cuda, n, batch):
    from apollofft_b200.hilbert import HilbertPlan
    x = np.random.default_rng(n + batch).standard_normal((batch, n))
    plan = HilbertPlan(n)
    z = plan.analytic_signal(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, raw = ref_analytic(x, oracle)
    # errors relative to the signal's norm (the quadrature of n = 2 is exactly zero)
    assert np.linalg.norm(z.imag - ref.imag) / np.linalg.norm(x) < 1e-12
    assert rel_l2(z, raw) < 1e-12           # the transform itself, real part included
    assert np.abs(z.real - x).max() < 1e-12 * max(1.0, np.abs(x).max())


@pytest.mark.parametrize("n", [1000, 4096])
def test_analytic_signal_f32(afc, oracle, cuda, n):
    from apollofft_b200.hilbert import HilbertPlan
    x = np.random.default_rng(n).standard_normal((8, n))
    plan = HilbertPlan(n, precision="f32")
    z = plan.analytic_signal(torch.from_numpy(x.astype(np.float32)).cuda()).cpu().numpy()
    ref, _ = ref_analytic(x.astype(np.float32).astype(np.float64), oracle)
    assert np.linalg.norm(z.imag - ref.imag) / np.linalg.norm(x) < 1e-5


def test_quadrature_of_cosine_and_observables(afc, cuda):
    """H{cos} = sin for a whole number of periods; envelope 1, phase linear."""
    from apollofft_b200.hilbert import HilbertPlan
    n, f = 1024, 17
    t = np.arange(n)
    x = np.cos(2 * np.pi * f * t / n)
    plan = HilbertPlan(n)
    xt = torch.from_numpy(x).cuda()
    h = plan.transform(xt).cpu().numpy()
    assert np.abs(h - np.sin(2 * np.pi * f * t / n)).max() < 1e-12
    env = plan.envelope(xt).cpu().numpy()
    assert np.abs(env - 1.0).max() < 1e-12
    ph = plan.phase(xt).cpu().numpy()
    want = np.angle(np.exp(2j * np.pi * f * t / n))
    assert np.abs(np.angle(np.exp(1j * (ph - want)))).max() < 1e-11


def test_length_one_validation_and_unsupported(afc, cuda):
    from apollofft_b200.hilbert import HilbertPlan
    x = torch.tensor([[2.5], [-1.0]], dtype=torch.float64, device="cuda")
    z = HilbertPlan(1).analytic_signal(x).cpu().numpy()
    assert np.array_equal(z, np.array([[2.5 + 0j], [-1.0 + 0j]]))
    with pytest.raises(ValueError):
        HilbertPlan(0)
    with pytest.raises(ValueError):
        HilbertPlan(16, precision="f16")
    with pytest.raises(Exception):
        HilbertPlan(1009)  # prime: no single-tile plan
    plan = HilbertPlan(64)
    with pytest.raises(ValueError):
        plan.analytic_signal(torch.zeros(63, dtype=torch.float64, device="cuda"))
