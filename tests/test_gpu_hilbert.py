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


def _kat_signals():
    """The reference's own known answers (apollo-hilbert verification/mod.rs:11-135)."""
    t16, t32, t64 = np.arange(16), np.arange(32), np.arange(64)
    return {
        "cos16": np.cos(2 * np.pi * t16 / 16),
        "cos3_32": np.cos(2 * np.pi * 3 * t32 / 32),
        "const9": np.full(9, 4.0),
        "alt10": np.array([1.0 if i % 2 == 0 else -1.0 for i in range(10)]),
        "sin3_32": np.sin(2 * np.pi * 3 * t32 / 32),
        "cos5_64": np.cos(2 * np.pi * 5 * t64 / 64),
    }


def test_reference_known_answers(afc, cuda):
    from apollofft_b200.hilbert import HilbertPlan
    s = _kat_signals()

    def z_of(x):
        return HilbertPlan(len(x)).analytic_signal(torch.from_numpy(x).cuda()).cpu().numpy()

    # cosine -> sine quadrature (:11-25)
    assert np.abs(z_of(s["cos16"]).imag - np.sin(2 * np.pi * np.arange(16) / 16)).max() < 1e-11
    # real part kept, unit envelope (:28-46)
    z = z_of(s["cos3_32"])
    assert np.abs(z.real - s["cos3_32"]).max() < 1e-12 and np.abs(np.abs(z) - 1.0).max() < 1e-11
    # constant: zero quadrature, constant envelope (:49-59)
    z = z_of(s["const9"])
    assert np.abs(z.real - 4.0).max() < 1e-12 and np.abs(z.imag).max() < 1e-12
    # even-length Nyquist tone has zero quadrature (:62-72)
    assert np.abs(z_of(s["alt10"]).imag).max() < 1e-12
    # H{H{x}} = -x for a zero-mean tone (:124-137)
    p = HilbertPlan(32)
    h1 = p.transform(torch.from_numpy(s["sin3_32"]).cuda())
    h2 = p.transform(h1).cpu().numpy()
    assert np.abs(h2 + s["sin3_32"]).max() < 1e-10
    # constant instantaneous frequency k / n of a tone (:104-121)
    z = z_of(s["cos5_64"])
    f = np.diff(np.unwrap(np.angle(z))) / (2 * np.pi)
    assert np.abs(f - 5 / 64).max() < 1e-10
