"""Pins the CZT restatement the device tests compare against (the Bluestein
path of apollo-czt kernel/bluestein.rs:83-130 with the plan's chirps,
czt/dimension_1d.rs:60-95, on the oracle's FFT) to apollo-czt's own known
answers (czt/dimension_1d.rs:485-597), on the CPU."""
import cmath

import numpy as np

from test_gpu_czt import czt_direct, czt_reference


def test_bluestein_equals_direct_for_fixed_inputs(oracle):  # dimension_1d.rs:503-526
    for n, m in [(3, 3), (5, 7), (11, 11), (13, 8)]:
        a = cmath.rect(0.9, 0.3)
        w = cmath.rect(1.0, -2 * cmath.pi / n * 0.8)
        x = np.array([complex(np.sin(i * 0.31), -np.cos(i * 0.19)) for i in range(n)])
        fast = czt_reference(x, m, a, w, oracle)
        direct = czt_direct(x, m, a, w)
        assert np.abs(fast - direct).max() < 1e-9, (n, m)


def test_small_sequence_and_dft_parameters(oracle):  # dimension_1d.rs:485-500, 529-547, 580-597
    x = np.array([1.0, 2.0 - 1.0j, 0.5 + 0.25j, -0.75 + 0.5j])
    w = cmath.rect(1.0, -2 * cmath.pi / 8)
    assert np.abs(czt_reference(x, 4, 1.0, w, oracle) - czt_direct(x, 4, 1.0, w)).max() < 1e-9
    rng = np.random.default_rng(8)
    x8 = rng.standard_normal(8) + 1j * rng.standard_normal(8)
    got = czt_reference(x8, 8, 1.0, cmath.exp(-2j * cmath.pi / 8), oracle)
    assert np.abs(got - np.fft.fft(x8)).max() < 1e-9
