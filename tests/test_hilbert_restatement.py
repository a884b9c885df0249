"""Pins the analytic-signal restatement the device tests compare against
(oracle FFT, the analytic mask of infrastructure/kernel/direct.rs:130-143,
normalized inverse, real part reset) to apollo-hilbert's own known answers
(verification/mod.rs:11-137), on the CPU."""
import numpy as np

from test_gpu_hilbert import _kat_signals, ref_analytic


def test_restatement_matches_reference_known_answers(oracle):
    s = _kat_signals()
    z, _ = ref_analytic(s["cos16"][None, :], oracle)
    assert np.abs(z[0].imag - np.sin(2 * np.pi * np.arange(16) / 16)).max() < 1e-11
    z, _ = ref_analytic(s["cos3_32"][None, :], oracle)
    assert np.abs(z[0].real - s["cos3_32"]).max() < 1e-12 and np.abs(np.abs(z[0]) - 1.0).max() < 1e-11
    z, _ = ref_analytic(s["const9"][None, :], oracle)
    assert np.abs(z[0].imag).max() < 1e-12
    z, _ = ref_analytic(s["alt10"][None, :], oracle)
    assert np.abs(z[0].imag).max() < 1e-12
    h1 = ref_analytic(s["sin3_32"][None, :], oracle)[0].imag
    h2 = ref_analytic(h1, oracle)[0].imag
    assert np.abs(h2[0] + s["sin3_32"]).max() < 1e-10
    z, _ = ref_analytic(s["cos5_64"][None, :], oracle)
    f = np.diff(np.unwrap(np.angle(z[0]))) / (2 * np.pi)
    assert np.abs(f - 5 / 64).max() < 1e-10
