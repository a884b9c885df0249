"""Oracle float layer pinned to the reference's fixtures and to independent
truth (long-double direct DFT, scipy.fft).  CPU only."""
import numpy as np
import pytest
import scipy.fft

from conftest import rel_l2


def test_dft4_fixture(oracle):  # apollo-validation suite.rs:742-757, limit 1e-12
    y = oracle.fft1d(np.array([1, 0, -1, 0], dtype=np.complex128))
    np.testing.assert_allclose(y, [0, 2, 0, 2], atol=1e-12)


def test_idft4_fixture(oracle):  # suite.rs:1020 (fft_inverse_four_point_fixture)
    y = oracle.fft1d(np.ones(4, dtype=np.complex128), inverse=True)
    np.testing.assert_allclose(y, [1, 0, 0, 0], atol=1e-12)


def test_impulse_full_spectrum_fixture(oracle):  # apollo-python tests/test_smoke.py:28-35
    x = np.zeros((2, 2, 4), dtype=np.complex128)
    x[0, 0, 0] = 1
    np.testing.assert_allclose(oracle.fft3d(x), np.ones((2, 2, 4)), atol=1e-12)


@pytest.mark.parametrize("n", list(range(1, 130)) + [192, 243, 250, 256, 343, 512, 521, 1009, 1024, 1031, 2048, 2053])
def test_oracle_matches_direct_dft(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    if oracle.dispatch_strategy(n) == "untransformed":
        np.testing.assert_array_equal(oracle.dispatch(x), x)  # reference leaves p^k (p > 23) as is
        return
    assert rel_l2(oracle.dispatch(x), oracle.direct_dft(x)) < 1e-12
    assert rel_l2(oracle.dispatch(oracle.direct_dft(x), inverse=True, normalize=True), x) < 1e-12


def test_rader_half_cyclic_against_direct(oracle):  # rader/mod.rs:413-443 (521 at 1e-8)
    for p in (2053, 4099):
        rng = np.random.default_rng(p)
        x = rng.standard_normal(p) + 1j * rng.standard_normal(p)
        assert oracle.dispatch_strategy(p) == "rader_half"
        assert rel_l2(oracle.dispatch(x), oracle.direct_dft(x)) < 1e-12


def test_f32_oracle_tolerance_n45(oracle):  # kernel/mod.rs:272-282 (f32 5e-4 at N=45)
    rng = np.random.default_rng(45)
    x = (rng.standard_normal(45) + 1j * rng.standard_normal(45)).astype(np.complex64)
    y = oracle.dispatch(x)
    ref = oracle.direct_dft(x.astype(np.complex128))
    assert np.max(np.abs(y - ref)) < 5e-4


@pytest.mark.parametrize("shape", [(4, 4, 4), (8, 6, 10), (9, 10, 7), (3, 250, 7)])
def test_oracle_3d_matches_scipy(oracle, shape):
    rng = np.random.default_rng(7)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert rel_l2(oracle.fft3d(x), scipy.fft.fftn(x)) < 1e-13
    assert rel_l2(oracle.fft3d(oracle.fft3d(x), inverse=True), x) < 1e-13


def test_oracle_2d_batch_matches_scipy(oracle):
    rng = np.random.default_rng(8)
    x = rng.standard_normal((3, 48, 30)) + 1j * rng.standard_normal((3, 48, 30))
    assert rel_l2(oracle.fft2d(x), scipy.fft.fft2(x)) < 1e-13


def test_golden_fixtures_reproduce(oracle):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
    assert rel_l2(oracle.fft1d(g["c1_x"]), g["c1_fwd"]) == 0.0
    assert rel_l2(oracle.fft3d(g["c2b_x"]), g["c2b_fwd"]) == 0.0
    for n in (12, 243, 1009, 4099):
        assert rel_l2(g[f"len_{n}_oracle"], g[f"len_{n}_fwd"]) < 1e-12


@pytest.mark.parametrize("shape", [(7, 12), (16, 2048), (5, 30), (6, 10, 34)])
def test_oracle_real_input_spectrum_is_hermitian_in_trailing_axes(oracle, shape):
    """The identity the Hermitian column pass stores: for a real input the
    spectrum after the last two axes satisfies Y[k][n1 - c] =
    conj(Y[(n0 - k) mod n0][c]) in every plane of the leading axes."""
    rng = np.random.default_rng(len(shape) + shape[-1])
    x = rng.standard_normal(shape)
    y = oracle.fft3d(x.reshape((1,) * (3 - len(shape)) + shape).astype(np.complex128)).reshape(shape)
    # the leading axis of a 3D shape is transformed too; the identity holds
    # for the partial transform over the last two axes, so undo the first axis
    if len(shape) == 3:
        y = np.fft.ifft(y, axis=0)
    n0, n1 = shape[-2], shape[-1]
    part = np.conj(np.take(np.take(y, (-np.arange(n0)) % n0, axis=-2), (-np.arange(n1)) % n1, axis=-1))
    assert rel_l2(part, y) < 1e-13
