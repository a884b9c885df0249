"""Pins the NUFFT restatements of oracle/nufft.py, which the device tests compare against (1D:
transform/dimension_1d.rs, 3D: transform/dimension_3d.rs) on the CPU: the
reference's own known answers (DC mode = sum of values, type 2 at the origin =
sum of modes) and its accuracy bound against the exact sums
(fast_3d_tracks_exact: max error / max magnitude < 1e-6 at width 6)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle.nufft import RefPlan, RefPlan3, exact1_1d, exact2_1d, exact1_3d as exact1, exact2_3d as exact2


def test_restatement_1d_tracks_exact(oracle):
    rng = np.random.default_rng(3)
    n, dx = 32, 0.25
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, 60)
    val = rng.standard_normal(60) + 1j * rng.standard_normal(60)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = RefPlan(n, dx, 2, 6)
    assert rel_l2(ref.type1(pos, val, oracle), exact1_1d(pos, val, n, L)) < 1e-6
    assert rel_l2(ref.type2(coeffs, pos, oracle), exact2_1d(coeffs, pos, n, L)) < 1e-6


def test_restatement_3d_reference_known_answers(oracle):  # dimension_3d.rs:777-843
    pos = np.array([(0.0, 0.0, 0.0), (0.1, 0.2, 0.3), (0.25, 0.15, 0.05)])
    val = np.array([1.0, 0.5 - 0.25j, -0.2 + 0.75j])
    ref = RefPlan3((4, 4, 4), (0.1, 0.1, 0.1), 2, 6)
    assert ref.m == [16, 16, 16]
    y = ref.type1(pos, val, oracle)
    assert abs(y[0, 0, 0] - (1.3 + 0.5j)) < 1e-6
    e = exact1(pos, val, (4, 4, 4), [0.4] * 3)
    assert abs(e[0, 0, 0] - (1.3 + 0.5j)) < 1e-12
    assert np.abs(y - e).max() / max(1.0, np.abs(e).max()) < 1e-6
    kx, ky, kz = np.meshgrid(np.arange(3), np.arange(2), np.arange(2), indexing="ij")
    modes = (0.25 + 0.1 * kx - 0.05 * ky + 0.03 * kz) + 1j * (-0.4 + 0.07 * kx + 0.11 * ky - 0.02 * kz)
    g = exact2(modes, np.zeros((1, 3)), (3, 2, 2), [1.5, 1.5, 2.0])
    assert abs(g[0] - modes.sum()) < 1e-12


@pytest.mark.parametrize("w", [4, 6])
def test_restatement_3d_type2_scale(oracle, w):
    """The reference's 3D type 2 carries 1 / (mx my mz) (normalized inverse passes)."""
    rng = np.random.default_rng(w)
    shape, spacing = (6, 5, 4), (0.5, 0.4, 0.25)
    L = [n * d for n, d in zip(shape, spacing)]
    pos = np.stack([rng.uniform(0, l, 25) for l in L], -1)
    modes = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = RefPlan3(shape, spacing, 2, w)
    got = ref.type2(modes, pos, oracle) * np.prod(ref.m)
    assert rel_l2(got, exact2(modes, pos, shape, L)) < (1e-6 if w == 6 else 1e-3)


def test_cpp_restatement_matches_numpy_restatement(oracle):
    """The C++ plans (the timed CPU baseline) and the numpy plans agree."""
    from oracle import nufft as N
    rng = np.random.default_rng(21)
    n, dx = 48, 0.125
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, 80)
    val = rng.standard_normal(80) + 1j * rng.standard_normal(80)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = RefPlan(n, dx, 2, 6)
    assert rel_l2(N.c_type1_1d(n, dx, 2, 6, pos, val), ref.type1(pos, val, oracle)) < 1e-13
    assert rel_l2(N.c_type2_1d(n, dx, 2, 6, coeffs, pos), ref.type2(coeffs, pos, oracle)) < 1e-13
    shape, spacing = (6, 5, 4), (0.5, 0.4, 0.25)
    Ls = [a * b for a, b in zip(shape, spacing)]
    pos3 = np.stack([rng.uniform(-0.5 * l, 1.5 * l, 40) for l in Ls], -1)
    val3 = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    modes = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref3 = RefPlan3(shape, spacing, 2, 6)
    assert rel_l2(N.c_type1_3d(shape, spacing, 2, 6, pos3, val3), ref3.type1(pos3, val3, oracle)) < 1e-13
    assert rel_l2(N.c_type2_3d(shape, spacing, 2, 6, modes, pos3), ref3.type2(modes, pos3, oracle)) < 1e-13
