"""Device 1D NUFFT (afc_nufft1d_*) against the reference's algorithm restated in
numpy (oracle/nufft.py: transform/dimension_1d.rs:156-272, Kaiser-Bessel
spreading with the power-series I0 of kaiser_bessel.rs:55-116, the oracle's
FFT, deconvolution by the kernel's Fourier transform) and against the exact
sums of verification/mod.rs:97-98 within the reference's own accuracy bound."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.nufft import RefPlan, exact1_1d as exact1, exact2_1d as exact2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dx,sigma,w,npts", [(32, 0.25, 2, 6, 200), (64, 0.05, 2, 4, 300), (128, 1.0, 3, 6, 500),
                                               (1536, 0.01, 2, 6, 2000)])
def test_nufft_type1_type2_vs_reference(afc, oracle, cuda, n, dx, sigma, w, npts):
    from apollofft_b200.nufft import NufftPlan1D
    rng = np.random.default_rng(n + npts)
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, npts)      # outside [0, L) too: periodic wrap
    val = rng.standard_normal(npts) + 1j * rng.standard_normal(npts)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = RefPlan(n, dx, sigma, w)
    plan = NufftPlan1D(n, dx, sigma, w)
    p_t = torch.from_numpy(pos).cuda()
    y1 = plan.type1(p_t, torch.from_numpy(val).cuda()).cpu().numpy()
    y2 = plan.type2(torch.from_numpy(coeffs).cuda(), p_t).cpu().numpy()
    r1 = ref.type1(pos, val, oracle)
    r2 = ref.type2(coeffs, pos, oracle)
    assert rel_l2(y1, r1) < 1e-12, rel_l2(y1, r1)
    assert rel_l2(y2, r2) < 1e-12, rel_l2(y2, r2)
    if w == 6:  # the reference's practical bound at the default width (verification/mod.rs:333-390)
        assert rel_l2(y1, exact1(pos, val, n, L)) < 1e-5
        assert rel_l2(y2, exact2(coeffs, pos, n, L)) < 1e-5
    # two calls in a row on the plan's shared grid give the same result
    y1b = plan.type1(p_t, torch.from_numpy(val).cuda()).cpu().numpy()
    assert rel_l2(y1b, y1) < 1e-14


def test_nufft_dc_mode_and_validation(afc, cuda):  # verification/mod.rs:34-80
    from apollofft_b200.nufft import NufftPlan1D
    pos = np.array([0.0, 0.3, 1.1, 1.9])
    val = np.array([1.0, 0.5 - 0.25j, -0.5 + 0.75j, 0.25 + 0.1j])
    plan = NufftPlan1D(8, 0.25)
    y = plan.type1(torch.from_numpy(pos).cuda(), torch.from_numpy(val).cuda()).cpu().numpy()
    assert abs(y[0] - val.sum()) < 1e-6
    for bad in [dict(n=0, dx=1.0), dict(n=8, dx=0.0), dict(n=8, dx=float("inf")), dict(n=8, dx=1.0, sigma=1),
                dict(n=8, dx=1.0, kernel_width=1)]:
        with pytest.raises(ValueError):
            NufftPlan1D(**bad)
