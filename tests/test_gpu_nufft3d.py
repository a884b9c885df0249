"""Device 3D NUFFT (afc_nufft3d_*) against the reference's algorithm restated in
numpy (oracle/nufft.py: transform/dimension_3d.rs:256-330 and 496-603: per-axis oversampled
length next_pow2(max(sigma n, 2w + 1)), separable Kaiser-Bessel weights over
(2w + 1)^3 cells, the oracle's 3D FFT, per-axis deconvolution; type 2 through
the normalized inverse passes) and against the exact sums of
dimension_3d.rs:679-739 within the reference's own bound (fast_3d_tracks_exact:
max error / max magnitude < 1e-6)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle.nufft import RefPlan3, exact1_3d as exact1, exact2_3d as exact2

pytestmark = pytest.mark.gpu


CASES = [((4, 4, 4), (0.1, 0.1, 0.1), 2, 6, 3),
         ((8, 6, 5), (0.25, 0.5, 0.2), 2, 6, 150),
         ((16, 12, 10), (1.0, 0.1, 0.3), 2, 4, 300),
         ((3, 2, 2), (0.5, 0.75, 1.0), 3, 6, 40),
         ((16, 16, 16), (0.0625, 0.0625, 0.0625), 2, 6, 2000),   # shared-memory tiles, B = 8
         ((6, 5, 4), (1.0, 1.0, 1.0), 2, 8, 60),                 # B = 4 tiles
         ((4, 4, 4), (1.0, 1.0, 1.0), 2, 10, 30)]                # too wide for a tile: per-point kernels


@pytest.mark.parametrize("shape,spacing,sigma,w,npts", CASES)
def test_nufft3d_vs_reference(afc, oracle, cuda, shape, spacing, sigma, w, npts):
    from apollofft_b200.nufft import NufftPlan3D
    rng = np.random.default_rng(sum(shape) + npts)
    L = [n * d for n, d in zip(shape, spacing)]
    if npts == 3:  # the reference's fast_3d_tracks_exact points
        pos = np.array([(0.0, 0.0, 0.0), (0.1, 0.2, 0.3), (0.25, 0.15, 0.05)])
        val = np.array([1.0, 0.5 - 0.25j, -0.2 + 0.75j])
    else:
        pos = np.stack([rng.uniform(-0.5 * l, 1.5 * l, npts) for l in L], -1)  # periodic wrap too
        val = rng.standard_normal(npts) + 1j * rng.standard_normal(npts)
    modes = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = RefPlan3(shape, spacing, sigma, w)
    plan = NufftPlan3D(shape, spacing, sigma, w)
    assert plan.oversampled == tuple(ref.m)
    p_t = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    y1 = plan.type1(p_t, torch.from_numpy(val).cuda()).cpu().numpy()
    y2 = plan.type2(torch.from_numpy(modes).cuda(), p_t).cpu().numpy()
    r1 = ref.type1(pos, val, oracle)
    r2 = ref.type2(modes, pos, oracle)
    assert rel_l2(y1, r1) < 1e-12, rel_l2(y1, r1)
    assert rel_l2(y2, r2) < 1e-12, rel_l2(y2, r2)
    if w == 6:
        e1 = exact1(pos, val, shape, L)
        scale = max(1.0, np.abs(e1).max())
        assert np.abs(y1 - e1).max() / scale < 1e-6
        e2 = exact2(modes, pos, shape, L) / np.prod(ref.m)  # the reference's 1/(mx my mz)
        assert rel_l2(y2, e2) < 1e-5


def test_nufft3d_dc_and_origin(afc, cuda):  # dimension_3d.rs:777-823
    from apollofft_b200.nufft import NufftPlan3D
    pos = np.array([(0.0, 0.0, 0.0), (0.1, 0.2, 0.3), (0.25, 0.15, 0.05)])
    val = np.array([1.0, 0.5 - 0.25j, -0.2 + 0.75j])
    plan = NufftPlan3D((4, 4, 4), (0.1, 0.1, 0.1))
    y = plan.type1(torch.from_numpy(pos).cuda(), torch.from_numpy(val).cuda()).cpu().numpy()
    assert abs(y[0, 0, 0] - (1.3 + 0.5j)) < 1e-6
    assert np.isfinite(y).all()
    kx, ky, kz = np.meshgrid(np.arange(3), np.arange(2), np.arange(2), indexing="ij")
    modes = (0.25 + 0.1 * kx - 0.05 * ky + 0.03 * kz) + 1j * (-0.4 + 0.07 * kx + 0.11 * ky - 0.02 * kz)
    plan2 = NufftPlan3D((3, 2, 2), (0.5, 0.75, 1.0))
    g = plan2.type2(torch.from_numpy(np.ascontiguousarray(modes)).cuda(),
                    torch.zeros((1, 3), dtype=torch.float64, device="cuda")).cpu().numpy()
    m = np.prod(plan2.oversampled)
    assert abs(g[0] * m - modes.sum()) < 1e-5 * max(1.0, abs(modes.sum()))


def test_nufft3d_empty_and_validation(afc, cuda):
    from apollofft_b200.nufft import NufftPlan3D
    plan = NufftPlan3D((4, 3, 2), (1.0, 1.0, 1.0))
    y = plan.type1(torch.zeros((0, 3), dtype=torch.float64, device="cuda"),
                   torch.zeros(0, dtype=torch.complex128, device="cuda")).cpu().numpy()
    assert y.shape == (4, 3, 2) and np.all(y == 0)
    g = plan.type2(torch.ones((4, 3, 2), dtype=torch.complex128, device="cuda"),
                   torch.zeros((0, 3), dtype=torch.float64, device="cuda"))
    assert g.numel() == 0
    for bad in [dict(shape=(0, 2, 2), spacing=(1, 1, 1)), dict(shape=(2, 2, 2), spacing=(1, 0, 1)),
                dict(shape=(2, 2, 2), spacing=(1, 1, float("nan"))), dict(shape=(2, 2, 2), spacing=(1, 1, 1), sigma=1),
                dict(shape=(2, 2, 2), spacing=(1, 1, 1), kernel_width=40)]:
        with pytest.raises(ValueError):
            NufftPlan3D(**bad)


def test_nufft3d_growing_and_clustered_points(afc, oracle, cuda):
    """Point buffers grow between calls; every point in one tile; repeat calls agree."""
    from apollofft_b200.nufft import NufftPlan3D
    shape, spacing = (8, 8, 8), (0.125, 0.125, 0.125)
    ref = RefPlan3(shape, spacing, 2, 6)
    plan = NufftPlan3D(shape, spacing)
    rng = np.random.default_rng(5)
    for npts, spread in [(10, 1.0), (400, 1.0), (300, 0.01), (600, 1.0)]:
        pos = rng.uniform(0.0, spread, (npts, 3))
        val = rng.standard_normal(npts) + 1j * rng.standard_normal(npts)
        p_t = torch.from_numpy(pos).cuda()
        y1 = plan.type1(p_t, torch.from_numpy(val).cuda()).cpu().numpy()
        assert rel_l2(y1, ref.type1(pos, val, oracle)) < 1e-12
        y1b = plan.type1(p_t, torch.from_numpy(val).cuda()).cpu().numpy()
        assert rel_l2(y1b, y1) < 1e-14
        modes = torch.from_numpy(np.ascontiguousarray(y1)).cuda()
        y2 = plan.type2(modes, p_t).cpu().numpy()
        assert rel_l2(y2, ref.type2(y1, pos, oracle)) < 1e-12
