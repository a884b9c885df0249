"""Committed fixtures of the fused caller operations (tests/golden/callers.npz,
made by tests/golden/make_callers_golden.py from the CPU restatements): the CPU
side checks that the restatements still reproduce them and that they meet the
reference's own bounds; the device side compares the library's outputs with
them (f64, relative L2 <= 1e-12; 1e-11 for the CZT)."""
import cmath
import os

import numpy as np
import pytest

from conftest import rel_l2

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "callers.npz"))


def test_fixtures_reproduce_and_meet_reference_bounds(oracle):
    from oracle import nufft as N
    ref = N.RefPlan(32, 0.25, 2, 6)
    assert rel_l2(ref.type1(G["nufft1_pos"], G["nufft1_val"], oracle), G["nufft1_type1"]) < 1e-14
    assert rel_l2(ref.type2(G["nufft1_coeffs"], G["nufft1_pos"], oracle), G["nufft1_type2"]) < 1e-14
    assert rel_l2(G["nufft1_type1"], N.exact1_1d(G["nufft1_pos"], G["nufft1_val"], 32, 8.0)) < 1e-6
    ref3 = N.RefPlan3((8, 6, 5), (0.25, 0.5, 0.2), 2, 6)
    assert rel_l2(ref3.type1(G["nufft3_pos"], G["nufft3_val"], oracle), G["nufft3_type1"]) < 1e-14
    e3 = N.exact1_3d(G["nufft3_pos"], G["nufft3_val"], (8, 6, 5), [2.0, 3.0, 1.0])
    assert np.abs(G["nufft3_type1"] - e3).max() / max(1.0, np.abs(e3).max()) < 1e-6
    # CZT fixture against the direct sum (czt/dimension_1d.rs:503-526 bound)
    a, w = G["czt_params"]
    x = G["czt_x"]
    direct = np.array([sum(x[j] * cmath.rect(abs(a) ** -j, cmath.phase(a) * -j) *
                           cmath.rect(abs(w) ** (j * k), cmath.phase(w) * j * k) for j in range(50))
                       for k in range(30)])
    assert np.abs(G["czt_out"] - direct).max() < 1e-9
    # analytic signal: real part is the input; the quadrature recomputed from the
    # oracle FFT and the analytic mask (hilbert infrastructure/kernel/direct.rs:85-143)
    assert np.array_equal(G["hilb_z"].real, G["hilb_x"])
    hx = G["hilb_x"]
    n = hx.shape[-1]
    k = np.arange(n)
    mask = np.where(k < (n + 1) // 2, 2.0, 0.0)
    mask[0] = 1.0
    if n % 2 == 0:
        mask[n // 2] = 1.0
    z = oracle.fft1d(oracle.fft1d(hx.astype(np.complex128)) * mask, inverse=True)
    assert rel_l2(z.imag, G["hilb_z"].imag) < 1e-14
    # STFT spectrum recomputed from the frame loop of apollo-stft (frames centred
    # at m hop - frame_len / 2, zero outside the signal, symmetric Hann window;
    # stft/dimension_1d.rs:96-108, 225-239) and the oracle's 1D plan
    sig = G["stft_signal"]
    frame, hop = G["stft_spec"].shape[1], 16
    win = 0.5 - 0.5 * np.cos(2 * np.pi * np.arange(frame) / (frame - 1))
    frames = 1 + -(-sig.size // hop)
    assert frames == G["stft_spec"].shape[0]
    fr = np.zeros((frames, frame), dtype=np.complex128)
    for mm in range(frames):
        st = mm * hop - frame // 2
        lo, hi = max(st, 0), min(st + frame, sig.size)
        fr[mm, lo - st:hi - st] = sig[lo:hi] * win[lo - st:hi - st]
    assert rel_l2(oracle.fft1d(fr), G["stft_spec"]) < 1e-14


@pytest.mark.gpu
def test_device_matches_fixtures(afc, cuda):
    import torch
    from apollofft_b200.czt import CztPlan
    from apollofft_b200.hilbert import HilbertPlan
    from apollofft_b200.nufft import NufftPlan1D, NufftPlan3D
    from apollofft_b200.stft import StftPlan

    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    p1 = NufftPlan1D(32, 0.25)
    assert rel_l2(p1.type1(t(G["nufft1_pos"]), t(G["nufft1_val"])).cpu().numpy(), G["nufft1_type1"]) < 1e-12
    assert rel_l2(p1.type2(t(G["nufft1_coeffs"]), t(G["nufft1_pos"])).cpu().numpy(), G["nufft1_type2"]) < 1e-12
    p3 = NufftPlan3D((8, 6, 5), (0.25, 0.5, 0.2))
    assert rel_l2(p3.type1(t(G["nufft3_pos"]), t(G["nufft3_val"])).cpu().numpy(), G["nufft3_type1"]) < 1e-12
    assert rel_l2(p3.type2(t(G["nufft3_modes"]), t(G["nufft3_pos"])).cpu().numpy(), G["nufft3_type2"]) < 1e-12
    z = HilbertPlan(100).analytic_signal(t(G["hilb_x"])).cpu().numpy()
    assert rel_l2(z, G["hilb_z"]) < 1e-12
    a, w = G["czt_params"]
    c = CztPlan(50, 30, complex(a), complex(w)).forward(t(G["czt_x"])).cpu().numpy()
    assert rel_l2(c, G["czt_out"]) < 1e-11  # chirps evaluated on the host in both; FFT rounding differs
    s = StftPlan(64, 16).forward(t(G["stft_signal"])).cpu().numpy()
    assert rel_l2(s, G["stft_spec"]) < 1e-12
