"""Fused STFT analysis frames (afc_stft_forward) against the reference's frame
loop restated in numpy: frames centred at m * hop, Hann window of
apollo-stft kernel/hann.rs:10-16, frame count 1 + ceil(signal_len / hop)
(stft/dimension_1d.rs:96-108), each frame transformed by the oracle."""
import numpy as np
import pytest
import torch

from conftest import rel_l2


def frames_ref(signal, window, frame_len, hop):
    n_sig = len(signal)
    frames = 0 if n_sig < frame_len else 1 + -(-n_sig // hop)
    out = np.zeros((frames, frame_len), dtype=np.complex128)
    for m in range(frames):
        start = m * hop - frame_len // 2
        for i in range(frame_len):
            j = start + i
            if 0 <= j < n_sig:
                out[m, i] = signal[j] * window[i]
    return out


def test_frame_count_matches_reference_rule(afc):
    from apollofft_b200 import _lib as L
    import ctypes
    for frame_len, hop, n_sig in [(8, 4, 12), (512, 128, 8192), (512, 128, 8191), (16, 16, 16), (16, 3, 100),
                                  (64, 1, 64), (64, 8, 63)]:
        out = ctypes.c_int64()
        assert L.lib().afc_stft_frame_count(frame_len, hop, n_sig, ctypes.byref(out)) == 0
        want = 0 if n_sig < frame_len else 1 + -(-n_sig // hop)
        assert out.value == want, (frame_len, hop, n_sig)
    assert L.lib().afc_stft_frame_count(8, 0, 12, ctypes.byref(out)) == 1  # AFC_ERR_VALIDATION


def test_hann_window_is_symmetric():  # apollo-stft stft/dimension_1d/tests.rs:11-16
    from apollofft_b200.stft import hann_window
    w = hann_window(8)
    assert np.allclose(w, w[::-1], atol=1e-12)
    assert hann_window(1).tolist() == [1.0]


@pytest.mark.gpu
@pytest.mark.parametrize("frame_len,hop,n_sig", [(512, 128, 8192), (256, 256, 1000), (1024, 300, 20000),
                                                 (64, 1, 64), (16, 5, 333), (4096, 1024, 50000), (243, 81, 5000),
                                                 # frames beyond one CTA: four-step and large-prime Bluestein plans
                                                 (16384, 4096, 100000), (10007, 2500, 60000)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stft_forward_vs_oracle(afc, oracle, cuda, frame_len, hop, n_sig, prec):
    from apollofft_b200.stft import StftPlan
    rng = np.random.default_rng(frame_len + hop + n_sig)
    sig = rng.standard_normal(n_sig)
    plan = StftPlan(frame_len, hop, precision=prec)
    rdt = np.float64 if prec == "f64" else np.float32
    y = plan.forward(torch.from_numpy(sig.astype(rdt)).cuda()).cpu().numpy()
    fr = frames_ref(sig.astype(rdt).astype(np.float64), plan.window.astype(rdt).astype(np.float64), frame_len, hop)
    ref = oracle.fft1d(fr)
    assert y.shape == ref.shape
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel_l2(y, ref) < tol, rel_l2(y, ref)
    # a caller-supplied window (forward_with_window)
    win = rng.uniform(0.5, 1.5, frame_len)
    y2 = plan.forward(torch.from_numpy(sig.astype(rdt)).cuda(), window=win.astype(rdt)).cpu().numpy()
    ref2 = oracle.fft1d(frames_ref(sig.astype(rdt).astype(np.float64), win.astype(rdt).astype(np.float64), frame_len, hop))
    assert rel_l2(y2, ref2) < tol


@pytest.mark.gpu
def test_stft_validation(afc, cuda):
    from apollofft_b200.stft import StftError, StftPlan
    with pytest.raises(StftError):
        StftPlan(0, 1)
    with pytest.raises(StftError):
        StftPlan(8, 0)
    with pytest.raises(StftError):
        StftPlan(8, 9)
    plan = StftPlan(64, 16)
    with pytest.raises(StftError):
        plan.forward(torch.zeros(63, dtype=torch.float64, device="cuda"))
    with pytest.raises(StftError):
        plan.forward(torch.zeros(100, dtype=torch.float64, device="cuda"), window=np.ones(10))


def istft_ref(spec, window, frame_len, hop, n_sig, oracle):
    frames = spec.shape[0]
    fr = oracle.fft1d(spec.astype(np.complex128), inverse=True).real * window
    overlap = np.zeros(n_sig)
    weight = np.zeros(n_sig)
    for m in range(frames):
        start = m * hop - frame_len // 2
        for i in range(frame_len):
            j = start + i
            if 0 <= j < n_sig:
                overlap[j] += fr[m, i]
                weight[j] += window[i] * window[i]
    out = np.where(weight > 0, overlap / np.where(weight > 0, weight, 1.0), 0.0)
    return out, weight


@pytest.mark.gpu
@pytest.mark.parametrize("frame_len,hop,n_sig", [(8, 4, 12), (512, 128, 8192), (256, 200, 1000), (1024, 256, 20001),
                                                 (243, 81, 5000), (16384, 4096, 100001)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stft_inverse_vs_reference_and_roundtrip(afc, oracle, cuda, frame_len, hop, n_sig, prec):
    from apollofft_b200.stft import StftPlan
    rng = np.random.default_rng(frame_len * 3 + hop + n_sig)
    sig = rng.standard_normal(n_sig)
    plan = StftPlan(frame_len, hop, precision=prec)
    rdt = np.float64 if prec == "f64" else np.float32
    cdt = np.complex128 if prec == "f64" else np.complex64
    spec = plan.forward(torch.from_numpy(sig.astype(rdt)).cuda())
    y = plan.inverse(spec, n_sig).cpu().numpy()
    ref, weight = istft_ref(spec.cpu().numpy().astype(np.complex128), plan.window.astype(rdt).astype(np.float64),
                            frame_len, hop, n_sig, oracle)
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel_l2(y, ref) < tol, rel_l2(y, ref)
    covered = weight > 1e-3
    assert rel_l2(y[covered], sig[covered]) < (1e-12 if prec == "f64" else 1e-5)
    # a spectrum of the wrong size is rejected
    from apollofft_b200.stft import StftError
    with pytest.raises(StftError):
        plan.inverse(spec[:-1].contiguous(), n_sig)


def test_restatement_roundtrip_reference_case(oracle):  # stft/dimension_1d/tests.rs:19-30
    """The analysis / synthesis restatements reproduce the reference's COLA
    round trip (frame 8, hop 4, its 12-sample signal) to its 1e-8 bound."""
    from apollofft_b200.stft import hann_window
    signal = np.array([1.0, -1.0, 0.5, 2.0, -0.75, 0.25, 1.5, -0.5, 0.125, 0.875, -1.25, 0.75])
    w = hann_window(8)
    spec = oracle.fft1d(frames_ref(signal, w, 8, 4))
    rec, _ = istft_ref(spec, w, 8, 4, len(signal), oracle)
    assert np.abs(rec - signal).max() < 1e-8
