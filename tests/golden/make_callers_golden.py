"""Generates tests/golden/callers.npz: fixtures for the fused caller operations,
from the CPU restatements of the reference's algorithms (run once; committed).

  nufft1_* : apollo-nufft NufftPlan1D, n = 32, dx = 0.25, sigma 2, width 6,
             60 points uniform on [-L/2, 3L/2), values / coefficients N(0,1)
             (oracle/nufft.py restatement)
  nufft3_* : NufftPlan3D, (8, 6, 5) modes, spacing (0.25, 0.5, 0.2), sigma 2,
             width 6, 40 points, N(0,1) values and modes
  hilb_*   : apollo-hilbert analytic signal, 2 lanes of 100 N(0,1) samples
             (oracle FFT, analytic mask, normalized inverse, real part reset)
  czt_*    : apollo-czt Bluestein CZT, n = 50, m = 30, A = e^0.2i,
             W = e^(-2 pi i 0.9 / 30), uniform [-1, 1) input
  stft_*   : apollo-stft analysis, frame 64, hop 16, 300 N(0,1) samples,
             symmetric Hann window
"""
import cmath
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
from oracle import nufft as N  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    # 1D NUFFT
    n, dx = 32, 0.25
    L = n * dx
    pos = rng.uniform(-0.5 * L, 1.5 * L, 60)
    val = rng.standard_normal(60) + 1j * rng.standard_normal(60)
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = N.RefPlan(n, dx, 2, 6)
    out.update(nufft1_pos=pos, nufft1_val=val, nufft1_coeffs=coeffs,
               nufft1_type1=ref.type1(pos, val, O), nufft1_type2=ref.type2(coeffs, pos, O))
    # 3D NUFFT
    shape, spacing = (8, 6, 5), (0.25, 0.5, 0.2)
    Ls = [a * b for a, b in zip(shape, spacing)]
    pos3 = np.stack([rng.uniform(-0.5 * l, 1.5 * l, 40) for l in Ls], -1)
    val3 = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    modes = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref3 = N.RefPlan3(shape, spacing, 2, 6)
    out.update(nufft3_pos=pos3, nufft3_val=val3, nufft3_modes=modes,
               nufft3_type1=ref3.type1(pos3, val3, O), nufft3_type2=ref3.type2(modes, pos3, O))
    # analytic signal
    x = rng.standard_normal((2, 100))
    k = np.arange(100)
    mask = np.where(k < 50, 2.0, 0.0)
    mask[0] = 1.0
    mask[50] = 1.0
    z = O.fft1d(O.fft1d(x.astype(np.complex128)) * mask, inverse=True)
    out.update(hilb_x=x, hilb_z=x + 1j * z.imag)
    # CZT (Bluestein with the plan's polar-form chirps)
    nn, m = 50, 30
    a, w = cmath.exp(0.2j), cmath.exp(-2j * cmath.pi * 0.9 / 30)

    def pw(zz, e):
        return cmath.rect(abs(zz) ** e, cmath.phase(zz) * e)

    xc = rng.uniform(-1, 1, nn) + 1j * rng.uniform(-1, 1, nn)
    Lc = 1
    while Lc < nn + m - 1:
        Lc <<= 1
    cn = np.array([pw(a, -j) * pw(w, 0.5 * j * j) for j in range(nn)])
    ck = np.array([pw(w, 0.5 * kk * kk) for kk in range(m)])
    ker = np.zeros(Lc, dtype=np.complex128)
    for kk in range(m):
        ker[kk] = pw(w, -0.5 * kk * kk)
    for j in range(1, nn):
        ker[Lc - j] = pw(w, -0.5 * j * j)
    ws = np.zeros(Lc, dtype=np.complex128)
    ws[:nn] = xc * cn
    ws = O.fft1d(O.fft1d(ws) * O.fft1d(ker), inverse=True)
    out.update(czt_x=xc, czt_params=np.array([a, w]), czt_out=ws[:m] * ck)
    # STFT analysis (frames centred at m hop - frame_len / 2, zero outside)
    frame, hop, ns = 64, 16, 300
    sig = rng.standard_normal(ns)
    win = 0.5 - 0.5 * np.cos(2 * np.pi * np.arange(frame) / (frame - 1))
    frames = 1 + -(-ns // hop)
    fr = np.zeros((frames, frame), dtype=np.complex128)
    for mm in range(frames):
        st = mm * hop - frame // 2
        for i in range(frame):
            j = st + i
            if 0 <= j < ns:
                fr[mm, i] = sig[j] * win[i]
    out.update(stft_signal=sig, stft_spec=O.fft1d(fr))
    np.savez_compressed(os.path.join(HERE, "callers.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
