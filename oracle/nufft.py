"""NUFFT restatement (numpy) of apollo-nufft's 1D and 3D plans.

TEST INFRASTRUCTURE ONLY: the checker of the device NUFFT, imported by tests/
and the CPU-baseline leg of bench.py; the apollofft_b200 library never
imports it.  Follows, step by step:
  * Kaiser-Bessel kernel phi(x) = I0(beta sqrt(1 - (x/w)^2)) / I0(beta), I0 by
    its power series, and its Fourier transform for the deconvolution
    (crates/apollo-nufft/src/domain/kernel/kaiser_bessel.rs:55-133);
  * NufftPlan1D (application/execution/transform/dimension_1d.rs:101-272):
    m = sigma n, spreading to round(m x / L) + p, forward FFT, bins
    k_signed mod m times the deconvolution; type 2 through the normalized
    inverse times m;
  * NufftPlan3D (transform/dimension_3d.rs:48-620): per axis
    m = next_pow2(max(sigma n, 2w + 1)), separable weights, 3D FFT, per-axis
    deconvolution; type 2 through the normalized inverse axis passes (no
    rescale, so values carry 1 / (mx my mz));
  * the exact direct sums (dimension_3d.rs:679-739, verification/mod.rs:97-98).
The FFTs are the oracle's (oracle.fft1d / fft3d).  Points are processed in
input order; the reference's bucket sort only reorders the additions.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def i0(z):
    scaled = 0.25 * z * z
    s, term = 1.0, 1.0
    for k in range(1, 257):
        term *= scaled / (k * k)
        s += term
        if term <= np.finfo(float).eps * s:
            break
    return s


def kb(x, w, beta, i0b):
    u2 = (x / w) ** 2
    return 0.0 if u2 >= 1.0 else i0(beta * math.sqrt(1.0 - u2)) / i0b


def kb_ft(xi, w, beta, i0b):
    t = 2.0 * math.pi * w * xi
    z2 = beta * beta - t * t
    pre = 2.0 * w / i0b
    if abs(z2) < 1e-30:
        return pre
    if z2 > 0:
        s = math.sqrt(z2)
        return pre * math.sinh(s) / s
    s = math.sqrt(-z2)
    return pre * math.sin(s) / s


def signed(k, n):
    return k if k <= n // 2 else k - n


def _centre(x, length, m):
    """x mod L (Euclidean), t = m x / L, m0 = round(t) (half away from zero), d = t - m0."""
    r = math.fmod(x, length)
    if r < 0:
        r += length
    t = m * r / length
    m0 = math.floor(t + 0.5) if t >= 0 else math.ceil(t - 0.5)
    return int(m0), t - m0


def _beta(sigma, w):
    return math.pi * (1.0 - 1.0 / (2.0 * sigma)) * (2 * w)


class RefPlan:
    """NufftPlan1D: n bins on [0, n dx), oversampled grid m = sigma n."""

    def __init__(self, n, dx, sigma, w):
        self.n, self.dx, self.m, self.w = n, dx, sigma * n, w
        self.beta = _beta(sigma, w)
        self.i0b = i0(self.beta)
        self.deconv = np.array([1.0 / kb_ft(signed(k, n) / self.m, w, self.beta, self.i0b) for k in range(n)])
        self.L = n * dx

    def _taps(self, x):
        m0, d = _centre(x, self.L, self.m)
        idx = np.array([(m0 + p) % self.m for p in range(-self.w, self.w + 1)])
        wt = np.array([kb(p - d, self.w, self.beta, self.i0b) for p in range(-self.w, self.w + 1)])
        return idx, wt

    def type1(self, pos, val, oracle=O):
        grid = np.zeros(self.m, dtype=np.complex128)
        for x, v in zip(pos, val):
            idx, wt = self._taps(x)
            np.add.at(grid, idx, v * wt)
        spec = oracle.fft1d(grid)
        return np.array([spec[signed(k, self.n) % self.m] * self.deconv[k] for k in range(self.n)])

    def type2(self, coeffs, pos, oracle=O):
        grid = np.zeros(self.m, dtype=np.complex128)
        for k in range(self.n):
            grid[signed(k, self.n) % self.m] = coeffs[k] * self.deconv[k]
        grid = oracle.fft1d(grid, inverse=True) * self.m
        out = np.zeros(len(pos), dtype=np.complex128)
        for j, x in enumerate(pos):
            idx, wt = self._taps(x)
            out[j] = np.sum(grid[idx] * wt)
        return out


def over_len(n, sigma, w):
    lower = max(n * sigma, 2 * w + 1)
    m = 1
    while m < lower:
        m <<= 1
    return m


class RefPlan3:
    """NufftPlan3D: (nx, ny, nz) modes on the box [0, n dx) per axis."""

    def __init__(self, shape, spacing, sigma, w):
        self.n = tuple(shape)
        self.L = [n * d for n, d in zip(shape, spacing)]
        self.m = [over_len(n, sigma, w) for n in shape]
        self.w = w
        self.beta = _beta(sigma, w)
        self.i0b = i0(self.beta)
        self.deconv = [np.array([1.0 / kb_ft(signed(k, n) / m, w, self.beta, self.i0b) for k in range(n)])
                       for n, m in zip(shape, self.m)]
        self.bins = [np.array([signed(k, n) % m for k in range(n)]) for n, m in zip(shape, self.m)]

    def taps(self, x, a):
        m0, d = _centre(x, self.L[a], self.m[a])
        idx = np.array([(m0 + p) % self.m[a] for p in range(-self.w, self.w + 1)])
        wt = np.array([kb(p - d, self.w, self.beta, self.i0b) for p in range(-self.w, self.w + 1)])
        return idx, wt

    def dec(self):
        return self.deconv[0][:, None, None] * self.deconv[1][None, :, None] * self.deconv[2][None, None, :]

    def type1(self, pos, val, oracle=O):
        grid = np.zeros(self.m, dtype=np.complex128)
        for (x, y, z), v in zip(pos, val):
            (ix, wx), (iy, wy), (iz, wz) = self.taps(x, 0), self.taps(y, 1), self.taps(z, 2)
            grid[np.ix_(ix, iy, iz)] += v * (wx[:, None, None] * wy[None, :, None] * wz[None, None, :])
        spec = oracle.fft3d(grid)
        return spec[np.ix_(*self.bins)] * self.dec()

    def type2(self, modes, pos, oracle=O):
        grid = np.zeros(self.m, dtype=np.complex128)
        grid[np.ix_(*self.bins)] = modes * self.dec()
        grid = oracle.fft3d(grid, inverse=True)  # normalized, as the reference's axis passes
        out = np.zeros(len(pos), dtype=np.complex128)
        for j, (x, y, z) in enumerate(pos):
            (ix, wx), (iy, wy), (iz, wz) = self.taps(x, 0), self.taps(y, 1), self.taps(z, 2)
            out[j] = np.sum(grid[np.ix_(ix, iy, iz)] * (wx[:, None, None] * wy[None, :, None] * wz[None, None, :]))
        return out


def exact1_1d(pos, val, n, L):
    ks = np.array([signed(k, n) for k in range(n)])
    return np.exp(-2j * np.pi * np.outer(ks, pos) / L) @ val


def exact2_1d(coeffs, pos, n, L):
    ks = np.array([signed(k, n) for k in range(n)])
    return np.exp(2j * np.pi * np.outer(pos, ks) / L) @ coeffs


def _kgrid(shape, L):
    ks = [np.array([signed(k, n) for k in range(n)]) / l for n, l in zip(shape, L)]
    return np.stack(np.meshgrid(*ks, indexing="ij"), -1).reshape(-1, 3)


def exact1_3d(pos, val, shape, L):
    return (np.exp(-2j * np.pi * _kgrid(shape, L) @ np.asarray(pos).T) @ val).reshape(shape)


def exact2_3d(modes, pos, shape, L):
    return np.exp(2j * np.pi * np.asarray(pos) @ _kgrid(shape, L).T) @ modes.reshape(-1)


# ── the same plans in C++ (oracle/nufft_oracle.cpp), one thread: the timed CPU
# baseline of the device NUFFT and a second restatement the tests pin ──

def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def c_type1_1d(n, dx, sigma, w, pos, val):
    pos, val = _c(pos, np.float64), _c(val, np.complex128)
    out = np.empty(n, dtype=np.complex128)
    O.lib().or_nufft1d_type1(n, dx, sigma, w, pos.ctypes.data, val.ctypes.data, len(pos), out.ctypes.data)
    return out


def c_type2_1d(n, dx, sigma, w, coeffs, pos):
    pos, coeffs = _c(pos, np.float64), _c(coeffs, np.complex128)
    out = np.empty(len(pos), dtype=np.complex128)
    O.lib().or_nufft1d_type2(n, dx, sigma, w, coeffs.ctypes.data, pos.ctypes.data, len(pos), out.ctypes.data)
    return out


def c_type1_3d(shape, spacing, sigma, w, pos, val):
    pos, val = _c(pos, np.float64), _c(val, np.complex128)
    out = np.empty(shape, dtype=np.complex128)
    O.lib().or_nufft3d_type1(*shape, *spacing, sigma, w, pos.ctypes.data, val.ctypes.data, len(val), out.ctypes.data)
    return out


def c_type2_3d(shape, spacing, sigma, w, modes, pos):
    pos, modes = _c(pos, np.float64), _c(modes, np.complex128)
    out = np.empty(len(pos), dtype=np.complex128)
    O.lib().or_nufft3d_type2(*shape, *spacing, sigma, w, modes.ctypes.data, pos.ctypes.data, len(pos),
                             out.ctypes.data)
    return out
