"""Seeded synthetic inputs of the measured configurations.

c1 : 1D C2C f64, N=4096, 64 contiguous lanes, re/im uniform [-1, 1)        (seed 1)
c2 : 3D C2C, 256^3 and 243x250x343, complex64/complex128, re/im N(0,1)    (seed 2)
c3 : 4096 uneven 1D complex64 lengths, log-uniform in [64, 65536]; the
     first third snapped to the nearest power of two, the second to the
     nearest 7-smooth length (2^a 3^b 5^c 7^d), the last to the nearest
     prime; values uniform [-1, 1)                                           (seed 3)
c4 : 16384 x 4096 complex64, rows N(0,1); a seeded 25% of rows scaled by
     10^k, k uniform in [-6, 6]                                              (seed 4)
c5 : 8 x 2048 x 2048 real f32 images N(0,1) and a seeded radial weight     (seed 5)
"""
from __future__ import annotations

import bisect
import math

import numpy as np


def _smooth7(limit: int):
    out = []
    p2 = 1
    while p2 <= limit:
        p3 = p2
        while p3 <= limit:
            p5 = p3
            while p5 <= limit:
                p7 = p5
                while p7 <= limit:
                    out.append(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def _primes(limit: int):
    sieve = np.ones(limit + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    return np.nonzero(sieve)[0].tolist()


def _nearest(sorted_vals, x):
    i = bisect.bisect_left(sorted_vals, x)
    cands = [sorted_vals[j] for j in (i - 1, i) if 0 <= j < len(sorted_vals)]
    return min(cands, key=lambda v: (abs(v - x), v))


def c3_lengths(count: int = 4096, lo: int = 64, hi: int = 65536, seed: int = 3):
    rng = np.random.default_rng(seed)
    raw = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    pow2 = [1 << k for k in range(int(math.log2(lo)), int(math.log2(hi)) + 1)]
    smooth = [v for v in _smooth7(hi) if v >= lo]
    primes = [p for p in _primes(hi) if p >= lo]
    third = count // 3
    out = []
    for i, x in enumerate(raw):
        if i < third:
            out.append(_nearest(pow2, x))
        elif i < 2 * third:
            out.append(_nearest(smooth, x))
        else:
            out.append(_nearest(primes, x))
    return np.asarray(out, dtype=np.int64)


def c3_values(lengths, seed: int = 3):
    rng = np.random.default_rng(seed + 1000)
    total = int(np.sum(lengths))
    return (rng.uniform(-1, 1, total) + 1j * rng.uniform(-1, 1, total)).astype(np.complex64)


def c1_input(seed: int = 1):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, (64, 4096)) + 1j * rng.uniform(-1, 1, (64, 4096))).astype(np.complex128)


def c4_rows(rows: int = 16384, n: int = 4096, seed: int = 4, hdr_fraction: float = 0.25):
    """Returns (data complex64 [rows, n], scale exponent per row (0 for plain rows))."""
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((rows, n), dtype=np.float32) + 1j * rng.standard_normal((rows, n), dtype=np.float32))
    k = np.zeros(rows)
    hdr = rng.random(rows) < hdr_fraction
    k[hdr] = rng.uniform(-6, 6, int(hdr.sum()))
    x = x * (10.0 ** k)[:, None].astype(np.float32)
    return x.astype(np.complex64), k


def radial_weight(n: int, seed: int = 5):
    rng = np.random.default_rng(seed)
    kf = np.fft.fftfreq(n)
    r = np.sqrt(kf[:, None] ** 2 + kf[None, :] ** 2)
    a, b = rng.uniform(0.5, 2.0, 2)
    return (a * np.exp(-b * r * 8) + 0.1).astype(np.float64)
