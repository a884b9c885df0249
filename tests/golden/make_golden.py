"""Generates tests/golden/*.npz from the CPU oracle (run once; fixtures are committed).

Seeded inputs (numpy PCG64) with the value distributions of the workloads the
library is measured on, at sizes small enough to commit:
  c1_*   : 1D f64 N=4096 lanes, re/im uniform [-1, 1)
  c2_*   : 3D shapes 8x16x32 (pow2) and 9x10x7 (3^2 x 2*5 x 7), re/im N(0,1)
  c3_*   : uneven 1D f32 lengths (pow2 / 7-smooth / prime), uniform [-1, 1)
  c5_*   : 2D real f32 images 64x64, N(0,1), full-spectrum forward
  len_*  : single lanes of assorted lengths (Rader, Bluestein, PFA, composite)
Outputs are the oracle's forward transform (FftwCompatible: unnormalized) and,
where noted, the normalized inverse.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def cplx(rng, shape, dist):
    if dist == "uniform":
        return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(np.complex128)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex128)


def main():
    out = {}
    rng = np.random.default_rng(1)
    x = cplx(rng, (2, 4096), "uniform")
    out["c1_x"] = x
    out["c1_fwd"] = O.fft1d(x)
    out["c1_inv"] = O.fft1d(out["c1_fwd"], inverse=True)
    rng = np.random.default_rng(2)
    for name, shp in (("c2a", (8, 16, 32)), ("c2b", (9, 10, 7))):
        x = cplx(rng, shp, "normal")
        out[f"{name}_x"] = x
        out[f"{name}_fwd"] = O.fft3d(x)
        out[f"{name}_fwd32"] = O.fft3d(x.astype(np.complex64))
    rng = np.random.default_rng(3)
    lens = [64, 128, 96, 105, 97, 1031, 2053, 256, 343]
    xs = [cplx(rng, (n,), "uniform").astype(np.complex64) for n in lens]
    packed = np.concatenate(xs)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
    out["c3_lengths"] = np.asarray(lens, dtype=np.int64)
    out["c3_x"] = packed
    out["c3_fwd64"] = O.fft_uneven(packed.astype(np.complex128), offs, lens)
    rng = np.random.default_rng(5)
    img = rng.standard_normal((2, 64, 64)).astype(np.float32)
    out["c5_x"] = img
    out["c5_fwd64"] = O.fft2d(img.astype(np.complex128))
    rng = np.random.default_rng(6)
    for n in (1, 2, 3, 12, 30, 45, 60, 150, 192, 243, 250, 343, 361, 1009, 2048, 4099):
        x = cplx(rng, (n,), "normal")
        out[f"len_{n}_x"] = x
        out[f"len_{n}_fwd"] = O.direct_dft(x)
        out[f"len_{n}_oracle"] = O.dispatch(x)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
