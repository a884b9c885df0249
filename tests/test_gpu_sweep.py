"""Every 1D length from 1 to 2048 (f64 and f32) and a seeded sample of 3D
shapes up to 32^3, against the oracle, with guard bands around every device
buffer.

Each transform reads from and writes into the interior of a buffer whose 64
elements on either side hold a sentinel; after the forward (out of place) and
the inverse (in place) the sentinels must be untouched, so a kernel that
writes outside its array fails here even when its result is right.  Results:
f64 relative L2 <= 1e-12 against the oracle's dispatch (crates/apollo-fft/src/
application/execution/kernel/mixed_radix/dispatch.rs:26-86), f32 <= 1e-5
against the f64 oracle; where the reference path is not a DFT (prime powers
q^k with q = 19 or q > 23, which its dispatcher leaves untransformed, and
primes whose Rader convolution reaches one) the device is held to the exact
DFT instead.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
G = 64  # guard elements on each side (1 KiB in complex128: keeps 16-byte alignment)
SENTINEL = {"f64": 1.2345e300, "f32": 1.2345e30}


def guarded(x, prec, cuda):
    dt = torch.complex128 if prec == "f64" else torch.complex64
    buf = torch.full((x.size + 2 * G,), complex(SENTINEL[prec], -SENTINEL[prec]), dtype=dt, device=cuda)
    buf[G:G + x.size] = torch.from_numpy(x.reshape(-1)).to(cuda, dt)
    return buf


def guards_intact(buf, prec):
    s = complex(SENTINEL[prec], -SENTINEL[prec])
    return bool((buf[:G] == s).all().item() and (buf[-G:] == s).all().item())


def reference(oracle, x):
    """The oracle's result, or the exact DFT where the reference path is not one."""
    ref = oracle.fft1d(x)
    exact = np.fft.fft(x, axis=-1)
    if rel_l2(ref, exact) > 1e-10:
        return exact
    return ref


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_every_length_to_2048(afc, oracle, cuda, prec):
    rng = np.random.default_rng(2048)
    tol = 1e-12 if prec == "f64" else 1e-5
    failures = []
    for n in range(1, 2049):
        batch = 2
        x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
        ref = reference(oracle, x)
        p = afc.CudaPlan([n], precision=prec, batch=batch)
        src = guarded(x, prec, cuda)
        dst = guarded(np.zeros_like(x), prec, cuda)
        p.execute(src[G:G + x.size], out=dst[G:G + x.size])
        y = dst[G:G + x.size].cpu().numpy().reshape(x.shape)
        err = rel_l2(y, ref)
        # inverse in place on the output buffer
        p.execute(dst[G:G + x.size], out=dst[G:G + x.size], inverse=True)
        back = dst[G:G + x.size].cpu().numpy().reshape(x.shape)
        err_i = rel_l2(back, x)
        if err > tol or err_i > tol or not guards_intact(src, prec) or not guards_intact(dst, prec):
            failures.append((n, err, err_i, guards_intact(src, prec), guards_intact(dst, prec)))
    assert not failures, failures[:10]


def test_sampled_3d_shapes_to_32(afc, oracle, cuda):
    rng = np.random.default_rng(32)
    shapes = {tuple(int(v) for v in rng.integers(1, 33, 3)) for _ in range(240)}
    failures = []
    for shape in sorted(shapes):
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ref = oracle.fft3d(x)
        exact = np.fft.fftn(x)
        if rel_l2(ref, exact) > 1e-10:  # an axis the reference leaves untransformed
            ref = exact
        p = afc.CudaPlan(list(shape), precision="f64")
        src = guarded(x, "f64", cuda)
        dst = guarded(np.zeros_like(x), "f64", cuda)
        p.execute(src[G:G + x.size], out=dst[G:G + x.size])
        err = rel_l2(dst[G:G + x.size].cpu().numpy().reshape(shape), ref)
        p.execute(dst[G:G + x.size], out=dst[G:G + x.size], inverse=True)
        err_i = rel_l2(dst[G:G + x.size].cpu().numpy().reshape(shape), x)
        if err > 1e-12 or err_i > 1e-12 or not guards_intact(src, "f64") or not guards_intact(dst, "f64"):
            failures.append((shape, err, err_i))
    assert not failures, failures[:10]


@pytest.mark.parametrize("kind", ["r2c_full", "r2c_half"])
def test_real_kinds_guarded(afc, oracle, cuda, kind):
    """Real-input plans write only their output array: complex spectrum of the
    same shape (full) or of n/2 + 1 bins on the last axis (half)."""
    rng = np.random.default_rng(9)
    failures = []
    for shape in [(30,), (64,), (1024,), (12, 20), (7, 64), (6, 8, 10), (16, 16, 16)]:
        x = rng.standard_normal((2,) + shape)
        p = afc.CudaPlan(list(shape), precision="f64", kind=kind, batch=2)
        axes = tuple(range(1, len(shape) + 1))
        ref = np.fft.fftn(x, axes=axes) if kind == "r2c_full" else np.fft.rfftn(x, axes=axes)
        src = torch.full((x.size + 2 * G,), SENTINEL["f64"], dtype=torch.float64, device=cuda)
        src[G:G + x.size] = torch.from_numpy(x.reshape(-1)).to(cuda)
        dst = guarded(np.zeros(ref.size, dtype=np.complex128), "f64", cuda)
        p.execute(src[G:G + x.size], out=dst[G:G + ref.size])
        err = rel_l2(dst[G:G + ref.size].cpu().numpy().reshape(ref.shape), ref)
        src2 = torch.full((x.size + 2 * G,), SENTINEL["f64"], dtype=torch.float64, device=cuda)
        p.execute(dst[G:G + ref.size], out=src2[G:G + x.size], inverse=True)
        err_i = rel_l2(src2[G:G + x.size].cpu().numpy().reshape(x.shape), x)
        ok = bool((src2[:G] == SENTINEL["f64"]).all().item() and (src2[-G:] == SENTINEL["f64"]).all().item())
        if err > 1e-12 or err_i > 1e-12 or not guards_intact(dst, "f64") or not ok:
            failures.append((shape, err, err_i))
    assert not failures, failures
