"""Parity at every measured configuration, at its full size, against the oracle.

Each case uses the configuration's own seeded input and shape and compares the
device result with the oracle's restatement of the reference CPU plan
(FftPlan1D/2D/3D<f64>, crates/apollo-fft/src/application/execution/plan/fft/
dimension_{1,2,3}d.rs; the 3D axis order and per-axis 1/n of
dimension_3d.rs:148-169).  Bars: f64 relative L2 <= 1e-12, f32 <= 1e-5, both
against the f64 oracle; batched configurations are held per row / per lane.

* 3D C2C 256^3 and 243x250x343, complex128 and complex64, forward and
  normalized inverse (re/im N(0,1), seed 2);
* 1D C2C f64 N = 4096 x 64 contiguous lanes (re/im U[-1, 1), seed 1);
* the 4096-lane uneven complex64 batch (lengths log-uniform in [64, 65536],
  thirds power of two / 7-smooth / prime, seed 3), every lane against the
  oracle's per-length dispatch in f64;
* 16384 x 4096 complex64 rows with 25% high-dynamic-range rows (seed 4): the
  FP32 path and both split-precision tensor-core paths, per row;
* 8 x 2048^2 real f32 images (seed 5), full-spectrum R2C forward and the C2R
  inverse of the oracle's spectrum.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}


def c2_input(shape, seed=2):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def row_rel(a, b):
    a = a.reshape(b.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.mark.parametrize("shape", [(256, 256, 256), (243, 250, 343)])
def test_c2_3d_full_size_vs_oracle(afc, oracle, cuda, shape):
    x = c2_input(shape)
    ref = oracle.fft3d(x)
    back_ref = oracle.fft3d(ref, inverse=True)
    for prec, cdt in (("f64", torch.complex128), ("f32", torch.complex64)):
        p = afc.CudaPlan(list(shape), precision=prec)
        xt = torch.from_numpy(x).to(cuda, cdt)
        y = p.execute(xt)
        err = rel_l2(y.cpu().numpy(), ref)
        assert err < TOL[prec], (shape, prec, "forward", err)
        del xt
        yi = p.execute(torch.from_numpy(ref).to(cuda, cdt), inverse=True)
        err_i = rel_l2(yi.cpu().numpy(), back_ref)
        assert err_i < TOL[prec], (shape, prec, "inverse", err_i)
        del y, yi
        torch.cuda.empty_cache()


def test_c2_f32_matches_f32_oracle(afc, oracle, cuda):
    """The f32 plan against the reference's own f32 (low_precision) plan restated."""
    shape = (256, 256, 256)
    x = c2_input(shape).astype(np.complex64)
    ref32 = oracle.fft3d(x)
    ref64 = oracle.fft3d(x.astype(np.complex128))
    y = afc.CudaPlan(list(shape), precision="f32").execute(torch.from_numpy(x).to(cuda)).cpu().numpy()
    # both are f32 approximations of the same f64 result
    assert rel_l2(ref32, ref64) < 1e-5
    assert rel_l2(y, ref32) < 2e-5


def test_c1_as_configured(afc, oracle, cuda):
    from apollofft_b200 import workloads as W
    x = W.c1_input()
    assert x.shape == (64, 4096)
    ref = oracle.fft1d(x)
    p = afc.CudaPlan([4096], precision="f64", batch=64)
    y = p.execute(torch.from_numpy(x).to(cuda)).cpu().numpy()
    assert row_rel(y, ref).max() < 1e-12
    back = p.execute(torch.from_numpy(ref).to(cuda), inverse=True).cpu().numpy()
    assert row_rel(back, oracle.fft1d(ref, inverse=True)).max() < 1e-12


# Primes of the C3 batch whose reference result is not a DFT: the reference's
# Rader half-cyclic convolution of p - 1 reaches a prime power q^k (q = 19 or
# q > 23, k >= 2; 10830 = 2 3 5 19^2, 16810 = 2 5 41^2) for which
# dispatch_inplace (crates/apollo-fft/src/application/execution/kernel/
# mixed_radix/dispatch.rs:26-86) finds no strategy and returns the data
# unchanged (radix_shape.rs:277-285 pins 361 as unsupported), so its output is
# off by about 100%.  The oracle reproduces that; on these lanes the device is
# held to the exact DFT.
REFERENCE_DEFECT_PRIMES = {10831, 16811}


def test_c3_every_lane_vs_oracle(afc, oracle, cuda):
    from apollofft_b200 import workloads as W
    lens = W.c3_lengths()
    assert len(lens) == 4096
    xv = W.c3_values(lens)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]])
    x64 = xv.astype(np.complex128)
    ref = oracle.fft_uneven(x64, offs, lens)
    # lanes where the reference path is not a DFT (see REFERENCE_DEFECT_PRIMES)
    defect = set()
    for i, (o, n) in enumerate(zip(offs, lens)):
        if int(n) in REFERENCE_DEFECT_PRIMES or rel_l2(ref[o:o + n], np.fft.fft(x64[o:o + n])) > 1e-10:
            defect.add(i)
    assert {int(lens[i]) for i in defect} == REFERENCE_DEFECT_PRIMES & set(int(v) for v in lens)
    for i in defect:
        o, n = offs[i], lens[i]
        ref[o:o + n] = np.fft.fft(x64[o:o + n])
    bp = afc.BatchPlan(lens, precision="f32")
    xt = torch.from_numpy(xv).to(cuda)
    for mode in (0, 1):
        y = bp.execute(xt, mode=mode).cpu().numpy()
        errs = np.array([rel_l2(y[o:o + n], ref[o:o + n]) for o, n in zip(offs, lens)])
        assert errs.max() < 1e-5, (mode, float(errs.max()), int(lens[np.argmax(errs)]))


def test_c4_rows_vs_oracle(afc, oracle, cuda):
    from apollofft_b200 import workloads as W
    xs, k = W.c4_rows()
    ref = oracle.fft1d(xs.astype(np.complex128))
    xt = torch.from_numpy(xs).to(cuda)
    for prec in ("f32", "tc_fp16", "tc_bf16"):
        p = afc.CudaPlan([4096], precision=prec, batch=16384)
        y = p.execute(xt).cpu().numpy()
        err = row_rel(y, ref)
        # every path holds the 1e-5 bar on every row, including the rows
        # scaled by 10^k (per-butterfly power-of-two scaling in the FP16 split)
        assert err.max() < 1e-5, (prec, float(err.max()), float(k[np.argmax(err)]))
        del y


def test_c5_r2c_full_size_vs_oracle(afc, oracle, cuda):
    rng = np.random.default_rng(5)
    img = rng.standard_normal((8, 2048, 2048)).astype(np.float32)
    ref = oracle.fft2d(img.astype(np.complex128))
    p = afc.CudaPlan([2048, 2048], precision="f32", kind="r2c_full", batch=8)
    y = p.execute(torch.from_numpy(img).to(cuda)).cpu().numpy().reshape(ref.shape)
    assert row_rel(y, ref).max() < 1e-5
    back = p.execute(torch.from_numpy(ref.astype(np.complex64)).to(cuda), inverse=True).cpu().numpy()
    back_ref = oracle.fft2d(ref, inverse=True).real
    assert row_rel(back.reshape(back_ref.shape), back_ref).max() < 1e-5
