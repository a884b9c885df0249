"""Split-precision tensor-core radix-16 stages (tcgen05).

* one tensor-core tile D = A B^T with hi/lo operands against numpy (checks the
  UMMA descriptors and the TMEM read-back);
* 2^k-point transforms (16 <= n <= 4096: radix-16 stages on the tensor cores,
  the one radix-2/4/8 stage of lengths that are not 16^s on the CUDA cores)
  against the exact DFT, per row: FP16 split <= 1e-5 relative L2 (the accuracy
  bar of the split forms), BF16 split measured and bounded;
* high-dynamic-range rows (scaled by 10^k, k in [-6, 6]) keep the FP16 bar
  thanks to the per-butterfly power-of-two scaling.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fp16,tol", [(1, 2e-6), (0, 2e-4)])
def test_tc_tile_matches_numpy(afc, cuda, fp16, tol):
    rng = np.random.default_rng(1)
    A = rng.standard_normal((128, 32)).astype(np.float32)
    B = rng.standard_normal((32, 32)).astype(np.float32)
    D = np.zeros((128, 32), dtype=np.float32)
    st = afc._lib.lib().afc_test_tc_tile(A.ctypes.data, B.ctypes.data, D.ctypes.data, fp16)
    assert st == 0, afc._lib.last_error()
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    err = np.linalg.norm(D - ref) / np.linalg.norm(ref)
    assert err < tol, err


def row_errors(y, ref):
    return np.linalg.norm(y - ref, axis=-1) / np.linalg.norm(ref, axis=-1)


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
@pytest.mark.parametrize("prec,tol", [("tc_fp16", 1e-5), ("tc_bf16", 1e-4)])
def test_tc_fft_rows(afc, cuda, n, prec, tol):
    rng = np.random.default_rng(n)
    batch = 64
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(np.complex64)
    p = afc.CudaPlan([n], precision=prec, batch=batch)
    y = p.execute(torch.from_numpy(x).cuda()).cpu().numpy().reshape(batch, n)
    ref = np.fft.fft(x.astype(np.complex128), axis=-1)
    assert row_errors(y, ref).max() < tol
    xi = p.execute(torch.from_numpy(ref.astype(np.complex64)).cuda(), inverse=True).cpu().numpy().reshape(batch, n)
    assert row_errors(xi, x.astype(np.complex128)).max() < tol


def test_tc_fp16_high_dynamic_range_rows(afc, cuda):
    from apollofft_b200 import workloads as W
    xs, k = W.c4_rows(rows=256, n=4096, seed=4)
    p = afc.CudaPlan([4096], precision="tc_fp16", batch=256)
    y = p.execute(torch.from_numpy(xs).cuda()).cpu().numpy().reshape(256, 4096)
    ref = np.fft.fft(xs.astype(np.complex128), axis=-1)
    err = row_errors(y, ref)
    assert err.max() < 1e-5, (err.max(), k[np.argmax(err)])


def test_tc_plan_rejects_other_shapes(afc, cuda):
    for n in (1000, 8, 8192):
        with pytest.raises(afc.AfcError):
            afc.CudaPlan([n], precision="tc_fp16")
    with pytest.raises(afc.AfcError):
        afc.CudaPlan([16, 16], precision="tc_bf16")
