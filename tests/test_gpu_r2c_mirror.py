"""Full-spectrum R2C forward with Hermitian columns: after the real-input pass
over the last axis, the rows satisfy X[m][n - c] = conj(X[m][c]), so the next
pass (a TMA pass over strided lanes) transforms the columns up to just past
n / 2 and stores the others as conjugate, row-reversed mirrors.

Checked against the oracle's FftPlan2D/3D on the widened real input
(crates/apollo-fft/src/application/execution/plan/fft/dimension_{2,3}d.rs) at
f64 <= 1e-12 and f32 <= 1e-5, against the same plan with every column
transformed (AFC_R2C_MIRROR=0, read at every execution), bit for bit against
the real-row pass storing whole rows instead of only the columns the mirrored
pass reads (AFC_R2C_TRUNC=0), with every output element written (the buffer
starts as NaN), and, on the measured
2048 x 2048 shape, for the exact symmetry of the stored spectrum: a mirrored
column is the bitwise conjugate of its partner read backwards.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}
NEAR = {"f64": 1e-13, "f32": 1e-6}
RDT = {"f64": np.float64, "f32": np.float32}


def run(afc, cuda, monkeypatch, mirror, x, shape, prec, batch, trunc=True):
    """The output buffer starts as NaN, so a column that no pass stores shows."""
    monkeypatch.setenv("AFC_R2C_MIRROR", "1" if mirror else "0")
    monkeypatch.setenv("AFC_R2C_TRUNC", "1" if trunc else "0")
    p = afc.CudaPlan(list(shape), precision=prec, kind="r2c_full", batch=batch)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    out = torch.full(x.shape, complex("nan+nanj"), dtype=cdt, device=cuda)
    y = p.execute(torch.from_numpy(np.ascontiguousarray(x)).to(cuda), out=out)
    torch.cuda.synchronize()
    return y.cpu().numpy().reshape(x.shape)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape,batch", [((2048, 2048), 2), ((7, 12), 3), ((243, 250), 1), ((64, 2048), 1),
                                         ((5, 30), 2), ((256, 256), 2), ((6, 10, 34), 1), ((4, 256, 256), 1),
                                         ((33, 1030), 1), ((2048, 10), 1)])
def test_mirrored_columns_match_oracle_and_full_pass(afc, oracle, cuda, monkeypatch, prec, shape, batch):
    rng = np.random.default_rng(2 * len(shape) + batch + shape[-1])
    full = (batch,) + shape
    x = rng.standard_normal(full).astype(RDT[prec])
    y = run(afc, cuda, monkeypatch, True, x, shape, prec, batch)
    y_all = run(afc, cuda, monkeypatch, False, x, shape, prec, batch)
    x3 = x.astype(np.complex128).reshape((batch,) + (1,) * (3 - len(shape)) + shape)
    ref = np.stack([oracle.fft3d(v, threads=16) for v in x3]).reshape(full)
    assert np.isfinite(y).all() and np.isfinite(y_all).all()
    assert rel_l2(y, ref) < TOL[prec]
    assert rel_l2(y, y_all) < NEAR[prec]
    # the real-row pass storing whole rows changes no stored value
    y_whole = run(afc, cuda, monkeypatch, True, x, shape, prec, batch, trunc=False)
    assert np.array_equal(y, y_whole)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_mirror_exact_on_the_measured_shape(afc, cuda, monkeypatch, prec):
    """2 x 2048 x 2048 real: every column past the computed half (columns
    1028.. at 4 complex64 lanes per tile, 1025.. at one complex128 lane) is the
    exact conjugate of its partner (the mirror stores the computed value)."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 2048, 2048)).astype(RDT[prec])
    y = run(afc, cuda, monkeypatch, True, x, (2048, 2048), prec, 2)
    r = (-np.arange(2048)) % 2048
    cols = np.arange(1029, 2048)  # stored as mirrors at either tile width
    part = np.conj(y[:, r][:, :, 2048 - cols])
    assert np.array_equal(y[:, :, cols], part)
