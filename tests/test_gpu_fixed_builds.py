"""The fixed-address axis builds (every shared-memory offset a compile-time
constant) against the general build and the oracle: 256 points as radix
16 x 16 for contiguous lanes (1D batches, the last axis of a 3D volume) and
strided lanes (the middle and first axes), alone and inside the pass pair, and
4096 points as radix 16 x 16 x 16 on contiguous lanes, and the compile-time
stage lists of the smooth odd lengths 343 = 7 7 7, 243 = 9 9 3 and
250 = 10 5 5 on contiguous and strided lanes; forward and inverse with 1/N, in
and out of place.

AFC_TMA_N256 / AFC_TMA_N4096 (read by the library at every plan): 0 general
build, 1 the fixed build for complex64, 2 for complex128 as well (N256 default
1, N4096 default 2).  AFC_TMA_FIXED: 0 general build, 1 the stage lists
(default).  Results against the
oracle's FftPlan1D/3D (crates/apollo-fft/src/application/execution/plan/fft/
dimension_{1,3}d.rs) at f64 <= 1e-12 and f32 <= 1e-5; both builds compute the
same butterflies with the same twiddles in the same order, so their outputs
agree bit for bit.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}
SAME = {"f64": 1e-14, "f32": 1e-6}
DT = {"f64": torch.complex128, "f32": torch.complex64}


def cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def run(afc, cuda, monkeypatch, mode, shape, prec, x, inverse=False, batch=1):
    monkeypatch.setenv("AFC_TMA_N256", str(mode))
    monkeypatch.setenv("AFC_TMA_N4096", str(mode))
    monkeypatch.setenv("AFC_TMA_FIXED", "1" if mode else "0")
    monkeypatch.setenv("AFC_TMA_L4", "1" if mode else "0")
    p = afc.CudaPlan(list(shape), precision=prec, batch=batch)
    return p.execute(torch.from_numpy(x).to(cuda, DT[prec]), inverse=inverse).cpu().numpy()


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape,batch", [((256,), 37), ((256,), 1), ((3, 256, 256), 1), ((256, 256), 2),
                                         ((256, 8, 256), 1), ((256, 2, 2), 1), ((4096,), 1), ((4096,), 300),
                                         ((3, 4096), 2), ((5, 7, 4096), 1), ((343,), 50), ((243,), 33),
                                         ((250,), 64), ((7, 9, 343), 1), ((243, 250, 34), 1),
                                         ((250, 6, 243), 1), ((2048,), 37), ((2048, 10), 1), ((3, 2048, 6), 1)])
def test_fixed_build_matches_oracle_and_general(afc, oracle, cuda, monkeypatch, prec, shape, batch):
    rng = np.random.default_rng(256 + len(shape) + batch)
    full = (batch,) + shape if batch > 1 else shape
    x = cplx(rng, full)
    if len(shape) == 1:
        n = shape[0]
        ref, ref_inv = oracle.fft1d(x.reshape(-1, n)), oracle.fft1d(x.reshape(-1, n), inverse=True)
    else:
        x3 = x.reshape((-1,) + (1,) * (3 - len(shape)) + shape)
        ref = np.stack([oracle.fft3d(v) for v in x3])
        ref_inv = np.stack([oracle.fft3d(v, inverse=True) for v in x3])
    ref, ref_inv = ref.reshape(full), ref_inv.reshape(full)
    fixed = run(afc, cuda, monkeypatch, 2, shape, prec, x, batch=batch)
    general = run(afc, cuda, monkeypatch, 0, shape, prec, x, batch=batch)
    assert rel_l2(fixed, ref) < TOL[prec]
    assert rel_l2(fixed, general) < SAME[prec]
    fixed_i = run(afc, cuda, monkeypatch, 2, shape, prec, x, inverse=True, batch=batch)
    assert rel_l2(fixed_i, ref_inv) < TOL[prec]
    assert rel_l2(fixed_i, run(afc, cuda, monkeypatch, 0, shape, prec, x, inverse=True, batch=batch)) < SAME[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fixed_build_in_place_and_in_the_pair(afc, oracle, cuda, monkeypatch, prec):
    rng = np.random.default_rng(5)
    shape = (5, 256, 256)
    x = cplx(rng, shape)
    ref = oracle.fft3d(x)
    monkeypatch.setenv("AFC_TMA_N256", "2")
    p = afc.CudaPlan(list(shape), precision=prec)
    t = torch.from_numpy(x).to(cuda, DT[prec])
    p.execute(t, out=t)
    assert rel_l2(t.cpu().numpy(), ref) < TOL[prec]
    p.execute(t, out=t, inverse=True)
    assert rel_l2(t.cpu().numpy(), x) < TOL[prec]
    monkeypatch.setenv("AFC_PAIR", "1")
    p2 = afc.CudaPlan(list(shape), precision=prec)
    y = p2.execute(torch.from_numpy(x).to(cuda, DT[prec])).cpu().numpy()
    assert rel_l2(y, ref) < TOL[prec]
    back = p2.execute(torch.from_numpy(ref).to(cuda, DT[prec]), inverse=True).cpu().numpy()
    assert rel_l2(back, oracle.fft3d(ref, inverse=True)) < TOL[prec]


@pytest.mark.parametrize("kind", ["r2c_full", "r2c_half"])
@pytest.mark.parametrize("shape,batch", [((2048,), 6), ((2, 2048), 3), ((2048, 2048), 1)])
def test_fixed_real_lanes_2048(afc, cuda, monkeypatch, kind, shape, batch):
    """Real input rows widened in the first stage and real parts stored by the
    last stage of the in-place 2048-point build, against numpy (f32 <= 1e-5)
    and against the general build."""
    rng = np.random.default_rng(2048 + batch)
    x = rng.standard_normal((batch,) + shape).astype(np.float32)
    axes = tuple(range(1, len(shape) + 1))
    ref = np.fft.fftn(x.astype(np.float64), axes=axes)
    if kind == "r2c_half":
        ref = np.fft.rfftn(x.astype(np.float64), axes=axes)
    outs = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("AFC_TMA_FIXED", mode)
        monkeypatch.setenv("AFC_TMA_L4", mode)
        p = afc.CudaPlan(list(shape), precision="f32", kind=kind, batch=batch)
        y = p.execute(torch.from_numpy(x).to(cuda))
        back = p.execute(y, inverse=True)
        outs[mode] = (y.cpu().numpy().reshape(ref.shape), back.cpu().numpy().reshape(x.shape))
    assert rel_l2(outs["1"][0], ref) < 1e-5
    assert rel_l2(outs["1"][1], x) < 1e-5
    assert rel_l2(outs["1"][0], outs["0"][0]) < 1e-6
