"""The plane-by-plane pass pair (opt-in, AFC_PAIR=1): the last two axes of a
C2C plan run in one launch in which a thread-block cluster owns an x-plane,
transforms its first-axis tiles, meets at the cluster barrier and transforms
its second-axis tiles, so the intermediate stays in L2.

Results must match the oracle's FftPlan2D/3D (crates/apollo-fft/src/
application/execution/plan/fft/dimension_{2,3}d.rs: forward last axis first,
inverse first axis first, 1/N) at f64 <= 1e-12 and f32 <= 1e-5, and a 3D
transform on the pair must take two launches (pair + leading axis) instead of
three."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}


@pytest.fixture(autouse=True)
def pair_on(monkeypatch):
    """The pass pair is opt-in (AFC_PAIR=1, read by the library per execution);
    256 x 256 planes would take the cluster plane kernel first (AFC_PLANE=0
    keeps them on the pair)."""
    monkeypatch.setenv("AFC_PAIR", "1")
    monkeypatch.setenv("AFC_PLANE", "0")


def cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("shape", [(2, 256, 256), (5, 256, 256), (3, 128, 256), (7, 64, 64)])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_pair_3d_vs_oracle(afc, oracle, cuda, shape, prec):
    rng = np.random.default_rng(sum(shape))
    x = cplx(rng, shape)
    ref = oracle.fft3d(x)
    dt = torch.complex128 if prec == "f64" else torch.complex64
    p = afc.CudaPlan(list(shape), precision=prec)
    y = p.execute(torch.from_numpy(x).to(cuda, dt)).cpu().numpy()
    assert rel_l2(y, ref) < TOL[prec]
    back = p.execute(torch.from_numpy(ref).to(cuda, dt), inverse=True).cpu().numpy()
    assert rel_l2(back, oracle.fft3d(ref, inverse=True)) < TOL[prec]
    # in place as well
    t = torch.from_numpy(x).to(cuda, dt)
    p.execute(t, out=t)
    assert rel_l2(t.cpu().numpy(), ref) < TOL[prec]


def test_pair_takes_two_launches(afc, cuda):
    x = torch.zeros((4, 256, 256), dtype=torch.complex128, device=cuda)
    p = afc.CudaPlan([4, 256, 256], precision="f64")
    p.execute(x)
    torch.cuda.synchronize()
    n0 = afc.kernel_launch_count()
    p.execute(x)
    torch.cuda.synchronize()
    assert afc.kernel_launch_count() - n0 == 2


@pytest.mark.parametrize("dims,batch", [([256, 256], 3), ([64, 256], 5)])
def test_pair_2d_batches_vs_oracle(afc, oracle, cuda, dims, batch):
    rng = np.random.default_rng(7)
    x = cplx(rng, (batch,) + tuple(dims))
    ref = oracle.fft2d(x)
    p = afc.CudaPlan(dims, precision="f64", batch=batch)
    y = p.execute(torch.from_numpy(x).to(cuda)).cpu().numpy().reshape(x.shape)
    assert rel_l2(y, ref) < 1e-12
    back = p.execute(torch.from_numpy(ref).to(cuda), inverse=True).cpu().numpy().reshape(x.shape)
    assert rel_l2(back, x) < 1e-12


def test_pair_repeated_calls_are_identical(afc, cuda):
    """The per-plane counters are reset by every launch: repeated and
    alternating-direction calls give bit-identical results."""
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((6, 256, 256), dtype=torch.complex128, device=cuda, generator=g)
    p = afc.CudaPlan([6, 256, 256], precision="f64")
    first = p.execute(x).clone()
    for _ in range(3):
        y = p.execute(x)
        assert torch.equal(y, first)
        p.execute(y, inverse=True)


def test_default_runs_the_separate_passes(afc, cuda, monkeypatch):
    monkeypatch.delenv("AFC_PAIR", raising=False)
    x = torch.zeros((4, 256, 256), dtype=torch.complex128, device=cuda)
    p = afc.CudaPlan([4, 256, 256], precision="f64")
    p.execute(x)
    torch.cuda.synchronize()
    n0 = afc.kernel_launch_count()
    p.execute(x)
    torch.cuda.synchronize()
    assert afc.kernel_launch_count() - n0 == 3
