"""The cluster plane kernel: the last two axes of a C2C transform with
256 x 256 planes in one launch, a thread-block cluster per plane exchanging
columns through distributed shared memory.

Results against the oracle's FftPlan2D/3D (crates/apollo-fft/src/application/
execution/plan/fft/dimension_{2,3}d.rs) at f64 <= 1e-12 and f32 <= 1e-5, for
every kernel build (AFC_PLANE=2: clusters of 16 with two plane buffers, 3:
clusters of 16 with two CTAs per SM, 4: clusters of 8; 1 automatic; the
kernel is opt-in, off by default), forward
and inverse with 1/N, out of place and in place, plane counts below, at and
above the clusters in flight; a 3D transform takes two launches (plane kernel
+ leading axis), and repeated calls are bit-identical.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = {"f64": 1e-12, "f32": 1e-5}
DT = {"f64": torch.complex128, "f32": torch.complex64}


def cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("build", ["2", "3", "4", "1"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(1, 256, 256), (3, 256, 256), (37, 256, 256)])
def test_plane_3d_vs_oracle(afc, oracle, cuda, monkeypatch, build, prec, shape):
    monkeypatch.setenv("AFC_PLANE", build)
    rng = np.random.default_rng(shape[0] + int(build))
    x = cplx(rng, shape)
    ref = oracle.fft3d(x)
    p = afc.CudaPlan(list(shape), precision=prec)
    y = p.execute(torch.from_numpy(x).to(cuda, DT[prec])).cpu().numpy()
    assert rel_l2(y, ref) < TOL[prec]
    back = p.execute(torch.from_numpy(ref).to(cuda, DT[prec]), inverse=True).cpu().numpy()
    assert rel_l2(back, oracle.fft3d(ref, inverse=True)) < TOL[prec]
    t = torch.from_numpy(x).to(cuda, DT[prec])
    p.execute(t, out=t)
    assert rel_l2(t.cpu().numpy(), ref) < TOL[prec]
    p.execute(t, out=t, inverse=True)
    assert rel_l2(t.cpu().numpy(), x) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("batch", [1, 5])
def test_plane_2d_batches_vs_oracle(afc, oracle, cuda, monkeypatch, prec, batch):
    monkeypatch.setenv("AFC_PLANE", "1")
    rng = np.random.default_rng(batch)
    x = cplx(rng, (batch, 256, 256))
    ref = oracle.fft2d(x)
    p = afc.CudaPlan([256, 256], precision=prec, batch=batch)
    y = p.execute(torch.from_numpy(x).to(cuda, DT[prec])).cpu().numpy().reshape(x.shape)
    assert rel_l2(y, ref) < TOL[prec]
    back = p.execute(torch.from_numpy(ref).to(cuda, DT[prec]), inverse=True).cpu().numpy().reshape(x.shape)
    assert rel_l2(back, x) < TOL[prec]


def test_plane_takes_two_launches_and_repeats_bit_identically(afc, cuda, monkeypatch):
    monkeypatch.setenv("AFC_PLANE", "1")
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((6, 256, 256), dtype=torch.complex128, device=cuda, generator=g)
    p = afc.CudaPlan([6, 256, 256], precision="f64")
    first = p.execute(x).clone()
    torch.cuda.synchronize()
    n0 = afc.kernel_launch_count()
    y = p.execute(x)
    torch.cuda.synchronize()
    assert afc.kernel_launch_count() - n0 == 2
    assert torch.equal(y, first)
    for _ in range(2):
        p.execute(y, inverse=True)
        assert torch.equal(p.execute(x), first)


def test_plane_off_by_default(afc, cuda, monkeypatch):
    monkeypatch.delenv("AFC_PLANE", raising=False)
    x = torch.zeros((4, 256, 256), dtype=torch.complex128, device=cuda)
    p = afc.CudaPlan([4, 256, 256], precision="f64")
    p.execute(x)
    torch.cuda.synchronize()
    n0 = afc.kernel_launch_count()
    p.execute(x)
    torch.cuda.synchronize()
    assert afc.kernel_launch_count() - n0 == 3
