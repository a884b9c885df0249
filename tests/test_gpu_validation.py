"""Host-side validation: tensors that are not on a CUDA device, wrong dtypes and
mismatched output buffers are rejected with ValueError before any pointer
reaches the C ABI (a host pointer handed to a kernel would fault the device)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_plan_execute_rejects_host_tensors(afc, cuda):
    p = afc.CudaPlan([64], precision="f64", batch=2)
    x = torch.zeros(128, dtype=torch.complex128)
    with pytest.raises(ValueError):
        p.execute(x)
    xd = x.cuda()
    with pytest.raises(ValueError):
        p.execute(xd, out=torch.empty_like(x))
    with pytest.raises(ValueError):
        p.execute(xd.to(torch.complex64))
    with pytest.raises(ValueError):
        p.execute(xd[::2].contiguous())
    y = p.execute(xd)
    assert y.is_cuda and y.numel() == 128


def test_wrappers_reject_host_tensors(afc, cuda):
    from apollofft_b200.batch import BatchPlan
    from apollofft_b200.czt import CztPlan
    from apollofft_b200.hilbert import HilbertPlan
    from apollofft_b200.nufft import NufftPlan1D, NufftPlan3D
    from apollofft_b200.stft import StftPlan
    with pytest.raises(ValueError):
        HilbertPlan(64).analytic_signal(torch.zeros(64, dtype=torch.float64))
    with pytest.raises(ValueError):
        CztPlan(16, 16).forward(torch.zeros(16, dtype=torch.complex128))
    with pytest.raises(ValueError):
        StftPlan(64, 16).forward(torch.zeros(256, dtype=torch.float64))
    bp = BatchPlan([64, 100], precision="f32")
    with pytest.raises(ValueError):
        bp.execute(torch.zeros(164, dtype=torch.complex64))
    with pytest.raises(ValueError):
        bp.execute(torch.zeros(164, dtype=torch.complex64, device="cuda"),
                   out=torch.zeros(100, dtype=torch.complex64, device="cuda"))
    n1 = NufftPlan1D(16, 0.25)
    with pytest.raises(ValueError):
        n1.type1(torch.zeros(4, dtype=torch.float64), torch.zeros(4, dtype=torch.complex128, device="cuda"))
    n3 = NufftPlan3D((4, 4, 4), (0.25, 0.25, 0.25))
    with pytest.raises(ValueError):
        n3.type1(torch.zeros((4, 3), dtype=torch.float64, device="cuda"), torch.zeros(4, dtype=torch.complex128))
    with pytest.raises(ValueError):
        n3.type2(torch.zeros((4, 4, 4), dtype=torch.complex128), torch.zeros((2, 3), dtype=torch.float64, device="cuda"))


def test_tensors_on_another_device_are_rejected(afc, cuda):
    """A tensor on a GPU other than the plan's never reaches the kernels: with
    one GPU in the box the plan object is told it lives on device 1."""
    from apollofft_b200.batch import BatchPlan
    from apollofft_b200.czt import CztPlan
    from apollofft_b200.nufft import NufftPlan1D
    from apollofft_b200.stft import StftPlan
    x = torch.zeros(128, dtype=torch.complex128, device="cuda")
    p = afc.CudaPlan([64], precision="f64", batch=2, cached=False)
    p.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        p.execute(x)
    p.device = 0
    q = afc.CudaPlan([64], precision="f64", batch=2, cached=False)
    q.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        q.adjoint(x)
    q.device = 0
    bp = BatchPlan([64, 100], precision="f32")
    bp.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        bp.execute(torch.zeros(164, dtype=torch.complex64, device="cuda"))
    bp.device = 0
    c = CztPlan(16, 16)
    c.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        c.forward(torch.zeros(16, dtype=torch.complex128, device="cuda"))
    c.device = 0
    s = StftPlan(64, 16)
    s.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        s.forward(torch.zeros(256, dtype=torch.float64, device="cuda"))
    s.device = 0
    n1 = NufftPlan1D(16, 0.25)
    n1.device = 1
    with pytest.raises(ValueError, match="cuda:1"):
        n1.type1(torch.zeros(4, dtype=torch.float64, device="cuda"), torch.zeros(4, dtype=torch.complex128, device="cuda"))
    n1.device = 0
