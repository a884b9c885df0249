"""Failure detection without a GPU fault.

Every spin-wait in the kernels is bounded: on timeout the kernel records the
event in a device error word and returns, and the host reports
AFC_ERR_TIMEOUT.  The test runs one such wait on a barrier that nothing
completes, then checks that the context is still usable."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

AFC_ERR_TIMEOUT = 7
AFC_ERR_VALIDATION = 1


def test_bounded_wait_times_out_and_context_survives(afc, cuda):
    L = afc._lib.lib()
    assert L.afc_test_take_device_error() == 0
    assert L.afc_test_bounded_wait(1000) == AFC_ERR_TIMEOUT
    assert "timed out" in afc._lib.last_error()
    # the error word was cleared and the device still runs transforms
    assert L.afc_test_take_device_error() == 0
    x = (np.random.default_rng(0).standard_normal(4096) * (1 + 1j)).astype(np.complex128)
    p = afc.CudaPlan([4096], precision="f64")
    y = p.execute(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(y, np.fft.fft(x)) < 1e-12
    assert L.afc_test_take_device_error() == 0


def test_bounded_wait_rejects_bad_limits(afc, cuda):
    L = afc._lib.lib()
    assert L.afc_test_bounded_wait(0) == AFC_ERR_VALIDATION
    assert L.afc_test_bounded_wait(1 << 22) == AFC_ERR_VALIDATION
