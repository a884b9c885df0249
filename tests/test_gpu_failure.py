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


AFC_ERR_OUT_OF_MEMORY = 6


@pytest.mark.parametrize("dims", [[4096], [97], [20011], [64, 48, 40]])
def test_allocation_failure_reports_out_of_memory(afc, cuda, dims):
    """A failed device allocation during plan build (twiddles, Rader/Bluestein
    tables, workspaces) comes back as AFC_ERR_OUT_OF_MEMORY, and the next plan
    builds and runs normally."""
    L = afc._lib.lib()
    for k in (1, 2, 3):
        L.afc_test_fail_next_allocs(k)
        try:
            afc.CudaPlan(dims, precision="f64", cached=False)
            built = True
        except afc.AfcError as e:
            built = False
            assert e.status == AFC_ERR_OUT_OF_MEMORY, (e.status, str(e))
        finally:
            L.afc_test_fail_next_allocs(0)
        if built:
            break  # the plan needs fewer than k allocations: nothing left to fail
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(dims) + 1j * rng.standard_normal(dims)).astype(np.complex128)
    p = afc.CudaPlan(dims, precision="f64", cached=False)
    y = p.execute(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(y, np.fft.fftn(x)) < 1e-12
