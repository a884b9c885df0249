"""The allocation-free entry point (afc_execute_1d_no_alloc).

Some callers cannot allocate device memory while they run: cudaMalloc and
cudaFree can synchronize the whole device (stalling a streaming STFT/NUFFT
frame loop), are forbidden inside CUDA stream capture, and are unwelcome where
a caching allocator owns the memory.  This entry point runs the two-pass
(four-step) kernels with their intermediate in a static device array.  The
test calls it through the C ABI twice in a row and compares each result with
afc_execute on the same input (f64 relative L2 <= 1e-12, f32 <= 1e-5), with
every library device allocation made to fail during the call (so the call
provably allocates nothing), and checks the size limit.  It lives in a file of
its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


@pytest.mark.parametrize("prec,n,tol", [("f64", 1 << 16, 1e-12), ("f32", 1 << 17, 1e-5)])
def test_no_alloc_matches_execute_twice(afc, cuda, prec, n, tol):
    L = afc._lib
    batch = 4  # 4 MiB of scratch in both precisions
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    plan = afc.CudaPlan([n], precision=prec, batch=batch, cached=False)
    assert plan.describe(0)["gpu_algo"] == "four_step"
    st = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(11)
    for direction in (0, 1, 0):
        x = torch.randn(batch * n, dtype=cdt, device=cuda, generator=g)
        ref = plan.execute(x, inverse=bool(direction)).reshape(-1)
        out = torch.empty_like(x)
        torch.cuda.synchronize()
        # every device allocation the library attempts now fails: the call must not need one
        L.lib().afc_test_fail_next_allocs(1 << 20)
        try:
            status = L.lib().afc_execute_1d_no_alloc(plan._h, x.data_ptr(), out.data_ptr(), direction, st)
        finally:
            L.lib().afc_test_fail_next_allocs(0)
        L.check(status, "no_alloc")
        torch.cuda.synchronize()
        assert rel(out, ref) <= tol
    plan.close()


def test_no_alloc_rejects_oversize_and_other_plans(afc, cuda):
    L = afc._lib
    big = afc.CudaPlan([1 << 16], precision="f64", batch=32, cached=False)  # 32 MiB of scratch > 16 MiB
    x = torch.zeros(32 << 16, dtype=torch.complex128, device=cuda)
    st = L.lib().afc_execute_1d_no_alloc(big._h, x.data_ptr(), x.data_ptr(), 0, None)
    assert st == L.AFC_ERR_VALIDATION and "16 MiB" in L.last_error()
    small = afc.CudaPlan([256], precision="f64", cached=False)  # single-pass kernel, no scratch
    y = torch.zeros(256, dtype=torch.complex128, device=cuda)
    assert L.lib().afc_execute_1d_no_alloc(small._h, y.data_ptr(), y.data_ptr(), 0, None) == L.AFC_ERR_UNSUPPORTED
    big.close()
    small.close()
