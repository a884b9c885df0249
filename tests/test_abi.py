"""The C ABI library loads, exports every symbol the header declares and
validates arguments without a GPU (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "apollofft_cuda.h")).read()
    return sorted(set(re.findall(r"^AFC_API [^(]*?\b(afc_\w+)\(", txt, flags=re.M)))


def test_header_declares_expected_entry_points():
    syms = header_symbols()
    for s in ("afc_plan_create", "afc_plan_get_cached", "afc_plan_destroy", "afc_execute", "afc_execute_adjoint",
              "afc_execute_host", "afc_batch_plan_create", "afc_batch_execute", "afc_length_info"):
        assert s in syms


def test_library_exports_every_header_symbol(afc):
    lib = ctypes.CDLL(afc._lib.LIB_PATH)
    for s in header_symbols():
        assert hasattr(lib, s), s


def test_python_signatures_cover_header():
    from apollofft_b200 import _lib
    assert set(header_symbols()) == set(_lib.SIGNATURES)


def _create(afc, rank, dims, prec=1, kind=0, batch=1, device=0):
    h = ctypes.c_void_p()
    arr = (ctypes.c_int64 * max(len(dims), 1))(*dims)
    st = afc._lib.lib().afc_plan_create(ctypes.byref(h), rank, arr, prec, kind, batch, device)
    return st, h


def test_validation_errors(afc):
    L = afc._lib
    st, _ = _create(afc, 3, [4, 0, 4])
    assert st == L.AFC_ERR_VALIDATION
    assert "ny" in L.last_error() and "must be > 0" in L.last_error()
    st, _ = _create(afc, 4, [1, 1, 1, 1])
    assert st == L.AFC_ERR_VALIDATION
    st, _ = _create(afc, 1, [8], batch=0)
    assert st == L.AFC_ERR_VALIDATION
    st, _ = _create(afc, 1, [8], prec=7)
    assert st == L.AFC_ERR_VALIDATION and "precision" in L.last_error()
    st, _ = _create(afc, 2, [16, 16], prec=L.PREC_TC_FP16)  # tensor-core plans: rank-1, n = 16^s
    assert st == L.AFC_ERR_UNSUPPORTED
    assert afc._lib.lib().afc_execute(None, None, None, 0, None) == L.AFC_ERR_VALIDATION


def test_no_device_is_backend_unavailable(afc):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    st, _ = _create(afc, 1, [8])
    assert st == afc._lib.AFC_ERR_BACKEND_UNAVAILABLE


def test_python_api_validation_messages(afc):
    import numpy as np
    with pytest.raises(ValueError, match="C-contiguous"):
        afc.fft1(np.linspace(0.0, 1.0, 16)[::2])
    with pytest.raises(ValueError, match="expects float64/complex128 storage"):
        afc.fft1(np.arange(8, dtype=np.float32))
    with pytest.raises(ValueError, match="expects float32/complex64 storage"):
        afc.fft1(np.linspace(0.0, 1.0, 8), precision="low_precision")
    with pytest.raises(ValueError, match="inconsistent"):
        afc.irfft3(np.ones((2, 2, 3), dtype=np.complex128), 4)
    with pytest.raises(ValueError, match="unsupported precision"):
        afc.fft1(np.zeros(4), precision="bogus")


def test_caller_entry_points_validate_without_device(afc):
    """Argument checks of the fused caller entry points run before any device
    work (null handles, empty lengths, invalid spacing / oversampling / width /
    precision)."""
    L = afc._lib
    lib = L.lib()
    h = ctypes.c_void_p()
    # 3D NUFFT (apollo-nufft NufftPlan3D::new / UniformGrid3D::new contracts)
    for args, field in [((0, 4, 4, 1.0, 1.0, 1.0, 2, 6), "nx"), ((4, 4, 0, 1.0, 1.0, 1.0, 2, 6), "nz"),
                        ((4, 4, 4, 1.0, 0.0, 1.0, 2, 6), "dy"), ((4, 4, 4, 1.0, 1.0, float("inf"), 2, 6), "dz"),
                        ((4, 4, 4, 1.0, 1.0, 1.0, 1, 6), "sigma"), ((4, 4, 4, 1.0, 1.0, 1.0, 2, 1), "kernel_width"),
                        ((4, 4, 4, 1.0, 1.0, 1.0, 2, 33), "kernel_width")]:
        assert lib.afc_nufft3d_plan_create(ctypes.byref(h), *args, 0) == L.AFC_ERR_VALIDATION
        assert field in L.last_error()
    assert lib.afc_nufft3d_plan_create(None, 4, 4, 4, 1.0, 1.0, 1.0, 2, 6, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_nufft3d_type1(None, None, None, 0, None, None) == L.AFC_ERR_VALIDATION
    assert lib.afc_nufft3d_type2(None, None, None, 0, None, None) == L.AFC_ERR_VALIDATION
    m = (ctypes.c_int64 * 3)()
    assert lib.afc_nufft3d_grid_dims(None, m) == L.AFC_ERR_VALIDATION
    assert lib.afc_nufft3d_plan_destroy(None) == L.AFC_OK
    # 1D NUFFT
    assert lib.afc_nufft1d_plan_create(ctypes.byref(h), 0, 1.0, 2, 6, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_nufft1d_plan_create(ctypes.byref(h), 8, -1.0, 2, 6, 0) == L.AFC_ERR_VALIDATION
    # analytic signal (apollo-hilbert HilbertPlan::new rejects an empty signal)
    assert lib.afc_hilbert_plan_create(ctypes.byref(h), 0, L.PREC_F64, 0) == L.AFC_ERR_VALIDATION
    assert "len" in L.last_error()
    assert lib.afc_hilbert_plan_create(ctypes.byref(h), 16, 7, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_hilbert_plan_create(None, 16, L.PREC_F64, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_hilbert_analytic(None, None, None, 1, None) == L.AFC_ERR_VALIDATION
    assert lib.afc_hilbert_plan_destroy(None) == L.AFC_OK


def test_czt_entry_points_validate_without_device(afc):
    """apollo-czt CztPlan::new contracts (czt/dimension_1d.rs:61-75): positive
    lengths, finite non-zero A and W."""
    L = afc._lib
    lib = L.lib()
    h = ctypes.c_void_p()
    for args in [(0, 8, 1.0, 0.0, 0.0, 1.0), (8, 0, 1.0, 0.0, 0.0, 1.0), (8, 8, 0.0, 0.0, 0.0, 1.0),
                 (8, 8, 1.0, 0.0, 0.0, 0.0), (8, 8, float("nan"), 0.0, 0.0, 1.0)]:
        assert lib.afc_czt_plan_create(ctypes.byref(h), *args, L.PREC_F64, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_czt_plan_create(ctypes.byref(h), 8, 8, 1.0, 0.0, 0.0, 1.0, 9, 0) == L.AFC_ERR_VALIDATION
    assert lib.afc_czt_execute(None, None, None, 1, None) == L.AFC_ERR_VALIDATION
    v = ctypes.c_int64()
    assert lib.afc_czt_conv_len(None, ctypes.byref(v)) == L.AFC_ERR_VALIDATION
    assert lib.afc_czt_plan_destroy(None) == L.AFC_OK


@pytest.mark.parametrize("compiler,std,lang", [("gcc", "-std=c99", "c"), ("g++", "-std=c++17", "c++")])
def test_header_is_plain_c_and_cpp(tmp_path, compiler, std, lang):
    """include/apollofft_cuda.h is the C ABI: it compiles as strict C99 (no torch
    or CUDA types in the signatures) and as C++."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    src = tmp_path / "use_header.c"
    src.write_text('#include "apollofft_cuda.h"\nint main(void) { afc_plan p = 0; (void)p; return 0; }\n')
    cmd = [compiler, std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", lang,
           "-I", os.path.join(ROOT, "include"), str(src)]
    if lang == "c":
        cmd.insert(3, "-pedantic")
    subprocess.run(cmd, check=True)
