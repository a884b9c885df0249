"""ctypes binding of libapollofft_cuda.so (the C ABI in include/apollofft_cuda.h).

There is no fallback: if the shared library is missing the import fails with
instructions to build it, and every transform runs the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libapollofft_cuda.so")

AFC_OK = 0
AFC_ERR_VALIDATION = 1
AFC_ERR_SHAPE_MISMATCH = 2
AFC_ERR_NON_CONTIGUOUS = 3
AFC_ERR_BACKEND_UNAVAILABLE = 4
AFC_ERR_DEVICE = 5
AFC_ERR_OUT_OF_MEMORY = 6
AFC_ERR_TIMEOUT = 7
AFC_ERR_UNSUPPORTED = 8

PREC_F32, PREC_F64, PREC_TC_BF16, PREC_TC_FP16 = 0, 1, 2, 3
KIND_C2C, KIND_R2C_FULL, KIND_R2C_HALF = 0, 1, 2
FORWARD, INVERSE = 0, 1

ALGO_NAMES = {0: "smem_stockham", 1: "four_step", 2: "rader", 3: "bluestein", 4: "noop"}
STRATEGY_NAMES = {
    0: "noop", 1: "stockham", 2: "four_step", 3: "winograd", 4: "pfa_static",
    5: "composite", 6: "pfa_generic", 7: "rader_full", 8: "rader_half", 9: "untransformed",
}


class AfcError(RuntimeError):
    """A non-validation failure reported by the CUDA library."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class Capabilities(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("normalization", ctypes.c_int),
        ("supports_1d", ctypes.c_int), ("supports_2d", ctypes.c_int), ("supports_3d", ctypes.c_int),
        ("supports_real_to_complex", ctypes.c_int), ("supports_mixed_precision", ctypes.c_int),
        ("default_precision", ctypes.c_int), ("device_count", ctypes.c_int), ("sm_count", ctypes.c_int),
        ("cc_major", ctypes.c_int), ("cc_minor", ctypes.c_int), ("max_smem_per_block", ctypes.c_size_t),
    ]


class LengthInfo(ctypes.Structure):
    _fields_ = [
        ("strategy", ctypes.c_int), ("n_radices", ctypes.c_int), ("radices", ctypes.c_uint64 * 64),
        ("coprime_n1", ctypes.c_uint64), ("coprime_n2", ctypes.c_uint64),
        ("four_step_n1", ctypes.c_uint64), ("four_step_n2", ctypes.c_uint64),
        ("primitive_root", ctypes.c_uint64), ("primitive_root_inv", ctypes.c_uint64),
        ("is_prime", ctypes.c_int), ("is_short_winograd", ctypes.c_int),
        ("has_static_coprime_codelet", ctypes.c_int),
        ("gpu_algo", ctypes.c_int), ("gpu_n_radices", ctypes.c_int), ("gpu_radices", ctypes.c_int * 24),
        ("gpu_conv_len", ctypes.c_uint64), ("gpu_split_n1", ctypes.c_uint64), ("gpu_split_n2", ctypes.c_uint64),
    ]


# Every symbol include/apollofft_cuda.h declares, with its ctypes signature.
_vp, _i32, _i64, _u64, _dbl, _sz = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64,
                                     ctypes.c_double, ctypes.c_size_t)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pu64 = ctypes.POINTER(ctypes.c_uint64)
SIGNATURES = {
    "afc_plan_create": (_i32, [ctypes.POINTER(_vp), _i32, _pi64, _i32, _i32, _i64, _i32]),
    "afc_plan_get_cached": (_i32, [ctypes.POINTER(_vp), _i32, _pi64, _i32, _i32, _i64, _i32]),
    "afc_plan_destroy": (_i32, [_vp]),
    "afc_execute": (_i32, [_vp, _vp, _vp, _i32, _vp]),
    "afc_execute_scaled": (_i32, [_vp, _vp, _vp, _i32, _dbl, _vp]),
    "afc_execute_adjoint": (_i32, [_vp, _vp, _vp, _i32, _vp]),
    "afc_execute_host": (_i32, [_vp, _vp, _vp, _i32]),
    "afc_workspace_size": (_i32, [_vp, ctypes.POINTER(_sz)]),
    "afc_execute_ws": (_i32, [_vp, _vp, _vp, _i32, _dbl, _i32, _vp, _sz, _vp]),
    "afc_plan_io_elems": (_i32, [_vp, _i32, _pi64, _pi64]),
    "afc_batch_plan_create": (_i32, [ctypes.POINTER(_vp), _pi64, _i64, _i32, _i32]),
    "afc_batch_plan_destroy": (_i32, [_vp]),
    "afc_batch_execute": (_i32, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "afc_batch_total_elems": (_i32, [_vp, _pi64]),
    "afc_capabilities": (_i32, [ctypes.POINTER(Capabilities)]),
    "afc_length_info": (_i32, [_u64, ctypes.POINTER(LengthInfo)]),
    "afc_rader_maps": (_i32, [_u64, _pu64, _pu64]),
    "afc_pfa_perm": (_i32, [_u64, _u64, _pu64, _pu64]),
    "afc_plan_describe": (_i32, [_vp, _i32, ctypes.POINTER(LengthInfo)]),
    "afc_last_error_message": (ctypes.c_char_p, []),
    "afc_kernel_launch_count": (_u64, []),
    "afc_execute_1d_no_alloc": (_i32, [_vp, _vp, _vp, _i32, _vp]),
    "afc_stft_frame_count": (_i32, [_i64, _i64, _i64, _pi64]),
    "afc_stft_forward": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp]),
    "afc_stft_inverse_workspace": (_i32, [_vp, _i64, _i64, ctypes.POINTER(_sz)]),
    "afc_stft_inverse": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _sz, _vp]),
    "afc_czt_plan_create": (_i32, [ctypes.POINTER(_vp), _i64, _i64, _dbl, _dbl, _dbl, _dbl, _i32, _i32]),
    "afc_czt_execute": (_i32, [_vp, _vp, _vp, _i64, _vp]),
    "afc_czt_inverse": (_i32, [_vp, _vp, _vp, _i64, _vp]),
    "afc_czt_conv_len": (_i32, [_vp, _pi64]),
    "afc_czt_plan_destroy": (_i32, [_vp]),
    "afc_hilbert_plan_create": (_i32, [ctypes.POINTER(_vp), _i64, _i32, _i32]),
    "afc_hilbert_analytic": (_i32, [_vp, _vp, _vp, _i64, _vp]),
    "afc_hilbert_plan_destroy": (_i32, [_vp]),
    "afc_nufft1d_plan_create": (_i32, [ctypes.POINTER(_vp), _i64, _dbl, _i64, _i64, _i32]),
    "afc_nufft1d_type1": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "afc_nufft1d_type2": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "afc_nufft_plan_destroy": (_i32, [_vp]),
    "afc_nufft3d_plan_create": (_i32, [ctypes.POINTER(_vp), _i64, _i64, _i64, _dbl, _dbl, _dbl, _i64, _i64, _i32]),
    "afc_nufft3d_grid_dims": (_i32, [_vp, ctypes.POINTER(_i64)]),
    "afc_nufft3d_type1": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "afc_nufft3d_type2": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "afc_nufft3d_plan_destroy": (_i32, [_vp]),
    "afc_nudft1d_type1": (_i32, [_vp, _vp, _i64, _i64, _dbl, _vp, _i32, _vp]),
    "afc_nudft1d_type2": (_i32, [_vp, _i64, _vp, _i64, _dbl, _vp, _i32, _vp]),
    "afc_nudft3d_type1": (_i32, [_vp, _vp, _i64, _i64, _i64, _i64, _dbl, _dbl, _dbl, _vp, _i32, _vp]),
}

_lib = None


def lib():
    """Loads the CUDA library (raises ImportError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"apollofft_b200: {LIB_PATH} is missing; build it with `python -m apollofft_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L.afc_test_fail_next_allocs.restype = None
        L.afc_test_fail_next_allocs.argtypes = [ctypes.c_int]
        L.afc_test_tc_tile.restype = ctypes.c_int
        L.afc_test_tc_tile.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.afc_test_take_device_error.restype = ctypes.c_int
        L.afc_test_take_device_error.argtypes = []
        L.afc_test_bounded_wait.restype = ctypes.c_int
        L.afc_test_bounded_wait.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().afc_last_error_message()
    return msg.decode() if msg else ""


def check(status: int, what: str = "") -> None:
    """Raises ValueError for validation-type failures (like the reference's
    PyValueError), AfcError for device / memory / timeout failures."""
    if status == AFC_OK:
        return
    msg = last_error()
    if what:
        msg = f"{what}: {msg}"
    if status in (AFC_ERR_VALIDATION, AFC_ERR_SHAPE_MISMATCH, AFC_ERR_NON_CONTIGUOUS):
        raise ValueError(msg)
    raise AfcError(status, msg)


def length_info(n: int) -> dict:
    info = LengthInfo()
    check(lib().afc_length_info(n, ctypes.byref(info)), "length_info")
    return _info_dict(info)


def _info_dict(info: LengthInfo) -> dict:
    return {
        "strategy": STRATEGY_NAMES[info.strategy],
        "radices": None if info.n_radices < 0 else [int(info.radices[i]) for i in range(info.n_radices)],
        "coprime": (int(info.coprime_n1), int(info.coprime_n2)) if info.coprime_n1 else None,
        "four_step": (int(info.four_step_n1), int(info.four_step_n2)) if info.four_step_n1 else None,
        "primitive_root": int(info.primitive_root) if info.is_prime else None,
        "primitive_root_inv": int(info.primitive_root_inv) if info.is_prime else None,
        "is_prime": bool(info.is_prime),
        "is_short_winograd": bool(info.is_short_winograd),
        "has_static_coprime_codelet": bool(info.has_static_coprime_codelet),
        "gpu_algo": ALGO_NAMES[info.gpu_algo],
        "gpu_radices": [int(info.gpu_radices[i]) for i in range(info.gpu_n_radices)],
        "gpu_conv_len": int(info.gpu_conv_len),
        "gpu_split": (int(info.gpu_split_n1), int(info.gpu_split_n2)),
    }


def rader_maps(p: int):
    import numpy as np
    g = (ctypes.c_uint64 * (p - 1))()
    s = (ctypes.c_uint64 * (p - 1))()
    check(lib().afc_rader_maps(p, g, s), "rader_maps")
    return (np.frombuffer(g, dtype=np.uint64).astype(np.int64),
            np.frombuffer(s, dtype=np.uint64).astype(np.int64))


def pfa_perm(n1: int, n2: int):
    import numpy as np
    n = n1 * n2
    a = (ctypes.c_uint64 * n)()
    b = (ctypes.c_uint64 * n)()
    check(lib().afc_pfa_perm(n1, n2, a, b), "pfa_perm")
    return (np.frombuffer(a, dtype=np.uint64).astype(np.int64),
            np.frombuffer(b, dtype=np.uint64).astype(np.int64))


def capabilities() -> dict:
    c = Capabilities()
    check(lib().afc_capabilities(ctypes.byref(c)), "capabilities")
    return {f: getattr(c, f) for f, _ in Capabilities._fields_}


def kernel_launch_count() -> int:
    return int(lib().afc_kernel_launch_count())
