"""ctypes view of the CPU oracle (oracle/apollo_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The apollofft_b200 library never
imports it.  The oracle restates apollo-fft's CPU plans (f64 `high_accuracy`
and f32 `low_precision`) and its integer maps; see apollo_oracle.cpp for the
reference file:line each function follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libapollo_oracle.so")
_lib = None

# Strategy codes of the reference dispatcher (mixed_radix/dispatch.rs:26-82).
STRATEGY_NAMES = {
    0: "noop", 1: "stockham", 2: "four_step", 3: "winograd", 4: "pfa_static",
    5: "composite", 6: "pfa_generic", 7: "rader_full", 8: "rader_half", 9: "untransformed",
}


def build() -> str:
    """Compile the oracle shared library (make, g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        u64, i32, dbl, i64 = ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_int64
        pu64 = ctypes.POINTER(ctypes.c_uint64)
        vp = ctypes.c_void_p
        sig = {
            "or_factorize_composite": (i32, [u64, pu64, i32]),
            "or_lower_radix4": (i32, [pu64, i32, pu64]),
            "or_prime23_radices": (i32, [u64, pu64, i32]),
            "or_coprime_factors": (i32, [u64, pu64, pu64]),
            "or_is_prime": (i32, [u64]),
            "or_prime_factors_all": (i32, [u64, pu64, i32]),
            "or_mod_pow": (u64, [u64, u64, u64]),
            "or_modular_inverse": (u64, [u64, u64]),
            "or_primitive_root": (u64, [u64]),
            "or_primitive_root_dynamic": (u64, [u64]),
            "or_inverse_mod": (u64, [u64, u64]),
            "or_generator_order": (None, [u64, u64, pu64]),
            "or_inverse_generator_order": (None, [u64, u64, pu64]),
            "or_pfa_perm": (None, [u64, u64, pu64, pu64]),
            "or_is_short_winograd": (i32, [u64]),
            "or_has_static_coprime_codelet": (i32, [u64, u64]),
            "or_dispatch_strategy": (i32, [u64]),
            "or_four_step_split": (None, [u64, pu64, pu64]),
            "or_twiddle_table_f64": (None, [u64, dbl, vp]),
            "or_fft1d_c128": (None, [vp, u64, u64, i32, i32]),
            "or_fft1d_c64": (None, [vp, u64, u64, i32, i32]),
            "or_dispatch_c128": (None, [vp, u64, i32, i32]),
            "or_dispatch_c64": (None, [vp, u64, i32, i32]),
            "or_fft2d_c128": (None, [vp, u64, u64, u64, i32, i32]),
            "or_fft2d_c64": (None, [vp, u64, u64, u64, i32, i32]),
            "or_fft3d_c128": (None, [vp, u64, u64, u64, i32, i32]),
            "or_fft3d_c64": (None, [vp, u64, u64, u64, i32, i32]),
            "or_fft_uneven_c64": (None, [vp, pu64, pu64, u64, i32, i32]),
            "or_fft_uneven_c128": (None, [vp, pu64, pu64, u64, i32, i32]),
            "or_direct_dft": (None, [vp, vp, u64, i32]),
            "or_max_threads": (i32, []),
            "or_nufft1d_type1": (None, [i64, dbl, i64, i64, vp, vp, i64, vp]),
            "or_nufft1d_type2": (None, [i64, dbl, i64, i64, vp, vp, i64, vp]),
            "or_nufft3d_type1": (None, [i64, i64, i64, dbl, dbl, dbl, i64, i64, vp, vp, i64, vp]),
            "or_nufft3d_type2": (None, [i64, i64, i64, dbl, dbl, dbl, i64, i64, vp, vp, i64, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _u64buf(n):
    return (ctypes.c_uint64 * max(n, 1))()


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


# ── integer layer ──────────────────────────────────────────────────────────

def factorize_composite(n: int):
    buf = _u64buf(64)
    c = lib().or_factorize_composite(n, buf, 64)
    return None if c < 0 else [int(buf[i]) for i in range(c)]


def lower_radix2_pairs_to_radix4(radices):
    inp = (ctypes.c_uint64 * max(len(radices), 1))(*radices)
    out = _u64buf(len(radices) + 1)
    c = lib().or_lower_radix4(inp, len(radices), out)
    return [int(out[i]) for i in range(c)]


def prime23_radices(n: int):
    buf = _u64buf(64)
    c = lib().or_prime23_radices(n, buf, 64)
    return None if c < 0 else [int(buf[i]) for i in range(c)]


def coprime_factors(n: int):
    a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
    ok = lib().or_coprime_factors(n, ctypes.byref(a), ctypes.byref(b))
    return (int(a.value), int(b.value)) if ok else None


def is_prime(n: int) -> bool:
    return bool(lib().or_is_prime(n))


def prime_factors_all(n: int):
    buf = _u64buf(64)
    c = lib().or_prime_factors_all(n, buf, 64)
    return [int(buf[i]) for i in range(c)]


def mod_pow(b, e, m):
    return int(lib().or_mod_pow(b, e, m))


def modular_inverse(a, m):
    return int(lib().or_modular_inverse(a, m))


def primitive_root(p):
    return int(lib().or_primitive_root(p))


def primitive_root_dynamic(p):
    return int(lib().or_primitive_root_dynamic(p))


def inverse_mod(a, m):
    return int(lib().or_inverse_mod(a, m))


def generator_order(p, g):
    buf = _u64buf(p - 1)
    lib().or_generator_order(p, g, buf)
    return np.frombuffer(buf, dtype=np.uint64, count=p - 1).astype(np.int64)


def inverse_generator_order(p, g):
    buf = _u64buf(p - 1)
    lib().or_inverse_generator_order(p, g, buf)
    return np.frombuffer(buf, dtype=np.uint64, count=p - 1).astype(np.int64)


def pfa_perm(n1, n2):
    n = n1 * n2
    a, b = _u64buf(n), _u64buf(n)
    lib().or_pfa_perm(n1, n2, a, b)
    return (np.frombuffer(a, dtype=np.uint64, count=n).astype(np.int64),
            np.frombuffer(b, dtype=np.uint64, count=n).astype(np.int64))


def is_short_winograd(n):
    return bool(lib().or_is_short_winograd(n))


def has_static_coprime_codelet(n1, n2):
    return bool(lib().or_has_static_coprime_codelet(n1, n2))


def dispatch_strategy(n) -> str:
    return STRATEGY_NAMES[lib().or_dispatch_strategy(n)]


def four_step_split(n):
    a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
    lib().or_four_step_split(n, ctypes.byref(a), ctypes.byref(b))
    return int(a.value), int(b.value)


def twiddle_table(n, sign=-1.0):
    out = np.zeros(max(n - 1, 0), dtype=np.complex128)
    if n > 1:
        lib().or_twiddle_table_f64(n, sign, _ptr(out))
    return out


# ── float layer ────────────────────────────────────────────────────────────

def _prep(x, dtype):
    a = np.ascontiguousarray(x, dtype=dtype).copy()
    return a


def fft1d(x, inverse=False, threads=0):
    """Plan-level 1D transform over the last axis (forward unnormalized,
    inverse 1/N), complex128 -> f64 plan, complex64 -> f32 plan."""
    x = np.asarray(x)
    dt = np.complex64 if x.dtype == np.complex64 else np.complex128
    a = _prep(x, dt)
    n = a.shape[-1]
    lanes = a.size // n if n else 0
    if a.size:
        fn = lib().or_fft1d_c64 if dt == np.complex64 else lib().or_fft1d_c128
        fn(_ptr(a), n, lanes, int(inverse), threads)
    return a


def dispatch(x, inverse=False, normalize=False):
    """Single-lane dispatch_inplace (unnormalized unless `normalize`)."""
    x = np.asarray(x)
    dt = np.complex64 if x.dtype == np.complex64 else np.complex128
    a = _prep(x, dt)
    fn = lib().or_dispatch_c64 if dt == np.complex64 else lib().or_dispatch_c128
    fn(_ptr(a), a.size, int(inverse), int(normalize))
    return a


def fft2d(x, inverse=False, threads=0):
    """FftPlan2D over the last two axes (leading axes are a batch)."""
    x = np.asarray(x)
    dt = np.complex64 if x.dtype == np.complex64 else np.complex128
    a = _prep(x, dt)
    nx, ny = a.shape[-2], a.shape[-1]
    batch = a.size // (nx * ny)
    fn = lib().or_fft2d_c64 if dt == np.complex64 else lib().or_fft2d_c128
    fn(_ptr(a), nx, ny, batch, int(inverse), threads)
    return a


def fft3d(x, inverse=False, threads=0):
    """FftPlan3D on a (nx, ny, nz) array."""
    x = np.asarray(x)
    dt = np.complex64 if x.dtype == np.complex64 else np.complex128
    a = _prep(x, dt)
    nx, ny, nz = a.shape
    fn = lib().or_fft3d_c64 if dt == np.complex64 else lib().or_fft3d_c128
    fn(_ptr(a), nx, ny, nz, int(inverse), threads)
    return a


def fft_uneven(packed, offsets, lengths, inverse=False, threads=0):
    """Per-length dispatch over lanes packed back to back (uneven batch)."""
    packed = np.asarray(packed)
    dt = np.complex64 if packed.dtype == np.complex64 else np.complex128
    a = _prep(packed, dt)
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    ln = np.ascontiguousarray(lengths, dtype=np.uint64)
    fn = lib().or_fft_uneven_c64 if dt == np.complex64 else lib().or_fft_uneven_c128
    fn(_ptr(a), off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
       ln.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(ln), int(inverse), threads)
    return a


def direct_dft(x, inverse=False):
    """Long-double direct DFT (kernel/direct.rs:147-244 restated), independent truth."""
    a = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.zeros_like(a)
    lib().or_direct_dft(_ptr(a), _ptr(out), a.size, int(inverse))
    return out


def max_threads() -> int:
    return int(lib().or_max_threads())
