"""ctypes wrapper around oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle is a plain-C restatement of the reference's CPU NTT / coset-LDE
path (see oracle.h for the file:line map).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference legs import this module, and only as
the checker or the timed CPU baseline.  The product library never uses it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

BB_P = 2013265921
M31_P = 2147483647
KB_P = 2130706433  # KoalaBear, 2^31 - 2^24 + 1 (no reference implementation)

_u32p = ctypes.POINTER(ctypes.c_uint32)
_lib = None


class CPoint(ctypes.Structure):
    """orc_cpoint: a point (x, y) of the circle x^2 + y^2 = 1 over M31."""
    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32)]


def build() -> Path:
    """Compile liboracle.so with the committed Makefile (no-op when fresh)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        u32, u64, sz, i = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
        sig = {
            "orc_bb_monty_reduce": (u32, [u64]),
            "orc_bb_to_monty": (u32, [u32]),
            "orc_bb_from_monty": (u32, [u32]),
            "orc_bb_add": (u32, [u32, u32]),
            "orc_bb_sub": (u32, [u32, u32]),
            "orc_bb_mul": (u32, [u32, u32]),
            "orc_bb_reduce": (u32, [u64]),
            "orc_bb_inv": (u32, [u32]),
            "orc_bb_two_adic_generator": (u32, [u32]),
            "orc_m31_reduce": (u32, [u64]),
            "orc_m31_add": (u32, [u32, u32]),
            "orc_m31_sub": (u32, [u32, u32]),
            "orc_m31_mul": (u32, [u32, u32]),
            "orc_m31_inv": (u32, [u32]),
            "orc_circle_add": (CPoint, [CPoint, CPoint]),
            "orc_circle_double": (CPoint, [CPoint]),
            "orc_circle_mul_scalar": (CPoint, [CPoint, u32]),
            "orc_circle_subgroup_gen": (CPoint, [u32]),
            "orc_bb_twiddles": (None, [u32, i, _u32p]),
            "orc_m31_twiddles": (None, [u32, i, _u32p]),
            "orc_bb_forward": (i, [_u32p, sz]),
            "orc_bb_inverse": (i, [_u32p, sz]),
            "orc_m31_forward": (i, [_u32p, sz]),
            "orc_m31_inverse": (i, [_u32p, sz]),
            "orc_bb_coset_lde": (i, [_u32p, _u32p, u32, u32, u32, u32, i]),
            "orc_m31_lde": (i, [_u32p, _u32p, u32, u32, u32, i]),
            "orc_bb_forward_batch": (i, [_u32p, u32, u32, i]),
            "orc_bb_inverse_batch": (i, [_u32p, u32, u32, i]),
            "orc_lcg_fill": (u64, [_u32p, sz, u64, u32, i]),
            "orc_circle_twiddles": (None, [u32, i, _u32p]),
            "orc_circle_ntt": (i, [_u32p, u32, u32, i]),
            "orc_circle_lde": (i, [_u32p, _u32p, u32, u32, u32, i]),
            "orc_cm31_mul": (None, [_u32p, _u32p, _u32p, sz]),
            "orc_cm31_ntt": (i, [_u32p, u32, u32, i]),
            "orc_kb_to_monty": (u32, [u32]),
            "orc_kb_from_monty": (u32, [u32]),
            "orc_kb_mul": (u32, [u32, u32]),
            "orc_kb_two_adic_generator": (u32, [u32]),
            "orc_kb_twiddles": (None, [u32, i, _u32p]),
            "orc_kb_forward": (i, [_u32p, sz]),
            "orc_kb_inverse": (i, [_u32p, sz]),
            "orc_kb_forward_batch": (i, [_u32p, u32, u32, i]),
            "orc_kb_inverse_batch": (i, [_u32p, u32, u32, i]),
            "orc_kb_coset_lde": (i, [_u32p, _u32p, u32, u32, u32, u32, i]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def _arr(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32))


class InvalidSize(ValueError):
    pass


# ---- field scalars ---------------------------------------------------------
def bb_to_monty(v: int) -> int: return lib().orc_bb_to_monty(v)
def bb_from_monty(m: int) -> int: return lib().orc_bb_from_monty(m)
def bb_add(a, b): return lib().orc_bb_add(a, b)
def bb_sub(a, b): return lib().orc_bb_sub(a, b)
def bb_mul(a, b): return lib().orc_bb_mul(a, b)
def bb_inv(a): return lib().orc_bb_inv(a)
def bb_reduce(v): return lib().orc_bb_reduce(v)
def bb_monty_reduce(t): return lib().orc_bb_monty_reduce(t)
def bb_two_adic_generator(k): return lib().orc_bb_two_adic_generator(k)
def kb_to_monty(v: int) -> int: return lib().orc_kb_to_monty(v)
def kb_from_monty(m: int) -> int: return lib().orc_kb_from_monty(m)
def kb_mul(a, b): return lib().orc_kb_mul(a, b)
def kb_two_adic_generator(k): return lib().orc_kb_two_adic_generator(k)
def m31_add(a, b): return lib().orc_m31_add(a, b)
def m31_sub(a, b): return lib().orc_m31_sub(a, b)
def m31_mul(a, b): return lib().orc_m31_mul(a, b)
def m31_inv(a): return lib().orc_m31_inv(a)
def m31_reduce(v): return lib().orc_m31_reduce(v)


def bb_to_monty_array(v) -> np.ndarray:
    return np.array([bb_to_monty(int(x)) for x in np.asarray(v).ravel()], dtype=np.uint32)


def bb_from_monty_array(v) -> np.ndarray:
    return np.array([bb_from_monty(int(x)) for x in np.asarray(v).ravel()], dtype=np.uint32)


# ---- twiddles ----------------------------------------------------------------
def bb_twiddles(log_n: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(max((1 << log_n) - 1, 1), dtype=np.uint32)
    lib().orc_bb_twiddles(log_n, int(inverse), _ptr(out))
    return out[: (1 << log_n) - 1]


def kb_twiddles(log_n: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(max((1 << log_n) - 1, 1), dtype=np.uint32)
    lib().orc_kb_twiddles(log_n, int(inverse), _ptr(out))
    return out[: (1 << log_n) - 1]


def m31_twiddles(log_n: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(max((1 << log_n) - 1, 1), dtype=np.uint32)
    lib().orc_m31_twiddles(log_n, int(inverse), _ptr(out))
    return out[: (1 << log_n) - 1]


# ---- transforms (return new arrays) ----------------------------------------
def _one(fn, data) -> np.ndarray:
    a = _arr(data).copy()
    if fn(_ptr(a) if a.size else None, a.size) != 0:
        raise InvalidSize(a.size)
    return a


def bb_forward(data) -> np.ndarray: return _one(lib().orc_bb_forward, data)
def bb_inverse(data) -> np.ndarray: return _one(lib().orc_bb_inverse, data)
def kb_forward(data) -> np.ndarray: return _one(lib().orc_kb_forward, data)
def kb_inverse(data) -> np.ndarray: return _one(lib().orc_kb_inverse, data)
def m31_forward(data) -> np.ndarray: return _one(lib().orc_m31_forward, data)
def m31_inverse(data) -> np.ndarray: return _one(lib().orc_m31_inverse, data)


def _batch(fn, data, log_n: int, batch: int, threads: int) -> np.ndarray:
    a = _arr(data).copy()
    assert a.size == batch << log_n
    if fn(_ptr(a), log_n, batch, threads) != 0:
        raise InvalidSize(a.size)
    return a


def bb_forward_batch(data, log_n: int, batch: int, threads: int = 1) -> np.ndarray:
    return _batch(lib().orc_bb_forward_batch, data, log_n, batch, threads)


def bb_inverse_batch(data, log_n: int, batch: int, threads: int = 1) -> np.ndarray:
    return _batch(lib().orc_bb_inverse_batch, data, log_n, batch, threads)


def kb_forward_batch(data, log_n: int, batch: int, threads: int = 1) -> np.ndarray:
    return _batch(lib().orc_kb_forward_batch, data, log_n, batch, threads)


def kb_inverse_batch(data, log_n: int, batch: int, threads: int = 1) -> np.ndarray:
    return _batch(lib().orc_kb_inverse_batch, data, log_n, batch, threads)


def _coset_lde(fn, data, log_n, batch, added_bits, shift_monty, threads) -> np.ndarray:
    a = _arr(data)
    if a.size != batch << log_n:
        raise InvalidSize(a.size)
    out = np.empty(batch << (log_n + added_bits), dtype=np.uint32)
    if fn(_ptr(a), _ptr(out), log_n, batch, added_bits, shift_monty, threads) != 0:
        raise InvalidSize(a.size)
    return out


def bb_coset_lde(data, log_n: int, batch: int, added_bits: int, shift_monty: int = 0,
                 threads: int = 1) -> np.ndarray:
    return _coset_lde(lib().orc_bb_coset_lde, data, log_n, batch, added_bits, shift_monty, threads)


def kb_coset_lde(data, log_n: int, batch: int, added_bits: int, shift_monty: int = 0,
                 threads: int = 1) -> np.ndarray:
    """KoalaBear coset LDE: the BabyBear algorithm over KoalaBear (Montgomery
    u32 in and out; shift_monty 0 = two_adic_generator(log_n + added_bits + 1))."""
    return _coset_lde(lib().orc_kb_coset_lde, data, log_n, batch, added_bits, shift_monty, threads)


def m31_lde(data, log_n: int, batch: int, added_bits: int, threads: int = 1) -> np.ndarray:
    a = _arr(data)
    if a.size != batch << log_n:
        raise InvalidSize(a.size)
    out = np.empty(batch << (log_n + added_bits), dtype=np.uint32)
    if lib().orc_m31_lde(_ptr(a), _ptr(out), log_n, batch, added_bits, threads) != 0:
        raise InvalidSize(a.size)
    return out


def circle_twiddles(log_n: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(max((1 << log_n) - 1, 1), dtype=np.uint32)
    lib().orc_circle_twiddles(log_n, int(inverse), _ptr(out))
    return out[: (1 << log_n) - 1]


def circle_ntt(data, log_n: int, batch: int = 1, inverse: bool = False) -> np.ndarray:
    """Canonic-coset circle FFT (evaluate) / its inverse (interpolate, times n^-1)."""
    a = _arr(data).copy()
    if a.size != batch << log_n or lib().orc_circle_ntt(_ptr(a) if a.size else None, log_n, batch,
                                                           int(inverse)) != 0:
        raise InvalidSize(a.size)
    return a


def circle_lde(data, log_n: int, batch: int, added_bits: int, threads: int = 1) -> np.ndarray:
    a = _arr(data)
    if a.size != batch << log_n:
        raise InvalidSize(a.size)
    out = np.empty(batch << (log_n + added_bits), dtype=np.uint32)
    if lib().orc_circle_lde(_ptr(a), _ptr(out), log_n, batch, added_bits, threads) != 0:
        raise InvalidSize(a.size)
    return out


def cm31_mul(a, b) -> np.ndarray:
    """CM31 products of interleaved (re, im) pairs."""
    a_, b_ = _arr(a), _arr(b)
    assert a_.size == b_.size and a_.size % 2 == 0
    out = np.empty_like(a_)
    lib().orc_cm31_mul(_ptr(a_), _ptr(b_), _ptr(out), a_.size // 2)
    return out


def cm31_ntt(pairs, log_n: int, batch: int, inverse: bool = False) -> np.ndarray:
    """Circle NTT of `batch` CM31 columns of 2^log_n interleaved pairs."""
    a = _arr(pairs).copy()
    if a.size != 2 * (batch << log_n):
        raise InvalidSize(a.size)
    if lib().orc_cm31_ntt(_ptr(a), log_n, batch, int(inverse)) != 0:
        raise InvalidSize(a.size)
    return a


def lcg(n: int, seed: int, p: int, monty: bool = False) -> np.ndarray:
    """The reference LCG (src/ntt/test_utils.rs:38-46): values (s>>33) % p,
    in p's Montgomery form when `monty` (BabyBear or KoalaBear by p)."""
    out = np.empty(n, dtype=np.uint32)
    if n:
        lib().orc_lcg_fill(_ptr(out), n, seed, p, (2 if p == KB_P else 1) if monty else 0)
    return out


def default_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1
