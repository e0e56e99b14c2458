"""ctypes binding of lib/libsfntt.so (declared in include/sfntt.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parents[1]
LIB_PATH = Path(os.environ.get("SFNTT_LIB", PKG_ROOT / "lib" / "libsfntt.so"))

u32, u64, sz, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
vp = ctypes.c_void_p
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)

# name -> (restype, argtypes); mirrors include/sfntt.h one to one
SIGNATURES = {
    "sfntt_ctx_create": (i32, [i32, ctypes.POINTER(vp)]),
    "sfntt_ctx_destroy": (None, [vp]),
    "sfntt_status_string": (ctypes.c_char_p, [i32]),
    "sfntt_last_error": (ctypes.c_char_p, [vp]),
    "sfntt_device_info": (i32, [vp, ctypes.c_char_p, sz]),
    "sfntt_forward": (i32, [vp, i32, i32, u32p, sz, u64p]),
    "sfntt_inverse": (i32, [vp, i32, i32, u32p, sz, u64p]),
    "sfntt_pointwise_mul": (i32, [vp, i32, u32p, sz, u32p, sz, u32p, sz]),
    "sfntt_forward_gpu": (i32, [vp, i32, i32, u32p, sz, u32, u32p, u64p]),
    "sfntt_inverse_gpu": (i32, [vp, i32, i32, u32p, sz, u32, u32p, u64p]),
    "sfntt_forward_batch": (i32, [vp, i32, u32p, sz, u32, u32, u32p, u64p]),
    "sfntt_inverse_batch": (i32, [vp, i32, u32p, sz, u32, u32, u32p, u64p]),
    "sfntt_bb_coset_lde": (i32, [vp, u32p, sz, u32, u32, u32, u32, i32, u32p, u64p]),
    "sfntt_m31_lde": (i32, [vp, u32p, sz, u32, u32, u32, u32p, u64p]),
    "sfntt_prepare": (i32, [vp, i32, u32]),
    "sfntt_prepare_lde": (i32, [vp, i32, u32, u32, u32]),
    "sfntt_forward_dev": (i32, [vp, i32, i32, vp, u32, u32, vp]),
    "sfntt_inverse_dev": (i32, [vp, i32, i32, vp, u32, u32, vp]),
    "sfntt_bb_coset_lde_dev": (i32, [vp, vp, vp, u32, u32, u32, u32, i32, vp]),
    "sfntt_m31_lde_dev": (i32, [vp, vp, vp, u32, u32, u32, vp]),
    "sfntt_coset_lde": (i32, [vp, i32, u32p, sz, u32, u32, u32, u32, i32, u32p, u64p]),
    "sfntt_coset_lde_dev": (i32, [vp, i32, vp, vp, u32, u32, u32, u32, i32, vp]),
    "sfntt_to_monty_dev": (i32, [vp, i32, vp, sz, vp]),
    "sfntt_circle_ntt": (i32, [vp, i32, u32p, sz, u32, u32, u32p, u64p]),
    "sfntt_circle_lde": (i32, [vp, u32p, sz, u32, u32, u32, u32p, u64p]),
    "sfntt_prepare_circle": (i32, [vp, u32, u32]),
    "sfntt_circle_ntt_dev": (i32, [vp, i32, vp, u32, u32, vp]),
    "sfntt_circle_lde_dev": (i32, [vp, vp, vp, u32, u32, u32, vp]),
    "sfntt_cm31_prepare": (i32, [vp, u32, u32]),
    "sfntt_cm31_ntt_dev": (i32, [vp, i32, vp, u32, u32, vp]),
    "sfntt_cm31_ntt": (i32, [vp, i32, u32p, sz, u32, u32, u32p, u64p]),
    "sfntt_cm31_mul_dev": (i32, [vp, vp, vp, vp, sz, vp]),
    "sfntt_from_monty_dev": (i32, [vp, i32, vp, sz, vp]),
    "sfntt_bb_to_monty_dev": (i32, [vp, vp, sz, vp]),
    "sfntt_layout_dev": (i32, [vp, vp, vp, u32, u32, i32, vp]),
    "sfntt_selftest_bounded_wait": (i32, [vp, u64, i32]),
    "sfntt_layout": (i32, [vp, u32p, sz, u32, u32, i32, u32p, u64p]),
    "sfntt_bb_from_monty_dev": (i32, [vp, vp, sz, vp]),
    "sfntt_stockham_noalloc": (i32, [vp, i32, i32, vp, u32, u32, vp]),
    "sfntt_batch_prepare": (i32, [vp, vp, sz]),
    "sfntt_batch_run": (i32, [vp, vp, sz, vp]),
    "sfntt_batch_graph_create": (i32, [vp, vp, sz, i32, ctypes.POINTER(vp)]),
    "sfntt_batch_persistent_create": (i32, [vp, vp, sz, i32, ctypes.POINTER(vp)]),
    "sfntt_graph_launch": (i32, [vp, vp]),
    "sfntt_graph_kernel_count": (u64, [vp]),
    "sfntt_graph_destroy": (None, [vp]),
    "sfntt_autotune": (i32, [vp, vp, sz, i32]),
    "sfntt_tune_save": (i32, [vp, ctypes.c_char_p]),
    "sfntt_tune_load": (i32, [vp, ctypes.c_char_p]),
    "sfntt_tune_lookup": (i32, [vp, vp]),
    "sfntt_server_create": (i32, [vp, sz, i32, ctypes.POINTER(vp)]),
    "sfntt_server_destroy": (None, [vp]),
    "sfntt_server_submit": (i32, [vp, vp, u64p]),
    "sfntt_server_submit_host": (i32, [vp, vp, vp, vp, u64p]),
    "sfntt_server_poll": (i32, [vp, u64p, sz, ctypes.POINTER(sz)]),
    "sfntt_server_result": (i32, [vp, u64, ctypes.POINTER(vp)]),
    "sfntt_server_release": (i32, [vp, u64]),
    "sfntt_server_pending": (sz, [vp]),
    "sfntt_server_set_packing": (i32, [vp, i32]),
    "sfntt_server_launches": (u64, [vp]),
    "sfntt_serve_trace": (i32, [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_double), sz, i32, sz,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "sfntt_serve_trace_packed": (i32, [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_double), sz, i32, i32, sz,
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), u64p]),
    "sfntt_host_alloc": (i32, [vp, sz, ctypes.POINTER(vp)]),
    "sfntt_host_free": (i32, [vp, vp]),
    "sfntt_launch_count": (u64, [vp]),
    "sfntt_check_device_error": (i32, [vp]),
    "sfntt_kernel_timing": (i32, [vp, i32]),
    "sfntt_kernel_times": (i32, [vp, ctypes.c_char_p, sz]),
    "sfntt_butterfly_peak": (i32, [vp, i32, ctypes.POINTER(ctypes.c_double)]),
}

class LdeItem(ctypes.Structure):
    """sfntt_lde_item (include/sfntt.h)."""
    _fields_ = [("field", ctypes.c_int), ("log_n", ctypes.c_uint32), ("batch", ctypes.c_uint32),
                ("added_bits", ctypes.c_uint32), ("shift_monty", ctypes.c_uint32),
                ("d_in", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("plan", ctypes.c_int)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C small-field-metal-ntt_b200` "
                          "(there is no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
