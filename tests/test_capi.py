"""CPU-side checks of the C ABI: the library loads, exports every function
include/sfntt.h declares, and reports a missing device as the reference's
NttError::DeviceNotFound.  No compute call is made without a GPU."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "sfntt.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sfntt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("sfntt_ctx_create", "sfntt_forward", "sfntt_inverse", "sfntt_pointwise_mul",
                 "sfntt_forward_batch", "sfntt_bb_coset_lde", "sfntt_bb_coset_lde_dev"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from sfntt import _ffi
    lib = _ffi.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in _ffi.SIGNATURES, f"{name} lacks a ctypes signature"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_ffi.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (sfntt_\w+)", out))
    assert set(declared_functions()) <= exported


def test_library_is_built_for_sm100a():
    """Every object of the library is compiled with the sm_100a target only
    (no PTX to JIT elsewhere): the Makefile passes one -gencode, and every
    compile and the link use it."""
    mk = (ROOT / "small-field-metal-ntt_b200" / "Makefile").read_text()
    arch = re.search(r"^ARCH\s*:=\s*(.+)$", mk, flags=re.M)
    assert arch and arch.group(1).strip() == "-gencode arch=compute_100a,code=sm_100a"
    assert re.search(r"^NVFLAGS\s*\?=.*\$\(ARCH\)", mk, flags=re.M)
    assert "$(NVCC) $(NVFLAGS) -c" in mk and "$(NVCC) $(ARCH) -shared" in mk
    assert "compute_" not in mk.replace("compute_100a", "")


def test_status_strings_and_no_device_path():
    from sfntt import _ffi
    import sfntt
    lib = _ffi.lib()
    assert lib.sfntt_status_string(0) == b"ok"
    assert lib.sfntt_status_string(1) == b"invalid size"
    assert lib.sfntt_status_string(7) == b"unsupported operation"
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the no-device path is not reachable")
    h = ctypes.c_void_p()
    assert lib.sfntt_ctx_create(0, ctypes.byref(h)) == 2  # SFNTT_DEVICE_NOT_FOUND
    with pytest.raises(sfntt.DeviceNotFound):
        sfntt.Context(0)
    # null context is rejected, not dereferenced
    assert lib.sfntt_forward(None, 1, 0, None, 0, None) == 9
    assert lib.sfntt_launch_count(None) == 0
