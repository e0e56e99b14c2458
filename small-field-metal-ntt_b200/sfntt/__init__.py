"""sfntt -- Python mirror of the reference's NTT / coset-LDE API over libsfntt.so.

The reference (moven0831/small-field-metal-ntt) exposes, in Rust:
  * trait NttBackend<F> { name, forward_ntt, inverse_ntt, pointwise_mul }
    (src/ntt/mod.rs:26-49) and the NttError enum (src/ntt/mod.rs:52-69);
  * per-variant backends V1..V4 for M31 and BabyBear with inherent
    forward_ntt_gpu / inverse_ntt_gpu (e.g. src/ntt/babybear/metal_ct_gs_r4.rs:87-172);
  * BbBatchNtt::forward_ntt_batch_gpu / inverse_ntt_batch_gpu
    (src/ntt/babybear/batch.rs:76-180);
  * CosetLdeBatch::new / execute -> LdeResult { data, total_ns } (src/lde/mod.rs:15-107).
This module provides the same names, argument meanings and error behaviour on
top of the CUDA library.  Field elements are numpy uint32 arrays holding the
reference's raw representation (M31 canonical, BabyBear Montgomery form).
The reference type names (MetalCtGsR4, BbMetalCtGsR4, ...) are kept as aliases
so that code written against the reference switches by import only.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _ffi

M31_P = 2147483647
BB_P = 2013265921
KB_P = 2130706433  # KoalaBear, 2^31 - 2^24 + 1
FIELD_M31 = 0
FIELD_BABYBEAR = 1
FIELD_KOALABEAR = 2  # planned in the reference (README.md:20); Montgomery u32 like BabyBear
BEST, V1, V2, V3, V4 = 0, 1, 2, 3, 4
LDE_FUSED, LDE_UNFUSED = 0, 1
LDE_NATURAL = 2  # flag: natural-order input and output rows (Plonky3's coset_lde_batch)
LAYOUT_NATURAL, LAYOUT_ROW_MAJOR = 1, 2


# --------------------------------------------------------------- errors ---
class NttError(Exception):
    """NttError (src/ntt/mod.rs:52-69)."""
    status = -1


class InvalidSize(NttError):
    status = 1

    def __init__(self, size: int, detail: str = ""):
        self.size = size
        super().__init__(f"Invalid NTT size: {size} (must be power of 2){': ' + detail if detail else ''}")


class DeviceNotFound(NttError):
    status = 2


class BufferAllocFailed(NttError):
    status = 3

    def __init__(self, msg: str = "", requested_bytes: int | None = None):
        self.requested_bytes = requested_bytes
        super().__init__(msg)


class ShaderCompileError(NttError):
    """No loadable sm_100a kernel image for this device (the reference's
    runtime shader-compilation failure)."""
    status = 4


class GpuExecutionError(NttError):
    status = 5


class CorrectnessMismatch(NttError):
    status = 6

    def __init__(self, index: int, expected: int, got: int):
        self.index, self.expected, self.got = index, expected, got
        super().__init__(f"Correctness mismatch at index {index}: expected {expected}, got {got}")


class Unsupported(NttError):
    """The reference panics here (V1 inverse is todo!())."""
    status = 7


class Timeout(NttError):
    status = 8


class InvalidArgument(NttError):
    status = 9


_ERRORS = {1: InvalidSize, 2: DeviceNotFound, 3: BufferAllocFailed, 4: ShaderCompileError,
           5: GpuExecutionError, 7: Unsupported, 8: Timeout, 9: InvalidArgument}


def _check(ctx, status: int, size: int = 0) -> None:
    if status == 0:
        return
    L = _ffi.lib()
    detail = L.sfntt_last_error(ctx).decode() if ctx else ""
    cls = _ERRORS.get(status, NttError)
    if cls is InvalidSize:
        raise InvalidSize(size, detail)
    raise cls(f"{L.sfntt_status_string(status).decode()}: {detail}")


# -------------------------------------------------------------- context ---
class Context:
    """A device context (the reference's MetalContext, src/gpu.rs:26-64):
    stream, device-resident twiddle caches and staging buffers."""

    def __init__(self, device: int = 0):
        L = _ffi.lib()
        h = ctypes.c_void_p()
        st = L.sfntt_ctx_create(device, ctypes.byref(h))
        if st != 0:
            cls = _ERRORS.get(st, NttError)
            raise cls(f"sfntt_ctx_create(device={device}): {L.sfntt_status_string(st).decode()}")
        self.handle = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            _ffi.lib().sfntt_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_info(self) -> str:
        buf = ctypes.create_string_buffer(256)
        _check(self.handle, _ffi.lib().sfntt_device_info(self.handle, buf, 256))
        return buf.value.decode()

    def check_device_error(self) -> int:
        """Status of the context's device error flag (SFNTT_TIMEOUT = 8 after a
        bounded wait ran out in a _dev call or graph), without raising."""
        return int(_ffi.lib().sfntt_check_device_error(self.handle))

    def launch_count(self) -> int:
        return int(_ffi.lib().sfntt_launch_count(self.handle))

    def kernel_timing(self, enable: bool = True) -> None:
        """Bracket every later launch with CUDA events (clears old records)."""
        _check(self.handle, _ffi.lib().sfntt_kernel_timing(self.handle, int(enable)))

    def butterfly_peak(self, gs: bool = True) -> float:
        """Measured butterflies/s with register-resident data (integer ceiling)."""
        out = ctypes.c_double()
        _check(self.handle, _ffi.lib().sfntt_butterfly_peak(self.handle, int(gs), ctypes.byref(out)))
        return out.value

    def kernel_times(self) -> dict:
        """{kernel: (launches, total_ms, algorithmic_bytes)} since kernel_timing()."""
        buf = ctypes.create_string_buffer(1 << 16)
        _check(self.handle, _ffi.lib().sfntt_kernel_times(self.handle, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, launches, ms, nbytes = line.split()
            out[name] = (int(launches), float(ms), int(nbytes))
        return out

    def selftest_bounded_wait(self, timeout_ns: int, arrive: bool) -> int:
        """Runs the tile engine's bounded mbarrier wait on a barrier that
        nothing arrives on (arrive=False) or that gets its arrival; returns
        the status (SFNTT_TIMEOUT = 8 or 0) without raising."""
        return int(_ffi.lib().sfntt_selftest_bounded_wait(self.handle, timeout_ns, int(arrive)))

    def prepare(self, field: int, log_n: int) -> None:
        _check(self.handle, _ffi.lib().sfntt_prepare(self.handle, field, log_n))

    def prepare_lde(self, field: int, log_n: int, added_bits: int, shift_monty: int = 0) -> None:
        _check(self.handle, _ffi.lib().sfntt_prepare_lde(self.handle, field, log_n, added_bits, shift_monty))

    def pinned(self, n: int) -> "PinnedBuffer":
        """Page-locked host buffer of n uint32 (full-bandwidth copies)."""
        return PinnedBuffer(self, n)


class PinnedBuffer:
    """Pinned host memory from sfntt_host_alloc; `.array` is a numpy view."""

    def __init__(self, ctx: Context, n: int):
        self.ctx = ctx
        p = ctypes.c_void_p()
        _check(ctx.handle, _ffi.lib().sfntt_host_alloc(ctx.handle, max(n, 1) * 4, ctypes.byref(p)))
        self.addr = p.value
        self.array = np.ctypeslib.as_array((ctypes.c_uint32 * max(n, 1)).from_address(self.addr))[:n]

    def free(self) -> None:
        if self.addr and self.ctx.handle:
            self.array = None
            _ffi.lib().sfntt_host_free(self.ctx.handle, ctypes.c_void_p(self.addr))
        self.addr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_DEFAULT: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    if device not in _DEFAULT:
        _DEFAULT[device] = Context(device)
    return _DEFAULT[device]


def _out_words(batch: int, log_n: int, added_bits: int) -> int:
    """Output length of an extension; 0 when the sizes are out of range, so
    that the library's own check reports InvalidSize."""
    return batch << (log_n + added_bits) if log_n + added_bits <= 40 else 0


def _u32(a) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.uint32))
    return arr


def _p(a: np.ndarray):
    return a.ctypes.data_as(_ffi.u32p) if a.size else None


# ------------------------------------------------------------- backends ---
class NttBackend:
    """trait NttBackend<F> (src/ntt/mod.rs:26-49), in place on uint32 arrays."""

    FIELD = FIELD_BABYBEAR
    VARIANT = BEST
    NAME = "cuda"

    def __init__(self, ctx: Context | None = None, device: int = 0):
        self.ctx = ctx or default_context(device)

    @classmethod
    def new(cls, shader_dir=None, device: int = 0):
        """Same shape as the reference's `new(shader_dir)`; the directory is
        not needed (kernels are compiled ahead of time for sm_100a)."""
        return cls(device=device)

    def name(self) -> str:
        return self.NAME

    def _inplace(self, fn, data) -> None:
        arr = data if isinstance(data, np.ndarray) and data.dtype == np.uint32 and data.flags["C_CONTIGUOUS"] \
            else None
        work = arr if arr is not None else _u32(data).copy()
        ns = ctypes.c_uint64()
        st = fn(self.ctx.handle, self.FIELD, self.VARIANT, _p(work), work.size, ctypes.byref(ns))
        _check(self.ctx.handle, st, work.size)
        if arr is None:
            data[:] = [int(v) for v in work]

    def forward_ntt(self, data, twiddles: Sequence[int] = ()) -> None:
        """Coefficients -> evaluations (bit-reversed order), in place.
        `twiddles` is ignored, as by every reference backend (src/ntt/mod.rs:33-36)."""
        self._inplace(_ffi.lib().sfntt_forward, data)

    def inverse_ntt(self, data, twiddles: Sequence[int] = ()) -> None:
        """Bit-reversed evaluations -> coefficients (x n^-1), in place."""
        self._inplace(_ffi.lib().sfntt_inverse, data)

    def pointwise_mul(self, a, b, out) -> None:
        a_, b_ = _u32(a), _u32(b)
        o = out if isinstance(out, np.ndarray) and out.dtype == np.uint32 and out.flags["C_CONTIGUOUS"] else None
        work = o if o is not None else np.empty(len(out), dtype=np.uint32)
        st = _ffi.lib().sfntt_pointwise_mul(self.ctx.handle, self.FIELD, _p(a_), a_.size, _p(b_), b_.size,
                                            _p(work), work.size)
        _check(self.ctx.handle, st, a_.size)
        if o is None:
            out[:] = [int(v) for v in work]

    def _gpu(self, fn, input, log_n: int):
        inp = _u32(input)
        out = np.empty_like(inp)
        ns = ctypes.c_uint64()
        st = fn(self.ctx.handle, self.FIELD, self.VARIANT, _p(inp), inp.size, log_n, _p(out), ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return out, int(ns.value)

    def forward_ntt_gpu(self, input, log_n: int):
        """-> (output, device ns) (src/ntt/babybear/metal_ct_gs_r4.rs:87-120)."""
        return self._gpu(_ffi.lib().sfntt_forward_gpu, input, log_n)

    def inverse_ntt_gpu(self, input, log_n: int):
        return self._gpu(_ffi.lib().sfntt_inverse_gpu, input, log_n)

    # batched SoA columns (BbBatchNtt, src/ntt/babybear/batch.rs:76-180)
    def _batch(self, fn, input, log_n: int, batch: int):
        inp = _u32(input)
        out = np.empty_like(inp)
        ns = ctypes.c_uint64()
        st = fn(self.ctx.handle, self.FIELD, _p(inp), inp.size, log_n, batch, _p(out), ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return out, int(ns.value)

    def forward_ntt_batch_gpu(self, input, log_n: int, batch: int):
        return self._batch(_ffi.lib().sfntt_forward_batch, input, log_n, batch)

    def inverse_ntt_batch_gpu(self, input, log_n: int, batch: int):
        return self._batch(_ffi.lib().sfntt_inverse_batch, input, log_n, batch)

    # device pointers (e.g. torch tensors' data_ptr()) on a CUDA stream handle
    def forward_dev(self, ptr: int, log_n: int, batch: int = 1, stream: int = 0) -> None:
        st = _ffi.lib().sfntt_forward_dev(self.ctx.handle, self.FIELD, self.VARIANT, ptr, log_n, batch, stream)
        _check(self.ctx.handle, st, batch << log_n)

    def inverse_dev(self, ptr: int, log_n: int, batch: int = 1, stream: int = 0) -> None:
        st = _ffi.lib().sfntt_inverse_dev(self.ctx.handle, self.FIELD, self.VARIANT, ptr, log_n, batch, stream)
        _check(self.ctx.handle, st, batch << log_n)


# M31 Circle NTT (DCCT) variants (src/ntt/m31/*)
class CudaCtDitR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_M31, V1, "cuda-ct-dit-r2"


class CudaCtGsR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_M31, V2, "cuda-ct-gs-r2"


class CudaStockhamR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_M31, V3, "cuda-stockham-r2"


class CudaCtGsR4(NttBackend):
    FIELD, VARIANT, NAME = FIELD_M31, V4, "cuda-ct-gs-r4"


# BabyBear variants (src/ntt/babybear/*)
class BbCudaCtDitR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_BABYBEAR, V1, "bb-cuda-ct-dit-r2"


class BbBatchNtt(NttBackend):
    FIELD, VARIANT, NAME = FIELD_BABYBEAR, V2, "bb-cuda-r2"


class BbCudaStockhamR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_BABYBEAR, V3, "bb-cuda-stockham-r2"


class BbCudaCtGsR4(NttBackend):
    FIELD, VARIANT, NAME = FIELD_BABYBEAR, V4, "bb-cuda-ct-gs-r4"


# KoalaBear (no reference implementation): the BabyBear variants over KoalaBear
class KbCudaCtDitR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_KOALABEAR, V1, "kb-cuda-ct-dit-r2"


class KbBatchNtt(NttBackend):
    FIELD, VARIANT, NAME = FIELD_KOALABEAR, V2, "kb-cuda-r2"


class KbCudaStockhamR2(NttBackend):
    FIELD, VARIANT, NAME = FIELD_KOALABEAR, V3, "kb-cuda-stockham-r2"


class KbCudaCtGsR4(NttBackend):
    FIELD, VARIANT, NAME = FIELD_KOALABEAR, V4, "kb-cuda-ct-gs-r4"


# reference type names (src/ntt/m31/*, src/ntt/babybear/*, src/ntt/metal_r2.rs:337-340)
MetalCtDitR2, MetalCtGsR2, MetalStockhamR2, MetalCtGsR4 = CudaCtDitR2, CudaCtGsR2, CudaStockhamR2, CudaCtGsR4
BbMetalCtDitR2, BbMetalR2, BbMetalStockhamR2, BbMetalCtGsR4 = BbCudaCtDitR2, BbBatchNtt, BbCudaStockhamR2, BbCudaCtGsR4


# -------------------------------------------------------------------- LDE ---
@dataclass
class LdeResult:
    """LdeResult (src/lde/mod.rs:20-25): SoA data[col * n_ext + row]."""
    data: np.ndarray
    total_ns: int


class CosetLdeBatch:
    """CosetLdeBatch (src/lde/mod.rs:15-107)."""

    FIELD = FIELD_BABYBEAR

    def __init__(self, ctx: Context | None = None, device: int = 0, fused: bool = True, natural: bool = False):
        """natural=True: natural-order input evaluations and output rows
        (Plonky3's convention) instead of the reference's bit-reversed ones."""
        self.ctx = ctx or default_context(device)
        self.mode = (LDE_FUSED if fused else LDE_UNFUSED) | (LDE_NATURAL if natural else 0)

    @classmethod
    def new(cls, shader_dir=None, device: int = 0):
        return cls(device=device)

    def execute(self, input, log_n: int, batch_size: int, added_bits: int, shift_monty: int = 0,
                out: np.ndarray | None = None) -> LdeResult:
        inp = _u32(input)
        dst = out if out is not None else np.empty(_out_words(batch_size, log_n, added_bits), dtype=np.uint32)
        ns = ctypes.c_uint64()
        st = _ffi.lib().sfntt_coset_lde(self.ctx.handle, self.FIELD, _p(inp), inp.size, log_n, batch_size,
                                        added_bits, shift_monty, self.mode, _p(dst), ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return LdeResult(dst, int(ns.value))

    def execute_dev(self, in_ptr: int, out_ptr: int, log_n: int, batch_size: int, added_bits: int,
                    shift_monty: int = 0, stream: int = 0) -> None:
        st = _ffi.lib().sfntt_coset_lde_dev(self.ctx.handle, self.FIELD, in_ptr, out_ptr, log_n, batch_size,
                                            added_bits, shift_monty, self.mode, stream)
        _check(self.ctx.handle, st, batch_size << log_n)

    def device_info(self) -> str:
        return self.ctx.device_info()


class KbCosetLdeBatch(CosetLdeBatch):
    """The coset LDE over KoalaBear (no reference implementation): the
    BabyBear algorithm with KoalaBear's constants; shift_monty 0 selects
    two_adic_generator(log_n + added_bits + 1), log_n + added_bits <= 23."""

    FIELD = FIELD_KOALABEAR


class M31Lde:
    """M31 blow-up: inverse on odds(log n) -> zero-pad -> forward on
    odds(log n + added_bits).  No reference counterpart (the reference has no
    M31 LDE); defined as that composition of reference functions."""

    def __init__(self, ctx: Context | None = None, device: int = 0):
        self.ctx = ctx or default_context(device)

    def execute(self, input, log_n: int, batch_size: int, added_bits: int,
                out: np.ndarray | None = None) -> LdeResult:
        inp = _u32(input)
        dst = out if out is not None else np.empty(_out_words(batch_size, log_n, added_bits), dtype=np.uint32)
        ns = ctypes.c_uint64()
        st = _ffi.lib().sfntt_m31_lde(self.ctx.handle, _p(inp), inp.size, log_n, batch_size, added_bits,
                                      _p(dst), ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return LdeResult(dst, int(ns.value))

    def execute_dev(self, in_ptr: int, out_ptr: int, log_n: int, batch_size: int, added_bits: int,
                    stream: int = 0) -> None:
        st = _ffi.lib().sfntt_m31_lde_dev(self.ctx.handle, in_ptr, out_ptr, log_n, batch_size, added_bits, stream)
        _check(self.ctx.handle, st, batch_size << log_n)


class CircleLde:
    """Canonic-coset circle FFT and circle LDE over M31 (Stwo-style): the
    reference's M31 network and conventions with circle-FFT twiddles (layer 0
    y(h), layer L >= 1 x(2^(L-1) h)) on odds(log n) ordered half coset then
    conjugates, values bit-reversed.  The LDE interpolates, zero-pads the
    coefficients and evaluates on odds(log n + added_bits): a genuine
    low-degree extension.  No reference counterpart (planned there)."""

    def __init__(self, ctx: Context | None = None, device: int = 0):
        self.ctx = ctx or default_context(device)

    def ntt(self, data, log_n: int, batch: int = 1, inverse: bool = False):
        inp = _u32(data)
        out = np.empty_like(inp)
        ns = ctypes.c_uint64()
        st = _ffi.lib().sfntt_circle_ntt(self.ctx.handle, int(inverse), _p(inp), inp.size, log_n, batch, _p(out),
                                         ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return out, int(ns.value)

    def execute(self, input, log_n: int, batch_size: int, added_bits: int,
                out: np.ndarray | None = None) -> LdeResult:
        inp = _u32(input)
        dst = out if out is not None else np.empty(_out_words(batch_size, log_n, added_bits), dtype=np.uint32)
        ns = ctypes.c_uint64()
        st = _ffi.lib().sfntt_circle_lde(self.ctx.handle, _p(inp), inp.size, log_n, batch_size, added_bits, _p(dst),
                                         ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return LdeResult(dst, int(ns.value))

    def prepare(self, log_n: int, added_bits: int) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_prepare_circle(self.ctx.handle, log_n, added_bits))

    def execute_dev(self, in_ptr: int, out_ptr: int, log_n: int, batch_size: int, added_bits: int,
                    stream: int = 0) -> None:
        st = _ffi.lib().sfntt_circle_lde_dev(self.ctx.handle, in_ptr, out_ptr, log_n, batch_size, added_bits, stream)
        _check(self.ctx.handle, st, batch_size << log_n)

    def ntt_dev(self, ptr: int, log_n: int, batch: int = 1, inverse: bool = False, stream: int = 0) -> None:
        st = _ffi.lib().sfntt_circle_ntt_dev(self.ctx.handle, int(inverse), ptr, log_n, batch, stream)
        _check(self.ctx.handle, st, batch << log_n)


class Cm31Ntt:
    """Circle NTT over the M31 quadratic extension CM31 = M31[i]/(i^2+1)
    (planned in the reference, TODOS.md:27-31): `batch` columns of 2^log_n
    interleaved (re, im) pairs of canonical M31 words; the M31 transform of
    each coordinate (the twiddles lie in M31)."""

    def __init__(self, ctx: Context | None = None, device: int = 0):
        self.ctx = ctx or default_context(device)

    def _host(self, inverse: bool, pairs, log_n: int, batch: int):
        inp = _u32(pairs)
        out = np.empty_like(inp)
        ns = ctypes.c_uint64()
        st = _ffi.lib().sfntt_cm31_ntt(self.ctx.handle, int(inverse), _p(inp), inp.size, log_n, batch, _p(out),
                                       ctypes.byref(ns))
        _check(self.ctx.handle, st, inp.size)
        return out, int(ns.value)

    def forward_batch_gpu(self, pairs, log_n: int, batch: int = 1):
        return self._host(False, pairs, log_n, batch)

    def inverse_batch_gpu(self, pairs, log_n: int, batch: int = 1):
        return self._host(True, pairs, log_n, batch)

    def prepare(self, log_n: int, batch: int) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_cm31_prepare(self.ctx.handle, log_n, batch))

    def forward_dev(self, ptr: int, log_n: int, batch: int = 1, stream: int = 0) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_cm31_ntt_dev(self.ctx.handle, 0, ptr, log_n, batch, stream))

    def inverse_dev(self, ptr: int, log_n: int, batch: int = 1, stream: int = 0) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_cm31_ntt_dev(self.ctx.handle, 1, ptr, log_n, batch, stream))

    def mul_dev(self, a_ptr: int, b_ptr: int, out_ptr: int, n: int, stream: int = 0) -> None:
        """out[k] = a[k] * b[k] for n CM31 pairs."""
        _check(self.ctx.handle, _ffi.lib().sfntt_cm31_mul_dev(self.ctx.handle, a_ptr, b_ptr, out_ptr, n, stream))


def convert_monty_dev(ctx: Context, field: int, ptr: int, n: int, to_monty: bool, stream: int = 0) -> None:
    """In-place canonical <-> Montgomery conversion of n device words
    (BabyBear::to_monty / from_monty, src/field/babybear.rs:54-65; KoalaBear alike)."""
    fn = _ffi.lib().sfntt_to_monty_dev if to_monty else _ffi.lib().sfntt_from_monty_dev
    _check(ctx.handle, fn(ctx.handle, field, ptr, n, stream), n)


# -------------------------------------------------------- output layout ---
def layout(data, log_n: int, batch: int, flags: int, ctx: Context | None = None) -> tuple[np.ndarray, int]:
    """Row order / row-major form of a SoA batch (sfntt_layout): flags
    LAYOUT_NATURAL (bit-reversed rows -> natural), LAYOUT_ROW_MAJOR
    (out[row * batch + col], the Merkle-commitment input).  -> (out, device ns)."""
    ctx = ctx or default_context()
    inp = _u32(data)
    out = np.empty_like(inp)
    ns = ctypes.c_uint64()
    st = _ffi.lib().sfntt_layout(ctx.handle, _p(inp), inp.size, log_n, batch, flags, _p(out), ctypes.byref(ns))
    _check(ctx.handle, st, inp.size)
    return out, int(ns.value)


def layout_dev(ctx: Context, in_ptr: int, out_ptr: int, log_n: int, batch: int, flags: int, stream: int = 0) -> None:
    """Device pointers; in place (in_ptr == out_ptr) for LAYOUT_NATURAL alone."""
    st = _ffi.lib().sfntt_layout_dev(ctx.handle, in_ptr, out_ptr, log_n, batch, flags, stream)
    _check(ctx.handle, st, batch << log_n)


# ------------------------------------------------------- uneven batches ---
PLAN_AUTO, PLAN_TMA, PLAN_TMA_FOUR_STEP, PLAN_TILE = 0, 1, 2, 3
PLAN_SPLIT12, PLAN_ONE_CTA = 4, 8  # flags on the TMA engines (layer split, one CTA per SM)


class LdeBatch:
    """Uneven batch of LDE / blow-up items (both fields, device pointers) run
    as a plain per-item loop, or captured once into a CUDA graph and replayed
    with one launch (sfntt_batch_*, sfntt_graph_*).  Items are dicts with
    keys field, log_n, batch, added_bits, d_in, d_out [, shift_monty, plan]."""

    def __init__(self, ctx: Context, items: list[dict]):
        self.ctx = ctx
        arr = (_ffi.LdeItem * max(len(items), 1))()
        for i, it in enumerate(items):
            arr[i] = _ffi.LdeItem(it["field"], it["log_n"], it["batch"], it["added_bits"],
                                  it.get("shift_monty", 0), it["d_in"], it["d_out"], it.get("plan", PLAN_AUTO))
        self.items = arr
        self.count = len(items)

    def prepare(self) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_batch_prepare(self.ctx.handle, self.items, self.count))

    def run(self, stream: int = 0) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_batch_run(self.ctx.handle, self.items, self.count, stream))

    def autotune(self, reps: int = 2) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_autotune(self.ctx.handle, self.items, self.count, reps))

    def plan_of(self, i: int) -> int:
        return _ffi.lib().sfntt_tune_lookup(self.ctx.handle, ctypes.byref(self.items[i]))

    def graph(self, lanes: int = 8) -> "Graph":
        h = ctypes.c_void_p()
        _check(self.ctx.handle, _ffi.lib().sfntt_batch_graph_create(self.ctx.handle, self.items, self.count, lanes,
                                                                    ctypes.byref(h)))
        return Graph(h)

    def persistent_graph(self, lanes: int = 8) -> "Graph":
        """The batch with its eligible items (BabyBear / M31, 2^13..2^21
        points, blow-up <= 16) in three persistent phase launches over a
        device work list, the rest per item on `lanes` streams, in one graph
        (sfntt_batch_persistent_create)."""
        h = ctypes.c_void_p()
        _check(self.ctx.handle, _ffi.lib().sfntt_batch_persistent_create(self.ctx.handle, self.items, self.count,
                                                                         lanes, ctypes.byref(h)))
        return Graph(h)


class Graph:
    """An instantiated CUDA graph of a whole batch (sfntt_graph)."""

    def __init__(self, handle):
        self.handle = handle

    def launch(self, stream: int = 0) -> None:
        st = _ffi.lib().sfntt_graph_launch(self.handle, stream)
        if st:
            raise _ERRORS.get(st, NttError)(f"sfntt_graph_launch: status {st}")

    def kernel_count(self) -> int:
        return int(_ffi.lib().sfntt_graph_kernel_count(self.handle))

    def close(self) -> None:
        if self.handle:
            _ffi.lib().sfntt_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_save(ctx: Context, path: str) -> None:
    _check(ctx.handle, _ffi.lib().sfntt_tune_save(ctx.handle, str(path).encode()))


def tune_load(ctx: Context, path: str) -> None:
    _check(ctx.handle, _ffi.lib().sfntt_tune_load(ctx.handle, str(path).encode()))


def uneven_workload(n_items: int = 64, seed: int = 2024, log_n_range=(12, 22), cols_range=(1, 128),
                    blowups=(0, 1, 2)) -> list[dict]:
    """The uneven-batch configuration: field 50/50 M31 / BabyBear, log n and
    columns uniform in their ranges, added_bits uniform over `blowups`
    (blow-up 1/2/4), seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_items):
        out.append({"field": int(rng.integers(0, 2)), "log_n": int(rng.integers(log_n_range[0], log_n_range[1] + 1)),
                    "batch": int(rng.integers(cols_range[0], cols_range[1] + 1)),
                    "added_bits": int(rng.choice(blowups))})
    return out


# ---------------------------------------------------------------- serving ---
def _item_struct(it: dict) -> "_ffi.LdeItem":
    return _ffi.LdeItem(it["field"], it["log_n"], it["batch"], it["added_bits"], it.get("shift_monty", 0),
                        it.get("d_in", 0) or 0, 0, it.get("plan", PLAN_AUTO))


class _DeviceWords:
    """__cuda_array_interface__ view of n u32 words at a device address (as int32)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3,
                                         "strides": None}


class Server:
    """Continuous-batching request server (sfntt_server_*): `slots` streams,
    one device arena of `budget_bytes` (the HBM admission budget).  Requests
    are dicts like LdeBatch items; `submit` takes the input at it["d_in"] on
    the device, `submit_host` copies from / to host arrays.  `poll` retires
    finished requests and admits queued ones in order while a slot is free
    and the arena has room."""

    def __init__(self, ctx: Context, budget_bytes: int, slots: int = 8):
        self.ctx = ctx
        h = ctypes.c_void_p()
        _check(ctx.handle, _ffi.lib().sfntt_server_create(ctx.handle, budget_bytes, slots, ctypes.byref(h)))
        self.handle = h
        self._host = {}  # ticket -> (in array, out array) kept alive until done

    def submit(self, it: dict) -> int:
        t = ctypes.c_uint64()
        req = _item_struct(it)
        _check(self.ctx.handle, _ffi.lib().sfntt_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t)))
        return t.value

    def submit_host(self, it: dict, x: np.ndarray) -> tuple[int, np.ndarray]:
        """Returns (ticket, out); out is filled when the ticket completes."""
        x = _u32(x)
        out = np.empty(it["batch"] << (it["log_n"] + it["added_bits"]), dtype=np.uint32)
        t = ctypes.c_uint64()
        req = _item_struct(it)
        _check(self.ctx.handle, _ffi.lib().sfntt_server_submit_host(
            self.handle, ctypes.byref(req), x.ctypes.data, out.ctypes.data, ctypes.byref(t)))
        self._host[t.value] = (x, out)
        return t.value, out

    def poll(self, cap: int = 256) -> list[int]:
        buf = (ctypes.c_uint64 * cap)()
        n = ctypes.c_size_t()
        _check(self.ctx.handle, _ffi.lib().sfntt_server_poll(self.handle, buf, cap, ctypes.byref(n)))
        done = [int(buf[i]) for i in range(n.value)]
        for t in done:
            self._host.pop(t, None)
        return done

    def result_ptr(self, ticket: int) -> int:
        p = ctypes.c_void_p()
        _check(self.ctx.handle, _ffi.lib().sfntt_server_result(self.handle, ticket, ctypes.byref(p)))
        return p.value

    def result(self, ticket: int, n_words: int):
        """A torch int32 view of a finished request's output (valid until release)."""
        import torch
        return torch.as_tensor(_DeviceWords(self.result_ptr(ticket), n_words), device=f"cuda:{self.ctx.device}")

    def release(self, ticket: int) -> None:
        _check(self.ctx.handle, _ffi.lib().sfntt_server_release(self.handle, ticket))

    def pending(self) -> int:
        return int(_ffi.lib().sfntt_server_pending(self.handle))

    def set_packing(self, max_requests: int) -> None:
        """Up to max_requests queued requests of one shape share a launch as
        columns of one batch (1: every request launches alone)."""
        _check(self.ctx.handle, _ffi.lib().sfntt_server_set_packing(self.handle, max_requests))

    def launches(self) -> int:
        return int(_ffi.lib().sfntt_server_launches(self.handle))

    def close(self) -> None:
        if self.handle:
            _ffi.lib().sfntt_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_trace(ctx: Context, reqs: list[dict], arrivals, slots: int, budget_bytes: int,
                host: list[tuple[np.ndarray, np.ndarray]] | None = None, max_pack: int = 1,
                stats: dict | None = None) -> tuple[np.ndarray, float]:
    """Replays a trace (sfntt_serve_trace_packed): request i submitted at
    arrivals[i] seconds; returns (latency seconds per request, makespan
    seconds).  slots=1 is the plain sequential per-request loop; max_pack > 1
    lets up to that many same-shape requests share a launch.  `host`:
    per-request (input, output) host arrays for host requests, else inputs at
    d_in on the device.  `stats` (optional) receives the launch count."""
    n = len(reqs)
    arr = (_ffi.LdeItem * max(n, 1))()
    for i, it in enumerate(reqs):
        arr[i] = _item_struct(it)
    t_arr = np.ascontiguousarray(arrivals, dtype=np.float64)
    lat = np.zeros(n, dtype=np.float64)
    mk = ctypes.c_double()
    dbl = ctypes.POINTER(ctypes.c_double)
    h_in = h_out = None
    if host is not None:
        h_in = (ctypes.c_void_p * max(n, 1))(*[h[0].ctypes.data for h in host])
        h_out = (ctypes.c_void_p * max(n, 1))(*[h[1].ctypes.data for h in host])
    launches = ctypes.c_uint64()
    _check(ctx.handle, _ffi.lib().sfntt_serve_trace_packed(ctx.handle, arr, h_in, h_out, t_arr.ctypes.data_as(dbl),
                                                           n, slots, max_pack, budget_bytes, lat.ctypes.data_as(dbl),
                                                           ctypes.byref(mk), ctypes.byref(launches)))
    if stats is not None:
        stats["launches"] = int(launches.value)
    return lat, mk.value


SERVED_LOG_N_WEIGHTS = {14: 1, 15: 1, 16: 2, 17: 3, 18: 6, 19: 6, 20: 6, 21: 2, 22: 1}


def served_workload(n_requests: int, rate: float, seed: int = 2025, cols_range=(8, 256), blowups=(1, 2),
                    log_n_weights: dict | None = None) -> tuple[list[dict], np.ndarray]:
    """The served stream: Poisson arrivals at `rate` req/s; field 50/50 M31 /
    BabyBear; log n in 14..22 weighted toward 18-20; columns uniform in
    cols_range; blow-up 2 or 4 (added_bits 1 or 2); seeded.  Returns
    (requests without buffers, sorted arrival times in seconds)."""
    w = log_n_weights or SERVED_LOG_N_WEIGHTS
    rng = np.random.default_rng(seed)
    logs = np.array(sorted(w), dtype=np.int64)
    p = np.array([w[k] for k in logs], dtype=np.float64)
    p /= p.sum()
    reqs = []
    for _ in range(n_requests):
        reqs.append({"field": int(rng.integers(0, 2)), "log_n": int(rng.choice(logs, p=p)),
                     "batch": int(rng.integers(cols_range[0], cols_range[1] + 1)),
                     "added_bits": int(rng.choice(blowups))})
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    return reqs, arrivals


__all__ = [n for n in dir() if not n.startswith("_")]
