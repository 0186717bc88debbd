"""gpupi_b200: B200-native batched multi-precision arithmetic and Chudnovsky pi.

Python binding of ``libgpupi_b200.so`` (C ABI in ``include/gpupi_c.h``).  The
functions mirror gpupi's batched API (``batch_arith.h``): every operand is a
batch of N unsigned integers stored as little-endian 32-bit limbs, item i at
``data + i*stride`` (stride 0 broadcasts one row).  Device memory is handled
with torch tensors (int32 storage reinterpreted as uint32 limbs); all
arithmetic runs in this library's CUDA kernels.

There is no CPU fallback: importing works without a GPU (for build checks),
but every compute call raises if the native library or a CUDA device is
missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgpupi_b200.so"
CLI_PATH = _HERE / "pi_bs_gpu"

_lib = None

_u32 = ctypes.c_uint32
_p = ctypes.c_void_p
_i32 = ctypes.c_int32

# (name, restype, argtypes) for every C ABI symbol in include/gpupi_c.h
_SIGS = [
    ("gpupi_version", ctypes.c_char_p, []),
    ("gpupi_launch_count", ctypes.c_uint64, []),
    ("gpupi_set_stream", ctypes.c_int, [_p]),
    ("gpupi_device_sync", ctypes.c_int, []),
    ("gpupi_ctx_create", _p, []),
    ("gpupi_ctx_destroy", None, [_p]),
    ("gpupi_ctx_workspace_size", ctypes.c_size_t, [_p]),
    ("gpupi_ctx_ensure_workspace", ctypes.c_int, [_p, ctypes.c_size_t]),
    ("gpupi_mp_mul", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_add", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_sub", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_shift_add", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_shift_sub", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_add_small", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_sub_small", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_mul_small", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_mp_exactdiv_small", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _u32]),
    ("gpupi_mp_shift_bits", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _i32]),
    ("gpupi_mp_bitlength_max", ctypes.c_int, [_p, _u32, _p, _u32, _u32, ctypes.POINTER(_u32)]),
    ("gpupi_mp_limblength_max", ctypes.c_int, [_p, _u32, _p, _u32, _u32, ctypes.POINTER(_u32)]),
    ("gpupi_mul_naive", ctypes.c_int, [_u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32]),
    ("gpupi_mul_ntt", ctypes.c_int, [_p, _u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32]),
    ("gpupi_mul_tc", ctypes.c_int, [_u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32]),
    ("gpupi_tc_error", ctypes.c_int, []),
    ("gpupi_tc_selftest_timeout", ctypes.c_int, [ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    ("gpupi_int_peak", ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("gpupi_fail_alloc", ctypes.c_int, [_u32, _u32]),
    ("gpupi_tree_graph_stats", ctypes.c_int, [_p]),
    ("gpupi_tree_graph_perturb", ctypes.c_int, []),
    ("gpupi_scratch_live_bytes", ctypes.c_uint64, []),
    ("gpupi_tune_load", ctypes.c_int, [ctypes.c_char_p]),
    ("gpupi_tune_load_text", ctypes.c_int, [ctypes.c_char_p]),
    ("gpupi_tune_reset", ctypes.c_int, []),
    ("gpupi_tune_describe", ctypes.c_size_t, [_p, ctypes.c_size_t]),
    ("gpupi_mul_kind", ctypes.c_int, [_u32, _u32, ctypes.c_int]),
    ("gpupi_ntt_shape", ctypes.c_int, [_u32, _u32, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("gpupi_autotune", ctypes.c_int, [_p, ctypes.c_char_p, ctypes.c_uint64]),
    ("gpupi_decimal_naive", ctypes.c_int, [_u32, _p, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_convert_decimal", ctypes.c_int, [_p, _p, _u32, _u32, _u32, _u32, _p]),
    ("gpupi_pi_compute", ctypes.c_int,
     [_p, _u32, _u32, _p, ctypes.c_size_t, _p, ctypes.c_size_t, ctypes.POINTER(_u32)]),
    ("gpupi_timer_enable", ctypes.c_int, [ctypes.c_int]),
    ("gpupi_timer_reset", ctypes.c_int, []),
    ("gpupi_timer_report", ctypes.c_size_t, [_p, ctypes.c_size_t]),
    ("gpupi_transfer_bytes", ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("gpupi_scratch_stats", ctypes.c_int,
     [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("gpupi_mp_add_noalloc", ctypes.c_int, [_u32, _p, _u32, _u32, _p, _u32, _u32, _p, _u32, _u32]),
    ("gpupi_set_mul_crossover", ctypes.c_int, [_u32]),
    ("gpupi_bbp_fractions", ctypes.c_int, [_p, _u32, _p]),
    ("gpupi_mp_mul_ragged", ctypes.c_int, [_p, _u32, _p, _p, _p, _p, _p, _p, _p, _p]),
    ("gpupi_mp_mul_spectra", ctypes.c_int, [_p, _u32, _p, _u32, _p, _u32, _p, _u32, _p, _u32, _p, _u32]),
    ("gpupi_pi_stream", ctypes.c_int, [_p, _u32, _u32, _p, _p, ctypes.c_size_t, _p]),
    ("gpupi_pi_compute_checkpointed", ctypes.c_int,
     [_p, _u32, _u32, ctypes.c_char_p, _p, ctypes.c_size_t, _p, ctypes.c_size_t, _p]),
]

_DIGIT_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)

C_ABI_SYMBOLS = [s[0] for s in _SIGS]


class GpupiError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise GpupiError(f"{LIB_PATH} is missing: run gpupi_b200/build.py (or __graft_entry__.build())")
        l = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in _SIGS:
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise GpupiError(f"{what} failed with cudaError {rc}")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise GpupiError("gpupi_b200 needs a CUDA device; there is no CPU fallback")
    return torch


# ---------------------------------------------------------------------------
# Device buffers
# ---------------------------------------------------------------------------
class DeviceLimbs:
    """A device buffer of uint32 limbs (torch int32 storage)."""

    def __init__(self, words: int):
        torch = _torch()
        self.t = torch.zeros(max(int(words), 1), dtype=torch.int32, device="cuda")
        self.words = int(words)

    @classmethod
    def from_numpy(cls, a: np.ndarray) -> "DeviceLimbs":
        torch = _torch()
        a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1)
        d = cls(a.size)
        if a.size:
            d.t[: a.size].copy_(torch.from_numpy(a.view(np.int32)))
        return d

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()

    def at(self, offset_words: int) -> int:
        return self.ptr + 4 * int(offset_words)

    def numpy(self) -> np.ndarray:
        _torch().cuda.synchronize()
        return self.t[: self.words].cpu().numpy().view(np.uint32)


class DeviceBytes:
    def __init__(self, n: int):
        torch = _torch()
        self.t = torch.zeros(max(int(n), 1), dtype=torch.uint8, device="cuda")
        self.n = int(n)

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()

    def text(self) -> str:
        _torch().cuda.synchronize()
        return bytes(self.t[: self.n].cpu().numpy()).decode("ascii")


# ---------------------------------------------------------------------------
# Context and batched ops (gpupi batch_arith.h)
# ---------------------------------------------------------------------------
class Context:
    """Wraps BatchMPContext (NTT tables + grow-only workspace)."""

    def __init__(self):
        _torch()
        self.h = lib().gpupi_ctx_create()
        if not self.h:
            raise GpupiError("gpupi_ctx_create failed")

    def close(self) -> None:
        if self.h:
            lib().gpupi_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def workspace_size(self) -> int:
        return lib().gpupi_ctx_workspace_size(self.h)

    # Each op takes raw device addresses (ints), lengths and strides.
    def mul(self, N, A, La, sA, B, Lb, sB, C, Lc, sC):
        _check(lib().gpupi_mp_mul(self.h, N, A, La, sA, B, Lb, sB, C, Lc, sC), "batch_mp_mul")

    def add(self, N, A, La, sA, B, Lb, sB, C, Lc, sC):
        _check(lib().gpupi_mp_add(self.h, N, A, La, sA, B, Lb, sB, C, Lc, sC), "batch_mp_add")

    def sub(self, N, A, La, sA, B, Lb, sB, C, Lc, sC):
        _check(lib().gpupi_mp_sub(self.h, N, A, La, sA, B, Lb, sB, C, Lc, sC), "batch_mp_sub")

    def shift_add(self, N, A, La, sA, B, Lb, sB, shift, C, Lc, sC):
        _check(lib().gpupi_mp_shift_add(self.h, N, A, La, sA, B, Lb, sB, shift, C, Lc, sC), "batch_mp_shift_add")

    def shift_sub(self, N, A, La, sA, B, Lb, sB, shift, C, Lc, sC):
        _check(lib().gpupi_mp_shift_sub(self.h, N, A, La, sA, B, Lb, sB, shift, C, Lc, sC), "batch_mp_shift_sub")

    def add_small(self, N, A, La, sA, b, C, Lc, sC):
        _check(lib().gpupi_mp_add_small(self.h, N, A, La, sA, b, C, Lc, sC), "batch_mp_add_small")

    def sub_small(self, N, A, La, sA, b, C, Lc, sC):
        _check(lib().gpupi_mp_sub_small(self.h, N, A, La, sA, b, C, Lc, sC), "batch_mp_sub_small")

    def mul_small(self, N, A, La, sA, b, C, Lc, sC):
        _check(lib().gpupi_mp_mul_small(self.h, N, A, La, sA, b, C, Lc, sC), "batch_mp_mul_small")

    def exactdiv_small(self, N, A, La, sA, b):
        _check(lib().gpupi_mp_exactdiv_small(self.h, N, A, La, sA, b), "batch_mp_exactdiv_small")

    def shift_bits(self, N, A, La, sA, B, Lb, sB, shift):
        _check(lib().gpupi_mp_shift_bits(self.h, N, A, La, sA, B, Lb, sB, shift), "batch_mp_shift_bits")

    def bitlength_max(self, N, A, La, sA) -> int:
        r = _u32(0)
        _check(lib().gpupi_mp_bitlength_max(self.h, N, A, La, sA, ctypes.byref(r)), "batch_mp_bitlength_max")
        return r.value

    def limblength_max(self, N, A, La, sA) -> int:
        r = _u32(0)
        _check(lib().gpupi_mp_limblength_max(self.h, N, A, La, sA, ctypes.byref(r)), "batch_mp_limblength_max")
        return r.value

    def mul_spectra(self, N, A, La, B, Lb, C, Lc, D=None, Ld=0, E=None, Le=0):
        """C = A B (+ D E) through shared-transform spectra; packed rows,
        device pointers (gpupi_mp_mul_spectra)."""
        _check(lib().gpupi_mp_mul_spectra(self.h, N, A, La, B, Lb, D, Ld, E, Le, C, Lc), "gpupi_mp_mul_spectra")

    def mul_ragged(self, A, offA, La, B, offB, Lb, C, offC):
        """Ragged batch: product i = A[offA[i]:+La[i]] * B[offB[i]:+Lb[i]] into
        C[offC[i]:+La[i]+Lb[i]] (device pointers A, B, C; host sequences for the
        offsets and lengths)."""
        n = len(La)
        oa, ob, oc = (np.ascontiguousarray(np.asarray(x, dtype=np.uint64)) for x in (offA, offB, offC))
        la, lb = (np.ascontiguousarray(np.asarray(x, dtype=np.uint32)) for x in (La, Lb))
        _check(lib().gpupi_mp_mul_ragged(self.h, n, A, oa.ctypes.data, la.ctypes.data, B, ob.ctypes.data,
                                         lb.ctypes.data, C, oc.ctypes.data), "gpupi_mp_mul_ragged")

    def mul_ntt(self, N, A, La, sA, B, Lb, sB, C, sC):
        _check(lib().gpupi_mul_ntt(self.h, N, A, La, sA, B, Lb, sB, C, sC), "batch_mul_ntt")

    def convert_decimal(self, X, Lx, input_bits, total_digits, leaf_digits, out):
        _check(lib().gpupi_convert_decimal(self.h, X, Lx, input_bits, total_digits, leaf_digits, out),
               "convert_decimal")


def mul_naive(N, A, La, sA, B, Lb, sB, C, sC):
    _torch()
    _check(lib().gpupi_mul_naive(N, A, La, sA, B, Lb, sB, C, sC), "batch_mul_naive")


def mul_tc(N, A, La, sA, B, Lb, sB, C, sC):
    """Schoolbook product on the tensor cores (int8 split-integer MMAs)."""
    _torch()
    _check(lib().gpupi_mul_tc(N, A, La, sA, B, Lb, sB, C, sC), "gpupi_mul_tc")


def tc_error() -> int:
    """Device error word of the tensor-core kernels (read and cleared)."""
    return int(lib().gpupi_tc_error())


def int_peak() -> dict:
    """Measured integer-pipe peaks (warp instructions per second)."""
    _torch()
    a, b = ctypes.c_double(0), ctypes.c_double(0)
    _check(lib().gpupi_int_peak(ctypes.byref(a), ctypes.byref(b)), "gpupi_int_peak")
    return {"imad_winst_per_s": a.value, "alu_winst_per_s": b.value}


ALLOC_SCRATCH, ALLOC_WORKSPACE, ALLOC_ARRAY = 1, 2, 4


def fail_alloc(kind_mask: int, nth: int) -> None:
    """Make the nth following device allocation of a category in kind_mask
    fail once (host-side injection for error-path tests; 0 disarms)."""
    lib().gpupi_fail_alloc(kind_mask, nth)


def tree_graph_stats() -> dict:
    """Counts of the splitting tree's graph path (recorded schedules, captured
    graphs, graph runs, fallbacks, sizes without a graph)."""
    out = (ctypes.c_uint64 * 5)()
    lib().gpupi_tree_graph_stats(ctypes.addressof(out))
    return dict(zip(("recorded", "captured", "replayed", "fallbacks", "disabled"), map(int, out)))


def tree_graph_perturb() -> None:
    lib().gpupi_tree_graph_perturb()


def scratch_live_bytes() -> int:
    return int(lib().gpupi_scratch_live_bytes())


MUL_KINDS = ("school", "tc", "ntt")
TUNE_TABLE_PATH = _HERE / "tune_table.txt"


def tune_load(path=None, text: str | None = None) -> int:
    """Load a tune table from a file or from text (host only, no GPU needed);
    returns the number of entries (raises on a malformed line)."""
    n = lib().gpupi_tune_load_text(text.encode()) if text is not None else lib().gpupi_tune_load(str(path).encode())
    if n < 0:
        raise GpupiError(f"tune table: malformed line {-n}" if n > -1000000 else "tune table: cannot read file")
    return n


def tune_reset() -> None:
    lib().gpupi_tune_reset()


def tune_describe() -> str:
    n = lib().gpupi_tune_describe(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib().gpupi_tune_describe(buf, n + 1)
    return buf.value.decode()


def mul_kind(La: int, Lb: int, public_api: bool = False) -> str:
    """Kernel a product of La x Lb limbs uses under the table in effect."""
    return MUL_KINDS[lib().gpupi_mul_kind(La, Lb, 1 if public_api else 0)]


def ntt_shape(La: int, Lb: int) -> tuple[int, int]:
    """(log_k, M): the NTT transform shape of an La x Lb product under the table in effect."""
    lk, m = ctypes.c_int(0), ctypes.c_int(0)
    _check(lib().gpupi_ntt_shape(La, Lb, ctypes.byref(lk), ctypes.byref(m)), "gpupi_ntt_shape")
    return lk.value, m.value


def autotune(ctx: "Context", path=TUNE_TABLE_PATH, budget_limbs: int = 1 << 24) -> str:
    """Measure every candidate on the current GPU, write the table to `path`
    and load it; returns the table text."""
    _torch()
    _check(lib().gpupi_autotune(ctx.h, str(path).encode(), budget_limbs), "gpupi_autotune")
    return Path(path).read_text()


def tc_selftest_timeout() -> tuple[int, int]:
    """(error word of the forced-timeout call, error word of a normal call after it)."""
    _torch()
    a, b = _u32(0), _u32(0)
    _check(lib().gpupi_tc_selftest_timeout(ctypes.byref(a), ctypes.byref(b)), "gpupi_tc_selftest_timeout")
    return a.value, b.value


def decimal_naive(N, A, L_limb, sA, out, L_dec, s_out):
    _torch()
    _check(lib().gpupi_decimal_naive(N, A, L_limb, sA, out, L_dec, s_out), "batch_decimal_naive")


def add_noalloc(N, A, La, sA, B, Lb, sB, C, Lc, sC) -> None:
    """C = A + B like Context.add, without a context and without any device
    allocation (gpupi_mp_add_noalloc); for callers that cannot allocate."""
    _torch()
    _check(lib().gpupi_mp_add_noalloc(N, A, La, sA, B, Lb, sB, C, Lc, sC), "gpupi_mp_add_noalloc")


def launch_count() -> int:
    return int(lib().gpupi_launch_count())


def timer_enable(on: bool) -> None:
    lib().gpupi_timer_enable(1 if on else 0)


def timer_reset() -> None:
    lib().gpupi_timer_reset()


def timer_report() -> dict:
    """{kernel family: (launches, total_ms, total_algorithmic_bytes)}"""
    l = lib()
    n = l.gpupi_timer_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    l.gpupi_timer_report(buf, n + 1)
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms, by = line.split()
        if not name.startswith("gap:"):
            out[name] = (int(cnt), float(ms), float(by))
    return out


def timer_gaps() -> dict:
    """{"prev>next": (count, device_ms, host_ms)}: time between consecutive
    timed launches of two kernel families (untimed kernels, synchronisations,
    launch starvation) on the device and on the host clock."""
    l = lib()
    n = l.gpupi_timer_report(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    l.gpupi_timer_report(buf, n + 1)
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms, host = line.split()
        if name.startswith("gap:"):
            out[name[4:]] = (int(cnt), float(ms), float(host))
    return out


def transfer_bytes() -> tuple[int, int]:
    h, d = ctypes.c_uint64(0), ctypes.c_uint64(0)
    lib().gpupi_transfer_bytes(ctypes.byref(h), ctypes.byref(d))
    return h.value, d.value


def scratch_stats() -> dict:
    """Scratch arena: {"block_bytes", "high_water", "spills"} (see gpupi_c.h)."""
    b, h, n = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
    lib().gpupi_scratch_stats(ctypes.byref(b), ctypes.byref(h), ctypes.byref(n))
    return {"block_bytes": b.value, "high_water": h.value, "spills": n.value}


def set_mul_crossover(v: int) -> None:
    _check(lib().gpupi_set_mul_crossover(v), "gpupi_set_mul_crossover")


# ---------------------------------------------------------------------------
# Whole pipeline
# ---------------------------------------------------------------------------
class PiResult:
    def __init__(self, digits, convert_digits, ret_len, elapsed_ms, workspace_mb, ret, dec, leaf_digits):
        self.digits = digits
        self.convert_digits = convert_digits
        self.ret_len = ret_len
        self.elapsed_ms = elapsed_ms
        self.workspace_mb = workspace_mb
        self.ret = ret
        self.dec = dec
        self.leaf_digits = leaf_digits


def ret_limbs_bound(digits: int) -> int:
    """An upper bound on RET's length in limbs for ``digits`` digits."""
    return (int(digits * 3.322) + 31) // 32 + 8


def pi_compute(digits: int, ctx: Context | None = None, copy_digits: int | None = None,
               ret_capacity: int | None = None, device_only: bool = False, profile: bool = False,
               host_digits=None, host_ret=None, plain: bool = False, checkpoint=None) -> PiResult:
    """Run pi_bs_gpu's pipeline for ``digits`` digits (pi_bs_gpu.cu main_fractional).

    ``host_digits`` / ``host_ret``: optional writable host buffers (e.g. pinned
    torch tensors: uint8 for the digits, 32-bit for RET, at least
    ret_limbs_bound(digits) limbs) receiving the digits and RET directly from
    the device.  ``device_only`` keeps RET and the digits on the device (no
    host copies at all).  ``plain`` runs the reference's op sequence (one
    batched product per op) instead of the default tuned form, which shares
    forward transforms within each merge level of the splitting tree; both
    give the same RET and digits.
    ``checkpoint``: a file for the splitting tree's result, loaded when valid
    for this digit count (the tree is skipped) and written otherwise;
    ``checkpoint_state`` on the result is 1 (loaded), 2 (written) or 3 (the
    file could not be written; the result is still complete)."""
    _torch()
    l = lib()
    if copy_digits is None:
        copy_digits = 0 if device_only else digits
    if host_ret is not None:
        ret_capacity = host_ret.numel() if hasattr(host_ret, "numel") else len(host_ret)
        ret = host_ret.numpy().view(np.uint32) if hasattr(host_ret, "numpy") else host_ret
    else:
        if ret_capacity is None:
            ret_capacity = 0 if device_only else ret_limbs_bound(digits)
        ret = np.empty(max(ret_capacity, 1), dtype=np.uint32)
    if host_digits is not None:
        dptr = host_digits.data_ptr() if hasattr(host_digits, "data_ptr") else ctypes.addressof(host_digits)
        dbuf = None
    else:
        dbuf = ctypes.create_string_buffer(max(copy_digits, 1))
        dptr = ctypes.addressof(dbuf) if copy_digits else None
    info = (_u32 * 8)()
    flags = (1 if profile else 0) | (2 if device_only else 0) | (4 if plain else 0)
    if checkpoint is not None:
        rc = l.gpupi_pi_compute_checkpointed(ctx.h if ctx else None, digits, flags, str(checkpoint).encode(),
                                             ret.ctypes.data if ret_capacity else None, ret_capacity, dptr,
                                             copy_digits, info)
    else:
        rc = l.gpupi_pi_compute(ctx.h if ctx else None, digits, flags, ret.ctypes.data if ret_capacity else None,
                                ret_capacity, dptr, copy_digits, info)
    _check(rc, "gpupi_pi_compute")
    ret_len = info[1]
    elapsed = np.frombuffer(np.uint32(info[2]).tobytes(), dtype=np.float32)[0]
    dec = dbuf.raw[:copy_digits].decode("ascii") if dbuf is not None else ""
    r = PiResult(digits, info[0], ret_len, float(elapsed), info[3],
                 ret[:ret_len] if ret_capacity else None, dec, info[5])
    r.checkpoint_state = int(info[7]) if checkpoint is not None else 0
    return r


def pi_stream(digits: int, write, ctx: Context | None = None, chunk: int = 0, plain: bool = False) -> PiResult:
    """Compute pi to ``digits`` digits and pass the digits after "3." to
    ``write(bytes)`` in order, in chunks of at most ``chunk`` bytes (0: 64 MiB),
    each chunk's device-to-host copy overlapping the previous write
    (gpupi_pi_stream).  ``write`` returning False stops the output.
    Returns the result without RET or digits; ``output_ms`` is the host time
    of the output."""
    _torch()
    failed = []

    def _sink(data, n, user):
        try:
            return 1 if write(ctypes.string_at(data, n)) is False else 0
        except Exception as e:   # surfaced after the call
            failed.append(e)
            return 1

    cb = _DIGIT_SINK(_sink)
    info = (_u32 * 8)()
    rc = lib().gpupi_pi_stream(ctx.h if ctx else None, digits, 4 if plain else 0,
                               ctypes.cast(cb, ctypes.c_void_p), None, chunk, info)
    if failed:
        raise failed[0]
    _check(rc, "gpupi_pi_stream")
    elapsed = np.frombuffer(np.uint32(info[2]).tobytes(), dtype=np.float32)[0]
    r = PiResult(digits, info[0], info[1], float(elapsed), info[3], None, "", info[5])
    r.output_ms = float(np.frombuffer(np.uint32(info[6]).tobytes(), dtype=np.float32)[0])
    return r


def pi_to_file(digits: int, path, ctx: Context | None = None, chunk: int = 0, plain: bool = False) -> PiResult:
    """Write "3<digits>\\n" to ``path`` (the CLI's output), streamed."""
    with open(path, "wb") as f:
        f.write(b"3")
        r = pi_stream(digits, f.write, ctx, chunk, plain)
        f.write(b"\n")
    return r


# ---------------------------------------------------------------------------
# BBP spot check of RET (independent of the binary-splitting pipeline)
# ---------------------------------------------------------------------------
def bbp_fractions(positions) -> np.ndarray:
    """floor(2^64 frac(16^n pi)) for each n in ``positions`` (0-based: n = 0
    gives the hex digits right after the point), computed on the GPU with
    integer fixed point; each value is within 8 (n + 17) units of exact."""
    _torch()
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64))
    out = np.zeros(len(pos), dtype=np.uint64)
    if len(pos):
        _check(lib().gpupi_bbp_fractions(pos.ctypes.data, len(pos), out.ctypes.data), "gpupi_bbp_fractions")
    return out


def ret_hex_bits(ret, n: int, bits: int = 24) -> int:
    """The ``bits`` bits of pi starting 4n bits below the point, read from
    RET (little-endian limbs, pi * 2^(32 (len - 1)) truncated: the top limb is
    the integer part 3, the next one holds hex digits 1..8)."""
    L = len(ret)
    top = 32 * (L - 1) - 4 * n      # bit index just above the window
    lo = top - bits
    if lo < 0:
        raise ValueError("position beyond RET")
    val = 0
    for i in range(lo // 32, (top - 1) // 32 + 1):
        val |= int(ret[i]) << (32 * i)
    return (val >> lo) & ((1 << bits) - 1)


def bbp_spot_check(ret, positions, bits: int = 24):
    """Compare ``bits`` bits of RET at each position with the BBP fraction.
    Returns (mismatches, inconclusive): a position is inconclusive when the
    BBP error bound could move the compared bits."""
    fr = bbp_fractions(positions)
    bad, unsure = [], []
    shift = 64 - bits
    for n, f in zip(positions, fr):
        f = int(f)
        err = 8 * (int(n) + 17)
        lo, hi = ((f - err) % (1 << 64)) >> shift, ((f + err) % (1 << 64)) >> shift
        if lo != hi:
            unsure.append(int(n))
        elif ret_hex_bits(ret, int(n), bits) != (f >> shift):
            bad.append(int(n))
    return bad, unsure
