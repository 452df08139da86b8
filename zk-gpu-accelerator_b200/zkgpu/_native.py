"""
zkgpu._native — ctypes binding of libzkb200.so (declared in include/zkb200.h).

This is the only module that touches the shared library. It loads it once,
declares every entry point's signature, and turns non-zero status codes into
the exception types the reference raises (ValueError, TypeError,
RuntimeError). There is no CPU fallback: without the library or a CUDA
device every operation raises RuntimeError.

Device buffers are torch tensors (dtype torch.uint64); a call passes their
data pointers and torch's current CUDA stream, so launches are ordered with
the caller's other torch work.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Any

LIB_PATH = Path(__file__).resolve().parent / "libzkb200.so"

ZKB_OK = 0
ZKB_EINVAL = 1
ZKB_ETYPE = 2
ZKB_ECUDA = 3
ZKB_ENOTONCURVE = 4
ZKB_EWORKSPACE = 5
ZKB_ETIMEOUT = 6

FIELD_GENERIC = 0
FIELD_BN254_FR = 1
FIELD_BN254_FQ = 2


class ZkbField(ctypes.Structure):
    """zkb_field from include/zkb200.h: a prime field's Montgomery parameters."""

    _fields_ = [
        ("modulus", ctypes.c_uint64 * 4),
        ("one", ctypes.c_uint64 * 4),
        ("r2", ctypes.c_uint64 * 4),
        ("ninv", ctypes.c_uint64),
        ("kind", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ZkbMsmJob(ctypes.Structure):
    """zkb_msm_job from include/zkb200.h: one MSM of a batch (device pointers)."""

    _fields_ = [
        ("points", ctypes.c_void_p),
        ("scalars", ctypes.c_void_p),
        ("n", ctypes.c_int64),
        ("result", ctypes.c_void_p),
        ("window_size", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ZkbNttJob(ctypes.Structure):
    """zkb_ntt_job from include/zkb200.h: one transform of a batch (device pointers)."""

    _fields_ = [
        ("input", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n", ctypes.c_int64),
        ("invert", ctypes.c_int32),
        ("has_coset", ctypes.c_int32),
        ("coset", ctypes.c_uint64 * 4),
    ]


class ZkbIntPeaks(ctypes.Structure):
    """zkb_int_peaks from include/zkb200.h: measured integer issue rates of the device."""

    _fields_ = [
        ("madlo_per_clk_sm", ctypes.c_double), ("madlo_per_s", ctypes.c_double), ("madlo_mhz", ctypes.c_double),
        ("madwide_per_clk_sm", ctypes.c_double), ("madwide_per_s", ctypes.c_double),
        ("madwide_mhz", ctypes.c_double),
        ("montmul_per_clk_sm", ctypes.c_double), ("montmul_per_s", ctypes.c_double),
        ("montmul_mhz", ctypes.c_double),
        ("sms", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


_u64p = ctypes.c_void_p  # device pointers travel as plain addresses
_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_fp = ctypes.POINTER(ZkbField)
_jobp = ctypes.POINTER(ZkbMsmJob)
_nttjobp = ctypes.POINTER(ZkbNttJob)

# name -> (restype, argtypes); the full C ABI of include/zkb200.h
SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "zkb_last_error": (ctypes.c_char_p, []),
    "zkb_version": (ctypes.c_int, []),
    "zkb_field_init": (ctypes.c_int, [_fp, ctypes.POINTER(ctypes.c_uint64)]),
    "zkb_field_mul": (ctypes.c_int, [_fp, _u64p, _i64, _u64p, _i64, _u64p, _i64, _vp]),
    "zkb_field_add": (ctypes.c_int, [_fp, _u64p, _i64, _u64p, _i64, _u64p, _i64, _vp]),
    "zkb_field_sub": (ctypes.c_int, [_fp, _u64p, _i64, _u64p, _i64, _u64p, _i64, _vp]),
    "zkb_field_to_mont": (ctypes.c_int, [_fp, _u64p, _u64p, _i64, _vp]),
    "zkb_field_from_mont": (ctypes.c_int, [_fp, _u64p, _u64p, _i64, _vp]),
    "zkb_ntt_workspace_bytes": (ctypes.c_size_t, [_i64]),
    "zkb_ntt_wait_timeouts": (ctypes.c_uint64, []),
    "zkb_ntt": (
        ctypes.c_int,
        [_fp, _u64p, _u64p, _i64, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
         ctypes.POINTER(ctypes.c_uint64), _vp, ctypes.c_size_t, _vp],
    ),
    "zkb_ntt_batch_workspace_bytes": (ctypes.c_size_t, [_nttjobp, ctypes.c_int]),
    "zkb_ntt_batch": (ctypes.c_int, [_fp, _nttjobp, ctypes.c_int, _vp, ctypes.c_size_t, _vp, _vp]),
    "zkb_quotient_pointwise": (ctypes.c_int, [_u64p, _u64p, _u64p, _u64p, _u64p, _i64, _vp]),
    "zkb_ntt_cross_step": (
        ctypes.c_int,
        [_fp, _u64p, _u64p, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
         _u64p, _vp],
    ),
    "zkb_u64_mul": (ctypes.c_int, [_u64p, _u64p, _u64p, _i64, _i64, _vp]),
    "zkb_u64_add": (ctypes.c_int, [_u64p, _u64p, _u64p, _i64, _i64, _vp]),
    "zkb_u64_pow": (ctypes.c_int, [_u64p, _u64p, _i64, _u64p, ctypes.c_int, _i64, _vp]),
    "zkb_ntt64_workspace_bytes": (ctypes.c_size_t, [_i64]),
    "zkb_ntt64": (ctypes.c_int, [_u64p, _u64p, _i64, _i64, _i64, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "zkb_g1_add": (ctypes.c_int, [_u64p, _i64, _u64p, _i64, _u64p, _i64, _vp]),
    "zkb_g1_add_affine": (ctypes.c_int, [_u64p, _i64, _u64p, _i64, _u64p, _i64, _vp]),
    "zkb_g1_double": (ctypes.c_int, [_u64p, _u64p, _i64, _vp]),
    "zkb_g1_to_affine": (ctypes.c_int, [_u64p, _u64p, _i64, _vp]),
    "zkb_g1_check_affine": (ctypes.c_int, [_u64p, _i64, _u64p, _vp]),
    "zkb_g1_mul_generator": (ctypes.c_int, [_u64p, _u64p, _i64, _vp]),
    "zkb_msm_default_window": (ctypes.c_int, [_i64]),
    "zkb_msm_workspace_bytes": (ctypes.c_size_t, [_i64, ctypes.c_int]),
    "zkb_msm": (ctypes.c_int, [_u64p, _u64p, _i64, ctypes.c_int, _u64p, _vp, ctypes.c_size_t, _vp]),
    "zkb_msm_no_alloc": (ctypes.c_int, [_u64p, _u64p, _i64, ctypes.c_int, _u64p, _vp]),
    "zkb_msm_no_alloc_capacity": (ctypes.c_size_t, []),
    "zkb_msm_batch_workspace_bytes": (ctypes.c_size_t, [_jobp, ctypes.c_int]),
    "zkb_msm_batch": (ctypes.c_int, [_jobp, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "zkb_msm_table_bytes": (ctypes.c_size_t, [_i64, ctypes.c_int]),
    "zkb_msm_table_build": (ctypes.c_int, [_u64p, _i64, ctypes.c_int, _u64p, _vp]),
    "zkb_msm_fixed_batch_workspace_bytes": (ctypes.c_size_t, [_jobp, ctypes.c_int]),
    "zkb_msm_fixed_batch": (ctypes.c_int, [_jobp, ctypes.c_int, _vp, ctypes.c_size_t, _vp]),
    "zkb_launch_count": (ctypes.c_uint64, []),
    "zkb_measure_int_peaks": (ctypes.c_int, [ctypes.POINTER(ZkbIntPeaks), _vp]),
    "zkb_tune_set": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "zkb_tune_get": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "zkb_tune_set_sized": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "zkb_tune_get_sized": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "zkb_profile_enable": (None, [ctypes.c_int]),
    "zkb_profile_report": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
}

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded library with every signature declared; RuntimeError if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built: run `python zk-gpu-accelerator_b200/build.py` "
                "(needs nvcc); this package has no CPU fallback"
            )
        handle = ctypes.CDLL(os.fspath(LIB_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().zkb_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = "") -> None:
    """Raise the reference's exception type for a non-zero status."""
    if status == ZKB_OK:
        return
    msg = last_error() or f"{what} failed with status {status}"
    if status in (ZKB_EINVAL, ZKB_ENOTONCURVE, ZKB_EWORKSPACE):
        raise ValueError(msg)
    if status == ZKB_ETYPE:
        raise TypeError(msg)
    raise RuntimeError(msg)


# ------------------------------------------------------------------
# Device plumbing (torch)
# ------------------------------------------------------------------

_torch: Any = None


def torch_module() -> Any:
    global _torch
    if _torch is None:
        import torch

        _torch = torch
    return _torch


def require_cuda() -> Any:
    """torch, after checking that a CUDA device is present (no CPU fallback exists)."""
    torch = torch_module()
    if not torch.cuda.is_available():
        raise RuntimeError(
            "zkgpu needs a CUDA device (an NVIDIA B200, sm_100a): no GPU is visible and this "
            "package has no CPU fallback"
        )
    lib()
    return torch


def stream_ptr() -> int:
    """Raw cudaStream_t of torch's current stream."""
    return int(torch_module().cuda.current_stream().cuda_stream)


def ptr(t: Any) -> int:
    return int(t.data_ptr())


def u64_array(values: list[int] | tuple[int, ...]) -> Any:
    """A ctypes uint64[4] for a 256-bit host integer given as 4 limbs."""
    return (ctypes.c_uint64 * 4)(*values)


def limbs(value: int) -> list[int]:
    return [(value >> (64 * j)) & (2**64 - 1) for j in range(4)]


def make_field(modulus: int) -> ZkbField:
    """zkb_field for *modulus* (validated by the library: odd, in [3, 2^255))."""
    f = ZkbField()
    check(lib().zkb_field_init(ctypes.byref(f), u64_array(limbs(modulus))), "zkb_field_init")
    return f


def tune_set(key: str, value: int) -> None:
    """Set a tuning knob of the library (see zkb_tune_set in include/zkb200.h)."""
    check(lib().zkb_tune_set(key.encode(), int(value)), "zkb_tune_set")


def tune_get(key: str) -> int:
    v = ctypes.c_int(0)
    check(lib().zkb_tune_get(key.encode(), ctypes.byref(v)), "zkb_tune_get")
    return v.value


def tune_set_sized(key: str, log_n: int, value: int) -> None:
    """Set (value > 0) or clear (0) one entry of a per-size tuning table (zkb_tune_set_sized)."""
    check(lib().zkb_tune_set_sized(key.encode(), int(log_n), int(value)), "zkb_tune_set_sized")


def tune_get_sized(key: str, log_n: int) -> int:
    v = ctypes.c_int(0)
    check(lib().zkb_tune_get_sized(key.encode(), int(log_n), ctypes.byref(v)), "zkb_tune_get_sized")
    return v.value


def profile_enable(on: bool) -> None:
    """Start (clearing the record) or stop per-stage CUDA-event timing inside the library."""
    lib().zkb_profile_enable(int(bool(on)))


def profile_report() -> dict[str, tuple[int, float]]:
    """{stage: (launch count, total ms)} for the stages recorded since profile_enable(True)."""
    need = lib().zkb_profile_report(None, 0)
    buf = ctypes.create_string_buffer(need + 1)
    lib().zkb_profile_report(buf, need + 1)
    out: dict[str, tuple[int, float]] = {}
    for line in buf.value.decode().splitlines():
        name, count, ms = line.split()
        out[name] = (int(count), float(ms))
    return out


def measure_int_peaks() -> dict[str, float]:
    """Measured issue rates of the current device (zkb_measure_int_peaks) as a dict: per SM per
    clock, per second over the GPU, and the SM clock implied, for mad.lo.u32, mad.wide.u32 and the
    library's Montgomery product over BN254 Fq."""
    require_cuda()
    out = ZkbIntPeaks()
    check(lib().zkb_measure_int_peaks(ctypes.byref(out), stream_ptr()), "zkb_measure_int_peaks")
    return {name: getattr(out, name) for name, _ in ZkbIntPeaks._fields_ if name != "reserved"}


def workspace(nbytes: int) -> Any:
    """A device scratch buffer of *nbytes* bytes from torch's caching allocator.

    Allocated on the current stream for one call: torch hands the block out
    again only to work queued after this call on the same stream, so
    concurrent calls on different streams never share scratch memory.
    """
    torch = torch_module()
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")
