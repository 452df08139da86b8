"""
zkgpu._rows — host packing of 256-bit integers and device-array intake.

Rows are (n, 4) uint64 arrays of little-endian 64-bit limbs, 32 bytes per
element, exactly the reference's layout (zkgpu/field256_gpu.py:239-247). On
the device they are torch tensors of dtype torch.uint64; anything exposing
DLPack (a CuPy array, say) or a NumPy uint64 array is accepted on input and
moved to the current CUDA device.
"""

from __future__ import annotations

from collections.abc import Iterable
from typing import Any

import numpy as np

from zkgpu import _native

LIMBS = 4


def ints_to_limbs(values: Iterable[int]) -> np.ndarray:
    """(n, 4) uint64 array of 256-bit little-endian limbs; every value must be in [0, 2^256)."""
    buf = b"".join(v.to_bytes(32, "little") for v in values)
    return np.frombuffer(buf, dtype="<u8").astype(np.uint64).reshape(-1, LIMBS)


def limbs_to_ints(limbs: np.ndarray) -> list[int]:
    buf = np.ascontiguousarray(limbs, dtype="<u8").tobytes()
    return [int.from_bytes(buf[k : k + 32], "little") for k in range(0, len(buf), 32)]


def _describe(x: Any) -> str:
    dtype = getattr(x, "dtype", type(x).__name__)
    return f"{dtype} with shape {tuple(getattr(x, 'shape', ())) if hasattr(x, 'shape') else None}"


def _is_uint64(x: Any) -> bool:
    dtype = getattr(x, "dtype", None)
    if dtype is None:
        return False
    torch = _native.torch_module()
    if isinstance(dtype, torch.dtype):
        return dtype == torch.uint64
    try:
        return np.dtype(dtype) == np.uint64
    except TypeError:
        return False


def shape_ok(x: Any, inner: tuple[int, ...]) -> bool:
    """True if *x* is a uint64 array of shape (n, *inner)."""
    if not _is_uint64(x):
        return False
    shape = tuple(getattr(x, "shape", ()))
    return len(shape) == 1 + len(inner) and shape[1:] == inner


def to_device(x: Any) -> Any:
    """*x* (already shape-checked) as a contiguous torch uint64 tensor on the current CUDA device."""
    torch = _native.require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
    elif isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x))
    elif hasattr(x, "__dlpack__"):
        t = torch.from_dlpack(x)
    else:  # pragma: no cover - shape_ok already rejected it
        raise TypeError(f"cannot use {type(x).__name__} as device rows")
    if t.device.type != "cuda":
        t = t.to("cuda", non_blocking=False)
    return t.contiguous()


def empty(shape: tuple[int, ...]) -> Any:
    torch = _native.require_cuda()
    return torch.empty(shape, dtype=torch.uint64, device="cuda")


def upload(host: np.ndarray) -> Any:
    """A host uint64 array copied to the current CUDA device."""
    torch = _native.require_cuda()
    return torch.from_numpy(np.ascontiguousarray(host)).to("cuda")


def download(t: Any) -> np.ndarray:
    """A device tensor copied back to a host uint64 NumPy array (synchronises its stream)."""
    return t.detach().to("cpu").numpy()
