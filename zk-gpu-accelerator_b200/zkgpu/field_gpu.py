"""
zkgpu.field_gpu — element-wise arithmetic over prime fields whose elements
fit one 64-bit word (moduli below 2^63), on the GPU.

Drop-in for the reference's int64 module (zkgpu/field_gpu.py): the same
functions, arguments, validation and exceptions. Results are torch int64
CUDA tensors (CuPy arrays in the reference); inputs may be torch tensors,
NumPy arrays or any DLPack producer of an integer dtype, and broadcast like
array arithmetic. Every element is computed by libzkb200.so (csrc/field64.cu):
Montgomery products with R = 2^64 for odd moduli, exact 128-bit remainders
for even ones. There is no CPU fallback.

Contract (as the reference's):
- 2 <= mod < 2^63;
- inputs are any integer values, reduced into [0, mod) first (negative ones
  land in the field); results lie in [0, mod);
- a negative exponent in gpu_batch_pow raises the inverse (Fermat, so mod
  must be prime) and refuses a base that is 0 mod `mod`.
"""

from __future__ import annotations

import operator
from typing import Any

import numpy as np

from zkgpu import _native

_INT64_MAX = 2**63 - 1


def _check_modulus(mod: Any) -> int:
    """*mod* as an int, or ValueError / TypeError if it cannot be an int64 field modulus."""
    mod = operator.index(mod)  # rejects floats such as 7.0 instead of truncating them
    if not 2 <= mod <= _INT64_MAX:
        raise ValueError(f"mod must satisfy 2 <= mod < 2^63 to fit in int64, got {mod}")
    return mod


def _dtype_kind(x: Any) -> str:
    torch = _native.torch_module()
    if isinstance(x, torch.Tensor):
        if x.dtype == torch.bool:
            return "b"
        if x.dtype.is_floating_point or x.dtype.is_complex:
            return "f"
        return "i"
    return np.dtype(x.dtype if hasattr(x, "dtype") else np.asarray(x).dtype).kind


def _check_integer_array(x: Any, name: str) -> None:
    """Non-integer arrays would be truncated silently: refuse them."""
    kind = _dtype_kind(x)
    if kind not in "iu":
        raise TypeError(f"{name} must be an integer array, got dtype {getattr(x, 'dtype', type(x).__name__)}")


def _device_int64(x: Any) -> Any:
    torch = _native.require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
    elif hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
        t = torch.from_dlpack(x)
    else:
        arr = np.asarray(x)
        t = torch.from_numpy(np.ascontiguousarray(arr.astype(np.int64, copy=False)))
    if t.dtype != torch.int64:
        # uint64 values of 2^63 and above wrap as they do in a C cast (the reference's astype)
        t = t.view(torch.int64) if t.dtype == torch.uint64 else t.to(torch.int64)
    return t.to("cuda")


def _binary(a: Any, b: Any, mod: Any, entry: str) -> Any:
    mod = _check_modulus(mod)
    _check_integer_array(a, "a")
    _check_integer_array(b, "b")
    torch = _native.require_cuda()
    x, y = torch.broadcast_tensors(_device_int64(a), _device_int64(b))
    x, y = x.contiguous(), y.contiguous()
    out = torch.empty_like(x)
    if out.numel():
        _native.check(getattr(_native.lib(), entry)(_native.ptr(x), _native.ptr(y), _native.ptr(out), out.numel(),
                                                   mod, _native.stream_ptr()), entry)
    return out


def gpu_batch_mul(a: Any, b: Any, mod: int) -> Any:
    """
    Element-wise modular multiplication: result[i] = (a[i] * b[i]) % mod.

    a, b : integer arrays (any values; reduced mod *mod* first), broadcast together
    mod  : 2 <= mod < 2^63

    Returns an int64 CUDA tensor with every element in [0, mod).
    ValueError if *mod* is outside [2, 2^63); TypeError if *mod* is not an
    integer or an input is not an integer array.
    """
    return _binary(a, b, mod, "zkb_u64_mul")


def gpu_batch_add(a: Any, b: Any, mod: int) -> Any:
    """Element-wise modular addition: result[i] = (a[i] + b[i]) % mod. Same contract as gpu_batch_mul."""
    return _binary(a, b, mod, "zkb_u64_add")


def gpu_batch_pow(bases: Any, exp: int, mod: int) -> Any:
    """
    Element-wise modular exponentiation: result[i] = bases[i]^exp % mod.

    A negative *exp* raises the inverse (a^-1 = a^(mod-2)) to |exp|, so *mod*
    must be prime; ValueError if some base is 0 mod *mod* then, as Python's pow().
    """
    mod = _check_modulus(mod)
    exp = operator.index(exp)
    _check_integer_array(bases, "bases")
    torch = _native.require_cuda()
    x = _device_int64(bases).contiguous()
    out = torch.empty_like(x)
    if exp < 0:
        if bool((torch.remainder(x, mod) == 0).any()):
            raise ValueError("base is not invertible for the given modulus")
        exp = (mod - 2) * (-exp)
    words = []
    while exp:
        words.append(exp & (2**64 - 1))
        exp >>= 64
    w = torch.from_numpy(np.array(words or [0], dtype=np.uint64).view(np.int64)).cuda()
    if out.numel():
        _native.check(_native.lib().zkb_u64_pow(_native.ptr(x), _native.ptr(out), out.numel(), _native.ptr(w),
                                                len(words), mod, _native.stream_ptr()), "zkb_u64_pow")
    return out
