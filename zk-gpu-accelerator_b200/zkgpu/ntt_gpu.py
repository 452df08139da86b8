"""
zkgpu.ntt_gpu — NTT over prime fields of one 64-bit word (moduli below 2^63).

Drop-in for the reference's ntt_gpu (zkgpu/ntt_gpu.py:86-155): same
arguments, roots (g^((p-1)/n) for the smallest non-residue g, as
zkgpu/ntt.py:98-124, so the transform equals the CPU NTT element for
element), validation and exceptions; the result is a torch int64 CUDA
tensor. libzkb200.so (csrc/field64.cu, zkb_ntt64) runs it as a radix-2 DIT
on bit-reversed input in two to four passes over HBM: the first pass gathers
the bit-reversed rows of a tile and runs its first stages in shared memory,
each later pass runs the next stages on tiles of rows at stride 2^S (Shoup
products with precomputed quotients, in plain form), and the last pass
multiplies by n^-1 for an inverse. There is no CPU fallback.
"""

from __future__ import annotations

from typing import Any

from zkgpu import _native
from zkgpu.field_gpu import _device_int64
from zkgpu.roots import get_ntt_root

_INT64_MAX = 2**63 - 1


def ntt_gpu(a: Any, mod: int, invert: bool = False) -> Any:
    """
    NTT of the int64 values *a* (any values; reduced mod *mod* first) over the
    odd prime *mod* < 2^63 with len(a) a power of two dividing mod - 1; the
    inverse (scaled by n^-1) when *invert*.

    Raises ValueError: mod >= 2^63, or the length / modulus errors of the CPU NTT.
    """
    if mod > _INT64_MAX:
        raise ValueError(
            f"ntt_gpu works on int64 elements, so mod must be below 2^63, got {mod}; "
            "use Field256.ntt for larger moduli such as BN254's r"
        )
    torch = _native.require_cuda()
    x = _device_int64(a).reshape(-1).contiguous()
    n = int(x.numel())
    if n & (n - 1):  # lets n == 0 through
        raise ValueError(f"NTT length must be a power of 2, got {n}")
    if n == 0:
        return torch.empty(0, dtype=torch.int64, device="cuda")
    omega = get_ntt_root(n, mod)  # validates mod (odd prime) and n | mod - 1, as the CPU NTT
    if n == 1:
        return torch.remainder(x, mod)
    lib = _native.lib()
    out = torch.empty_like(x)
    ws_bytes = int(lib.zkb_ntt64_workspace_bytes(n))
    ws = _native.workspace(ws_bytes)
    _native.check(lib.zkb_ntt64(_native.ptr(x), _native.ptr(out), n, mod, omega, int(bool(invert)),
                                _native.ptr(ws), ws_bytes, _native.stream_ptr()), "zkb_ntt64")
    return out
