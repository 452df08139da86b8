"""
zkgpu.field256_gpu — 256-bit prime-field arithmetic and the NTT on a B200.

Drop-in for the reference module of the same name (zkgpu/field256_gpu.py):
the same Field256 class, BN254_FR / BN254_FQ singletons and LIMBS, the same
row layout, broadcasting, return values and exceptions. The arithmetic runs
in libzkb200.so's hand-written sm_100a kernels (8 x 32-bit-limb Montgomery
CIOS with PTX carry chains; an NTT fused across stages in shared memory)
instead of NVRTC-compiled CuPy RawKernels.

Representation
--------------
A batch of n elements is an (n, 4) uint64 array, least significant limb
first, holding the Montgomery form a*R mod p with R = 2^256. Device arrays are
torch tensors of dtype torch.uint64 on the current CUDA device; inputs may be
torch tensors, NumPy uint64 arrays or any DLPack producer. Rows must be
canonical (below p) and are not re-checked on the GPU.

Contract (as the reference's)
-----------------------------
- The modulus must be odd and below 2^255.
- Either operand of a binary operation may be a single row, which broadcasts.
- There is no CPU fallback: without a CUDA device every method raises RuntimeError.
"""

from __future__ import annotations

import operator
from collections.abc import Iterable
from typing import Any

from zkgpu import _native, _rows
from zkgpu.curve import P as BN254_BASE_MODULUS, R as BN254_SCALAR_MODULUS
from zkgpu.roots import get_ntt_root

LIMBS = 4
_LIMB_BITS = 64
_R_BITS = LIMBS * _LIMB_BITS  # R = 2^256

_SELF_TEST_FAILED = (
    "{field!r}: the {op} kernel failed its self-test: libzkb200.so computes wrong field "
    "elements on this GPU. Rebuild it for sm_100a (zk-gpu-accelerator_b200/build.py)."
)


def _row_count(x: Any, name: str) -> int:
    """Rows of *x*, after checking it is an (n, 4) uint64 array of limbs."""
    if not _rows.shape_ok(x, (LIMBS,)):
        raise TypeError(
            f"{name} must be an (n, {LIMBS}) uint64 array from Field256.from_ints, "
            f"got {_rows._describe(x)}"
        )
    return int(x.shape[0])


def _broadcast_rows(a: Any, b: Any) -> int:
    rows_a, rows_b = _row_count(a, "a"), _row_count(b, "b")
    if rows_a == rows_b or rows_b == 1:
        return rows_a
    if rows_a == 1:
        return rows_b
    raise ValueError(f"cannot broadcast {rows_a} rows against {rows_b} rows")


class Field256:
    """
    Arithmetic modulo an odd *modulus* below 2^255 on (n, 4) uint64 limb arrays.

    BN254's two fields run kernels with the modulus compiled in; any other
    modulus runs the same kernels with the modulus passed at launch. Each
    instance self-tests the kernels against Python integers on first use.
    """

    def __init__(self, modulus: int) -> None:
        modulus = operator.index(modulus)
        if not (3 <= modulus < 2 ** (_R_BITS - 1) and modulus % 2 == 1):
            raise ValueError(f"modulus must be odd and in [3, 2^255), got {modulus}")
        self.modulus = modulus
        self._r2 = pow(2, 2 * _R_BITS, modulus)
        self._r_inv = pow(2**_R_BITS, -1, modulus)
        self._n_inv = -pow(modulus, -1, 2**_LIMB_BITS) % 2**_LIMB_BITS
        self._cfield: _native.ZkbField | None = None
        self._checked = False  # set once the self-test has passed
        self._checking = False

    def __repr__(self) -> str:
        return f"Field256({self.modulus:#x})"

    # ------------------------------------------------------------------
    # Plumbing
    # ------------------------------------------------------------------

    def _field(self) -> _native.ZkbField:
        if self._cfield is None:
            self._cfield = _native.make_field(self.modulus)
        return self._cfield

    def _ready(self) -> Any:
        """torch, once a device is present and the kernels passed their self-test."""
        torch = _native.require_cuda()
        if not self._checked and not self._checking:
            self._checking = True
            try:
                self._self_test()
                self._checked = True
            finally:
                self._checking = False
        return torch

    # ------------------------------------------------------------------
    # Conversion
    # ------------------------------------------------------------------

    def from_ints(self, values: Iterable[int]) -> Any:
        """Montgomery-form device rows for *values* (any ints; reduced mod the modulus first)."""
        reduced = [operator.index(v) % self.modulus for v in values]
        self._ready()
        plain = _rows.upload(_rows.ints_to_limbs(reduced))
        return self.to_montgomery(plain)

    def to_ints(self, x: Any) -> list[int]:
        """The values of Montgomery-form rows *x*, as Python ints in [0, modulus)."""
        n = _row_count(x, "x")
        self._ready()
        if n == 0:
            return []
        return _rows.limbs_to_ints(_rows.download(self.from_montgomery(x)))

    def to_montgomery(self, plain: Any) -> Any:
        """Montgomery rows for plain canonical limb rows (device or host), on the device."""
        n = _row_count(plain, "plain")
        self._ready()
        src = _rows.to_device(plain)
        out = _rows.empty((n, LIMBS))
        if n:
            _native.check(
                _native.lib().zkb_field_to_mont(
                    self._field(), _native.ptr(src), _native.ptr(out), n, _native.stream_ptr()
                )
            )
        return out

    def from_montgomery(self, x: Any) -> Any:
        """Plain canonical limb rows for Montgomery rows *x*, on the device."""
        n = _row_count(x, "x")
        self._ready()
        src = _rows.to_device(x)
        out = _rows.empty((n, LIMBS))
        if n:
            _native.check(
                _native.lib().zkb_field_from_mont(
                    self._field(), _native.ptr(src), _native.ptr(out), n, _native.stream_ptr()
                )
            )
        return out

    # ------------------------------------------------------------------
    # Arithmetic
    # ------------------------------------------------------------------

    def mul(self, a: Any, b: Any) -> Any:
        """Element-wise product of Montgomery-form rows (either may be one broadcast row)."""
        return self._binary("zkb_field_mul", a, b)

    def add(self, a: Any, b: Any) -> Any:
        """Element-wise sum of Montgomery-form rows (either may be one broadcast row)."""
        return self._binary("zkb_field_add", a, b)

    def sub(self, a: Any, b: Any) -> Any:
        """Element-wise difference a - b of Montgomery-form rows (either may be one broadcast row)."""
        return self._binary("zkb_field_sub", a, b)

    def _binary(self, fn: str, a: Any, b: Any) -> Any:
        n = _broadcast_rows(a, b)
        self._ready()
        da, db = _rows.to_device(a), _rows.to_device(b)
        out = _rows.empty((n, LIMBS))
        if n:
            step_a = 1 if da.shape[0] > 1 else 0
            step_b = 1 if db.shape[0] > 1 else 0
            _native.check(
                getattr(_native.lib(), fn)(
                    self._field(), _native.ptr(da), step_a, _native.ptr(db), step_b,
                    _native.ptr(out), n, _native.stream_ptr(),
                )
            )
        return out

    # ------------------------------------------------------------------
    # NTT
    # ------------------------------------------------------------------

    def ntt(self, x: Any, *, invert: bool = False, coset: int | None = None) -> Any:
        """
        Radix-2 NTT of Montgomery-form rows *x*; returns new rows, *x* is unchanged.

        Exactly the transform of the reference's zkgpu.ntt.ntt (same roots of
        unity w_n = g^((p-1)/n) for the smallest non-residue g, same natural
        output order), and so of Radix2Domain.fft / .ifft for BN254_FR.

        coset (an extension of the reference API): evaluate on the coset
        coset * H, as Radix2Domain.coset_fft does: the input is scaled by
        coset^j before a forward transform; with invert=True the result is
        scaled by coset^-j after the inverse transform (coset_ifft). The
        scaling is fused into the transform's first or last pass.

        Raises
        ------
        ValueError : if the row count is not a power of two, the modulus is
                     not an odd prime, or the row count does not divide modulus - 1
        """
        n = _row_count(x, "x")
        if n == 0:
            self._ready()
            return _rows.empty((0, LIMBS))
        if n & (n - 1):
            raise ValueError(f"NTT length must be a power of 2, got {n}")
        p = self.modulus
        omega = get_ntt_root(n, p)  # validates modulus and size before any work
        g = None
        if coset is not None:
            g = operator.index(coset) % p
            if g == 0:
                raise ValueError(f"coset offset {coset} must be non-zero")
        self._ready()
        src = _rows.to_device(x)
        out = _rows.empty((n, LIMBS))
        # BN254 Fr uses the library's built-in 2^28-th root (5^((r-1)/2^28)),
        # which yields the same w_n; other fields pass w_n explicitly.
        omega_arg = None if p == BN254_SCALAR_MODULUS else _native.u64_array(_native.limbs(omega))
        coset_arg = None if g is None else _native.u64_array(_native.limbs(g))
        ws_bytes = _native.lib().zkb_ntt_workspace_bytes(n)
        ws = _native.workspace(ws_bytes)
        _native.check(
            _native.lib().zkb_ntt(
                self._field(), _native.ptr(src), _native.ptr(out), n, int(bool(invert)),
                omega_arg, coset_arg, _native.ptr(ws), ws_bytes, _native.stream_ptr(),
            )
        )
        return out

    # ------------------------------------------------------------------
    # Source and self-test
    # ------------------------------------------------------------------

    def cuda_source(self) -> str:
        """
        This field's constants as C #defines: ZK_P0..3 (the modulus), ZK_ONE0..3
        (R mod p, Montgomery one) and ZK_NINV (-p^-1 mod 2^64), the names the
        reference's kernels use. The kernels themselves are precompiled in
        libzkb200.so (csrc/field.cuh holds their source).
        """
        defines = "".join(f"#define ZK_P{j} {limb:#x}ULL\n" for j, limb in enumerate(_native.limbs(self.modulus)))
        one = 2**_R_BITS % self.modulus
        defines += "".join(f"#define ZK_ONE{j} {limb:#x}ULL\n" for j, limb in enumerate(_native.limbs(one)))
        defines += f"#define ZK_NINV {self._n_inv:#x}ULL\n"
        return defines + "// device code: zk-gpu-accelerator_b200/csrc/field.cuh (zk_mont_mul -> zkb::fe_mul)\n"

    def compile(self) -> None:
        """Load the kernels and run their self-test now instead of on first use."""
        self._ready()

    def _self_test(self) -> None:
        """
        Check the kernels against Python ints, once per instance.

        Carry-heavy operands: zero, one, p - 1, and values with all-ones limbs
        (the reference's self-test operands, zkgpu/field256_gpu.py:434-464).
        """
        p = self.modulus
        a = [0, 1, 2, p - 1, p - 2, p // 2, (2**128 - 1) % p, (2**192 - 1) % p]
        b = [p - 1, p - 1, 3, p - 1, 5, p // 3, (2**64 - 1) % p, 2**254 % p]
        x, y = self.from_ints(a), self.from_ints(b)
        checks = {
            "mul": (self.mul(x, y), [u * v % p for u, v in zip(a, b, strict=True)]),
            "add": (self.add(x, y), [(u + v) % p for u, v in zip(a, b, strict=True)]),
            "sub": (self.sub(x, y), [(u - v) % p for u, v in zip(a, b, strict=True)]),
        }
        try:
            w = get_ntt_root(len(a), p)
        except ValueError:
            pass  # no NTT of this size modulo p
        else:
            n = len(a)
            expected = [sum(a[j] * pow(w, j * k, p) for j in range(n)) % p for k in range(n)]
            checks["ntt"] = (self.ntt(x), expected)
        for op, (rows, expected) in checks.items():
            if self.to_ints(rows) != expected:
                raise RuntimeError(_SELF_TEST_FAILED.format(field=self, op=op))


BN254_FR = Field256(BN254_SCALAR_MODULUS)  # scalar field r: NTT and polynomial arithmetic
BN254_FQ = Field256(BN254_BASE_MODULUS)  # base field p: curve point coordinates
