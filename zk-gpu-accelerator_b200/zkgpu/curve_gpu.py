"""
zkgpu.curve_gpu — BN254 G1 point arithmetic on a B200, in Jacobian coordinates.

Drop-in for the reference module of the same name (zkgpu/curve_gpu.py): the
same functions, row layouts, broadcasting and exceptions. The kernels
(libzkb200.so, csrc/curve.cuh) evaluate the reference's formulas (EFD
add-2007-bl, madd-2007-bl and dbl-2009-l for a = 0, with the same special
cases), so results are the reference's exact Jacobian coordinates, not
merely the same affine points.

Representation
--------------
- A batch of n Jacobian points is an (n, 3, 4) uint64 array: X, Y and Z, each
  a Montgomery-form BN254_FQ element. Z = 0 is the point at infinity, stored
  as (1, 1, 0).
- A batch of n affine points, the second operand of add_affine, is an
  (n, 2, 4) array of x and y; it cannot hold the point at infinity.
- Either operand of a binary operation may be a single point, broadcast
  against the other.
"""

from __future__ import annotations

from collections.abc import Iterable
from typing import Any

from zkgpu import _native, _rows
from zkgpu.curve import JACOBIAN_IDENTITY, KNOWN_MULTIPLES as _KNOWN_MULTIPLES, Jacobian, Point, to_jacobian
from zkgpu.field256_gpu import BN254_FQ, LIMBS

_SELF_TEST_FAILED = (
    "curve_gpu: the {op} kernel failed its self-test: libzkb200.so computes wrong points on "
    "this GPU. Rebuild it for sm_100a (zk-gpu-accelerator_b200/build.py)."
)

_checked = False


def cuda_source() -> str:
    """BN254_FQ's constants as #defines; the point code is csrc/curve.cuh in libzkb200.so."""
    return BN254_FQ.cuda_source() + "// point formulas: zk-gpu-accelerator_b200/csrc/curve.cuh\n"


def _ready() -> None:
    global _checked
    _native.require_cuda()
    if not _checked:
        _checked = True  # the self-test itself calls these functions
        try:
            _self_test()
        except Exception:
            _checked = False
            raise


def _self_test() -> None:
    """
    Check the kernels against known answers, once per process: doubling G,
    G + 2G (mixed and Jacobian), equal points (the doubling branch), inverse
    points (the identity) and the identity on either side.
    """
    g = Point(1, 2)
    two, three, four = (Point(*_KNOWN_MULTIPLES[k]) for k in (2, 3, 4))
    got = from_device(double(to_device([g, two, Point.identity()])))
    if got != [two, four, Point.identity()]:
        raise RuntimeError(_SELF_TEST_FAILED.format(op="double"))
    jac = to_device([g, two, g, Point.identity(), g])
    aff = affine_to_device([two, g, g, three, -g])
    got = from_device(add_affine(jac, aff))
    if got != [three, three, two, three, Point.identity()]:
        raise RuntimeError(_SELF_TEST_FAILED.format(op="add_affine"))
    a = to_device([g, two, g, Point.identity(), g])
    b = to_device([two, g, g, three, Point.identity()])
    got = from_device(add(a, b))
    if got != [three, three, two, three, g]:
        raise RuntimeError(_SELF_TEST_FAILED.format(op="add"))


def compile_kernels() -> None:
    """Load the point kernels and run their self-test now instead of on first use."""
    _ready()


# ------------------------------------------------------------------
# Conversion
# ------------------------------------------------------------------


def jacobian_to_device(points: Iterable[Jacobian]) -> Any:
    """(n, 3, 4) rows for Jacobian (X, Y, Z) int triples."""
    flat = [c for point in points for c in point]
    if len(flat) % 3:
        raise ValueError("Jacobian points must be (X, Y, Z) triples")
    return BN254_FQ.from_ints(flat).reshape(-1, 3, LIMBS)


def to_device(points: Iterable[Point]) -> Any:
    """(n, 3, 4) Jacobian rows for affine Points (Z = 1; the identity becomes (1, 1, 0))."""
    return jacobian_to_device(to_jacobian(p) for p in points)


def affine_to_device(points: Iterable[Point]) -> Any:
    """(n, 2, 4) affine rows, the second operand of add_affine; the identity is rejected."""
    flat: list[int] = []
    for p in points:
        if p.is_identity():
            raise ValueError("affine rows cannot hold the point at infinity; leave it out (it adds nothing)")
        flat.extend(p.affine())
    return BN254_FQ.from_ints(flat).reshape(-1, 2, LIMBS)


def jacobian_ints(x: Any) -> list[Jacobian]:
    """The exact (X, Y, Z) coordinates of Jacobian rows, as Python ints."""
    _point_count(x, "x", 3)
    flat = BN254_FQ.to_ints(x.reshape(-1, LIMBS))
    return [(flat[k], flat[k + 1], flat[k + 2]) for k in range(0, len(flat), 3)]


def from_device(x: Any) -> list[Point]:
    """Affine Points for Jacobian rows (one inversion per point on the GPU); each is
    re-validated on the curve by Point, so corrupted rows raise ValueError."""
    n = _point_count(x, "x", 3)
    _ready()
    if n == 0:
        return []
    src = _rows.to_device(x)
    out = _rows.empty((n, 2, LIMBS))
    _native.check(_native.lib().zkb_g1_to_affine(_native.ptr(src), _native.ptr(out), n, _native.stream_ptr()))
    coords = _rows.limbs_to_ints(_rows.download(out).reshape(-1, LIMBS))
    zs = _rows.download(src[:, 2, :])
    points = []
    for k in range(n):
        if not zs[k].any():
            points.append(Point.identity())
        else:
            points.append(Point(coords[2 * k], coords[2 * k + 1]))
    return points


def mul_generator(k: Any) -> Any:
    """
    (n, 2, 4) affine Montgomery rows of k_i G, for (n, 4) uint64 plain scalars k
    (each not 0 mod r): a base set built on the device, where the reference
    builds its bases with G * k on the CPU (zkgpu/curve.py:153-159).
    """
    if not _rows.shape_ok(k, (LIMBS,)):
        raise TypeError(f"k must be an (n, 4) uint64 array of scalar limbs, got {_rows._describe(k)}")
    n = int(k.shape[0])
    _ready()
    src = _rows.to_device(k)
    out = _rows.empty((n, 2, LIMBS))
    if n:
        _native.check(_native.lib().zkb_g1_mul_generator(_native.ptr(src), _native.ptr(out), n, _native.stream_ptr()))
    return out


# ------------------------------------------------------------------
# Arithmetic
# ------------------------------------------------------------------


def add(a: Any, b: Any) -> Any:
    """Element-wise a + b of Jacobian rows (either may be one broadcast point)."""
    return _launch_binary("zkb_g1_add", a, b, 3)


def add_affine(a: Any, b: Any) -> Any:
    """Element-wise a + b of Jacobian rows *a* and affine rows *b* (the cheaper mixed addition)."""
    return _launch_binary("zkb_g1_add_affine", a, b, 2)


def double(a: Any) -> Any:
    """Element-wise 2a of Jacobian rows."""
    n = _point_count(a, "a", 3)
    _ready()
    src = _rows.to_device(a)
    out = _rows.empty((n, 3, LIMBS))
    if n:
        _native.check(_native.lib().zkb_g1_double(_native.ptr(src), _native.ptr(out), n, _native.stream_ptr()))
    return out


# ------------------------------------------------------------------
# Internals
# ------------------------------------------------------------------


def _point_count(x: Any, name: str, coords: int) -> int:
    """Points in *x*, after checking it is an (n, coords, 4) uint64 array."""
    if not _rows.shape_ok(x, (coords, LIMBS)):
        kind = "Jacobian" if coords == 3 else "affine"
        raise TypeError(
            f"{name} must be an (n, {coords}, {LIMBS}) uint64 array of {kind} points, "
            f"got {_rows._describe(x)}"
        )
    return int(x.shape[0])


def _broadcast(a: Any, b: Any, b_coords: int) -> int:
    rows_a, rows_b = _point_count(a, "a", 3), _point_count(b, "b", b_coords)
    if rows_a == rows_b or rows_b == 1:
        return rows_a
    if rows_a == 1:
        return rows_b
    raise ValueError(f"cannot broadcast {rows_a} points against {rows_b} points")


def _launch_binary(fn: str, a: Any, b: Any, b_coords: int) -> Any:
    n = _broadcast(a, b, b_coords)
    _ready()
    da, db = _rows.to_device(a), _rows.to_device(b)
    out = _rows.empty((n, 3, LIMBS))
    if n:
        step_a = 1 if da.shape[0] > 1 else 0
        step_b = 1 if db.shape[0] > 1 else 0
        _native.check(
            getattr(_native.lib(), fn)(
                _native.ptr(da), step_a, _native.ptr(db), step_b, _native.ptr(out), n, _native.stream_ptr()
            )
        )
    return out


__all__ = [
    "JACOBIAN_IDENTITY",
    "add",
    "add_affine",
    "affine_to_device",
    "compile_kernels",
    "cuda_source",
    "double",
    "from_device",
    "jacobian_ints",
    "jacobian_to_device",
    "mul_generator",
    "to_device",
]
