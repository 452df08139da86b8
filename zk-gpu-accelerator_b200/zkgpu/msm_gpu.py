"""
zkgpu.msm_gpu — Pippenger multi-scalar multiplication over BN254 G1 on a B200.

Drop-in for the reference's msm_pippenger_gpu (zkgpu/msm_gpu.py:398-449):
same arguments, validation, exceptions and result (an affine Point). Every
step runs on the GPU in libzkb200.so (csrc/msm.cu), including the two the
reference leaves on the CPU, the window combination and the conversion to
affine (zkgpu/msm.py:156-169, zkgpu/curve.py:221-233):

  1. points are converted to Montgomery form and checked on the curve
     (the reference validates each one with Point() on the host);
  2. scalars are reduced mod r and recoded into signed w-bit digits;
  3. (bucket, point) pairs are radix-sorted; buckets are summed with mixed
     XYZZ additions, in fixed-size runs per thread so skewed scalars
     (boolean witnesses, one heavy bucket) cost no more than uniform ones;
  4. each window's buckets are reduced by parallel running sums;
  5. the windows are combined by Horner's rule and the sum is made affine.

msm_pippenger_rows is the device-resident form of the same computation:
points already in (n, 2, 4) Montgomery rows (curve_gpu.affine_to_device, or
a resident base set) and scalars as (n, 4) limb rows.
"""

from __future__ import annotations

import operator
from collections.abc import Iterable
from typing import Any, SupportsIndex

import numpy as np

from zkgpu import _native, _rows
from zkgpu.curve import KNOWN_MULTIPLES, P as _BASE_MODULUS, R as _GROUP_ORDER, Point
from zkgpu.field256_gpu import BN254_FQ, LIMBS

_SCALAR_BITS = _GROUP_ORDER.bit_length()  # 254

# window_size accepted from callers, as the reference (zkgpu/msm.py:39, :124-129)
MAX_WINDOW_SIZE = 16

_SELF_TEST_FAILED = (
    "msm_gpu: the MSM kernels failed their self-test: libzkb200.so computes wrong sums on "
    "this GPU. Rebuild it for sm_100a (zk-gpu-accelerator_b200/build.py)."
)

_checked = False


def pippenger_window_size(n: int) -> int:
    """The reference's cost-model window (zkgpu/msm.py:112-121): argmin_w ceil(254/w)(n + 2^(w+1))."""
    n = operator.index(n)
    return min(range(1, MAX_WINDOW_SIZE + 1), key=lambda w: -(-_SCALAR_BITS // w) * (n + 2 ** (w + 1)))


def default_window_size(n: int) -> int:
    """The window this library uses when none is given (signed digits, 2^(w-1) buckets)."""
    return int(_native.lib().zkb_msm_default_window(operator.index(n)))


def _check_window_size(window_size: int) -> int:
    window_size = operator.index(window_size)
    if not 1 <= window_size <= MAX_WINDOW_SIZE:
        raise ValueError(f"window_size must be in 1..{MAX_WINDOW_SIZE}, got {window_size}")
    return window_size


def _as_ints(values: Iterable[SupportsIndex], name: str) -> list[int]:
    try:
        return [operator.index(v) for v in values]
    except TypeError as exc:
        raise TypeError(f"{name} must contain integers: {exc}") from None


def _ready() -> None:
    global _checked
    _native.require_cuda()
    if not _checked:
        _checked = True  # the self-test runs MSMs itself
        try:
            _self_test()
        except Exception:
            _checked = False
            raise


def _self_test() -> None:
    """
    A small MSM against a known answer, once per process. The inputs reach
    every branch: several points per bucket, P and -P in one bucket (they
    cancel), P twice in one bucket (doubling), digit-0 entries, scalars of
    every size up to r - 1, and w = 6 (43 windows).
    """
    g = Point(1, 2)
    pts = [g, Point(*KNOWN_MULTIPLES[2]), Point(*KNOWN_MULTIPLES[3]), -g, g, Point(*KNOWN_MULTIPLES[4]), g, -g, g]
    scalars = [1, 1, 1, 3, 2, _GROUP_ORDER - 1, 2**200 + 3, 2**200, 2]
    # 1 + 2 + 3 - 3 + 2 - 4 + (2^200 + 3) - 2^200 + 2 = 6
    got = msm_pippenger_gpu([p.x for p in pts], [p.y for p in pts], scalars, window_size=6)
    if got != Point(*KNOWN_MULTIPLES[6]):
        raise RuntimeError(_SELF_TEST_FAILED)


def compile_kernels() -> None:
    """Load the MSM kernels and run their self-test now instead of on first use."""
    _ready()


def _result_point(res: np.ndarray) -> Point:
    """The Point for the library's 9-word result (x, y plain limbs, infinity flag)."""
    if res[8]:
        return Point.identity()
    x, y = _rows.limbs_to_ints(res[:8].reshape(2, LIMBS))
    return Point(x, y)


def _launch(points: Any, scalars: Any, n: int, w: int | None, check_points: bool) -> Point:
    torch = _native.require_cuda()
    lib = _native.lib()
    stream = _native.stream_ptr()
    # one buffer for the result (9 words) and the first off-curve index (1 word)
    out = torch.empty(10, dtype=torch.int64, device="cuda")
    if check_points:
        _native.check(lib.zkb_g1_check_affine(_native.ptr(points), n, _native.ptr(out) + 72, stream))
    wsz = 0 if w is None else w
    ws_bytes = lib.zkb_msm_workspace_bytes(n, wsz)
    if ws_bytes == 0 and n > 0:
        raise RuntimeError(_native.last_error() or "zkb_msm_workspace_bytes failed")
    ws = _native.workspace(ws_bytes)
    _native.check(
        lib.zkb_msm(_native.ptr(points), _native.ptr(scalars), n, wsz, _native.ptr(out),
                    _native.ptr(ws), ws_bytes, stream)
    )
    raw = out.to("cpu").numpy()
    res = raw.view(np.uint64)
    if check_points:
        bad = int(raw[9])
        if bad >= 0:
            xy = BN254_FQ.to_ints(points[bad].reshape(2, LIMBS))
            raise ValueError(f"({xy[0]}, {xy[1]}) is not on the BN254 curve y^2 = x^3 + 3")
    return _result_point(res)


def msm_pippenger_rows(points: Any, scalars: Any, *, window_size: int | None = None,
                       check_points: bool = True) -> Point:
    """
    Sum s_i P_i for device-resident inputs.

    points   : (n, 2, 4) uint64 affine rows in Montgomery form over BN254_FQ
               (curve_gpu.affine_to_device's layout), on the device or host
    scalars  : (n, 4) uint64 little-endian limbs of plain integers below 2^256;
               reduced mod r on the device
    check_points : validate every point on the curve on the device first
               (ValueError naming the first bad one)
    """
    if window_size is not None:
        window_size = _check_window_size(window_size)
    if not _rows.shape_ok(points, (2, LIMBS)):
        raise TypeError(f"points must be an (n, 2, 4) uint64 array of affine points, got {_rows._describe(points)}")
    if not _rows.shape_ok(scalars, (LIMBS,)):
        raise TypeError(f"scalars must be an (n, 4) uint64 array of limbs, got {_rows._describe(scalars)}")
    n = int(points.shape[0])
    if int(scalars.shape[0]) != n:
        raise ValueError(f"Length mismatch: {n} points, {int(scalars.shape[0])} scalars.")
    _ready()
    if n == 0:
        return Point.identity()
    return _launch(_rows.to_device(points), _rows.to_device(scalars), n, window_size, check_points)


def msm_pippenger_affine(points: Any, scalars: Any, *, window_size: int | None = None) -> Point:
    """
    Sum s_i P_i for points given as plain affine coordinates in limb rows: the
    reference's msm_pippenger_gpu inputs (coordinates as integers) in bulk
    array form, without Python integers on the way in.

    points   : (n, 2, 4) uint64 little-endian limbs of x and y (any values below
               2^256; reduced mod P like Point()), on the host or the device
    scalars  : (n, 4) uint64 limbs of plain integers below 2^256 (reduced mod r)

    The coordinates go to Montgomery form and are checked on the curve on the
    device (ValueError naming the first point that is not on it).
    """
    if window_size is not None:
        window_size = _check_window_size(window_size)
    if not _rows.shape_ok(points, (2, LIMBS)):
        raise TypeError(f"points must be an (n, 2, 4) uint64 array of affine points, got {_rows._describe(points)}")
    if not _rows.shape_ok(scalars, (LIMBS,)):
        raise TypeError(f"scalars must be an (n, 4) uint64 array of limbs, got {_rows._describe(scalars)}")
    n = int(points.shape[0])
    if int(scalars.shape[0]) != n:
        raise ValueError(f"Length mismatch: {n} points, {int(scalars.shape[0])} scalars.")
    _ready()
    if n == 0:
        return Point.identity()
    mont = BN254_FQ.to_montgomery(_rows.to_device(points).reshape(-1, LIMBS)).reshape(n, 2, LIMBS)
    return _launch(mont, _rows.to_device(scalars), n, window_size, True)


def msm_pippenger_gpu(
    points_x: Iterable[int],
    points_y: Iterable[int],
    scalars: Iterable[int],
    *,
    window_size: int | None = None,
) -> Point:
    """
    Pippenger MSM over BN254 G1, every step on the GPU.

    Parameters
    ----------
    points_x, points_y : affine coordinates of the points (Python ints or an
                         object-dtype array); reduced mod P like Point()
    scalars            : any integers, including negative and >= 2^256; they
                         are reduced mod r, which leaves every s_i P_i unchanged
    window_size        : bits per window (w), 1..16; by default the library's
                         own choice for N (default_window_size). Signed digits
                         give each window 2^(w-1) buckets.

    Returns
    -------
    Point : sum s_i P_i, which is Point.identity() for the point at infinity

    Raises
    ------
    ValueError : if the three inputs differ in length, window_size is out of
                 range, or a point is not on the curve
    TypeError  : if a coordinate or scalar is not an integer
    """
    if window_size is not None:
        window_size = _check_window_size(window_size)
    xs, ys = _as_ints(points_x, "points_x"), _as_ints(points_y, "points_y")
    reduced = [s % _GROUP_ORDER for s in _as_ints(scalars, "scalars")]
    if not len(xs) == len(ys) == len(reduced):
        raise ValueError(
            f"Length mismatch: {len(xs)} x-coordinates, {len(ys)} y-coordinates, {len(reduced)} scalars."
        )
    if not reduced:
        return Point.identity()
    _ready()
    n = len(reduced)
    coords = [c % _BASE_MODULUS for xy in zip(xs, ys, strict=True) for c in xy]
    plain = _rows.upload(_rows.ints_to_limbs(coords))
    points = BN254_FQ.to_montgomery(plain).reshape(n, 2, LIMBS)
    sc = _rows.upload(_rows.ints_to_limbs(reduced))
    return _launch(points, sc, n, window_size, True)


# ------------------------------------------------------------------
# Fixed-base tables: many MSMs over one resident base set
# ------------------------------------------------------------------

TABLE_WINDOWS = range(8, 25)


class FixedBaseTable:
    """
    Per-window multiples of a resident base set, for many MSMs over it or over
    any prefix of it (a prover's SRS). There is no counterpart in the
    reference, whose MSM takes its points with every call.

    The table holds, for each point P_i, the rows 2^(w k) P_i and phi(2^(w k) P_i)
    for the W = ceil(128 / w) windows of a GLV half (2 W x 64 bytes a point). An
    MSM over it adds every window's digits into one set of 2^(w-1) buckets, so
    it reduces one window instead of W and needs no doublings at the end; that
    leaves room for larger windows and so fewer mixed additions. Results equal
    msm_pippenger_rows over the same points.

    points      : (N, 2, 4) uint64 Montgomery affine rows of points on the curve
                  (not checked here: msm_pippenger_rows(..., check_points=True)
                  or curve_gpu's checks validate them), host or device
    window_size : 8..24 (default 20)
    """

    def __init__(self, points: Any, window_size: int = 20) -> None:
        w = operator.index(window_size)
        if w not in TABLE_WINDOWS:
            raise ValueError(f"window_size must be in {TABLE_WINDOWS.start}..{TABLE_WINDOWS.stop - 1}, got {w}")
        torch = _native.require_cuda()
        pts = _rows.to_device(points)
        if not _rows.shape_ok(pts, (2, LIMBS)):
            raise TypeError(f"points must be an (n, 2, 4) uint64 array of affine points, got {_rows._describe(pts)}")
        self.n = int(pts.shape[0])
        self.window_size = w
        lib = _native.lib()
        nbytes = int(lib.zkb_msm_table_bytes(self.n, w))
        self.table = torch.empty(max(nbytes // 8, 1), dtype=torch.uint64, device="cuda")
        if self.n:
            _native.check(lib.zkb_msm_table_build(_native.ptr(pts), self.n, w, _native.ptr(self.table),
                                                  _native.stream_ptr()), "zkb_msm_table_build")

    @property
    def nbytes(self) -> int:
        return int(self.table.numel()) * 8

    def msm(self, scalars: Any) -> Point:
        """sum s_i P_i over the first len(scalars) points of the table."""
        from zkgpu.batch import msm_fixed_batch

        return msm_fixed_batch(self, [scalars])[0]
