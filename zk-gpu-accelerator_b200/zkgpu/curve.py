"""
zkgpu.curve — BN254 G1 points as values: the type msm_pippenger_gpu returns.

The curve is y^2 = x^3 + 3 over F_P, with generator G = (1, 2)
(zkgpu/curve.py:28-38 of the reference). Point is an immutable, validated
affine point exactly like the reference's (zkgpu/curve.py:51-179):
coordinates are reduced into [0, P) and must satisfy the curve equation,
(None, None) is the point at infinity, and equal points compare and hash
equal. Rejecting off-curve input matters for security, not just tidiness:
the addition formulas never use B, so an off-curve "point" silently
computes on a different curve.

Group arithmetic on points (+ and *) runs on the GPU through
zkgpu.curve_gpu and zkgpu.msm_gpu; this module itself only validates.
"""

from __future__ import annotations

import operator
from dataclasses import dataclass

# BN254 base field prime (field of definition of the curve)
P: int = 21888242871839275222246405745257275088696311157297823662689037894645226208583
# Order r of G1, which is also the scalar field (zkgpu/field.py:17 of the reference)
R: int = 21888242871839275222246405745257275088548364400416034343698204186575808495617

A: int = 0
B: int = 3
GX: int = 1
GY: int = 2

Jacobian = tuple[int, int, int]
JACOBIAN_IDENTITY: Jacobian = (1, 1, 0)


@dataclass(frozen=True, slots=True)
class Point:
    """
    Affine point on BN254 G1; the point at infinity is (None, None).

    Raises
    ------
    ValueError : if exactly one coordinate is None, or (x, y) is not on the curve
    TypeError  : if a coordinate is not an integer
    """

    x: int | None
    y: int | None

    def __post_init__(self) -> None:
        if self.x is None and self.y is None:
            return
        if self.x is None or self.y is None:
            raise ValueError(f"only the identity has None coordinates, got ({self.x}, {self.y})")
        object.__setattr__(self, "x", operator.index(self.x) % P)
        object.__setattr__(self, "y", operator.index(self.y) % P)
        if not self.is_on_curve():
            raise ValueError(f"({self.x}, {self.y}) is not on the BN254 curve y^2 = x^3 + 3")

    @staticmethod
    def identity() -> Point:
        return Point(None, None)

    def is_identity(self) -> bool:
        return self.x is None and self.y is None

    def affine(self) -> tuple[int, int]:
        """(x, y) of a finite point; raises ValueError for the identity."""
        if self.x is None or self.y is None:
            raise ValueError("the point at infinity has no affine coordinates")
        return self.x, self.y

    def is_on_curve(self) -> bool:
        if self.is_identity():
            return True
        x, y = self.affine()
        return (y * y - pow(x, 3, P) - B) % P == 0

    def __neg__(self) -> Point:
        if self.is_identity():
            return Point.identity()
        x, y = self.affine()
        return Point(x, -y % P)

    # Group operations run on the GPU (one small launch each).

    def __add__(self, other: object) -> Point:
        if not isinstance(other, Point):
            return NotImplemented
        if other.is_identity():
            return self
        if self.is_identity():
            return other
        from zkgpu import curve_gpu

        total = curve_gpu.add_affine(curve_gpu.to_device([self]), curve_gpu.affine_to_device([other]))
        return curve_gpu.from_device(total)[0]

    def double(self) -> Point:
        from zkgpu import curve_gpu

        return curve_gpu.from_device(curve_gpu.double(curve_gpu.to_device([self])))[0]

    def __mul__(self, scalar: int) -> Point:
        try:
            scalar = operator.index(scalar)
        except TypeError:
            return NotImplemented
        if self.is_identity():
            return self
        from zkgpu.msm_gpu import msm_pippenger_gpu

        x, y = self.affine()
        return msm_pippenger_gpu([x], [y], [scalar])

    def __rmul__(self, scalar: int) -> Point:
        return self.__mul__(scalar)

    def __repr__(self) -> str:
        if self.is_identity():
            return "Point(∞)"
        return f"Point(x={self.x}, y={self.y})"


G: Point = Point(GX, GY)

# Known answers for the load-time self-tests: k*G in affine form, computed
# independently of this code (2G is py_ecc's published value for alt_bn128).
KNOWN_MULTIPLES: dict[int, tuple[int, int]] = {
    2: (
        1368015179489954701390400359078579693043519447331113978918064868415326638035,
        9918110051302171585080402603319702774565515993150576347155970296011118125764,
    ),
    3: (
        3353031288059533942658390886683067124040920775575537747144343083137631628272,
        19321533766552368860946552437480515441416830039777911637913418824951667761761,
    ),
    4: (
        3010198690406615200373504922352659861758983907867017329644089018310584441462,
        4027184618003122424972590350825261965929648733675738730716654005365300998076,
    ),
    5: (
        10744596414106452074759370245733544594153395043370666422502510773307029471145,
        848677436511517736191562425154572367705380862894644942948681172815252343932,
    ),
    6: (
        4503322228978077916651710446042370109107355802721800704639343137502100212473,
        6132642251294427119375180147349983541569387941788025780665104001559216576968,
    ),
    7: (
        10415861484417082502655338383609494480414113902179649885744799961447382638712,
        10196215078179488638353184030336251401353352596818396260819493263908881608606,
    ),
    8: (
        3932705576657793550893430333273221375907985235130430286685735064194643946083,
        18813763293032256545937756946359266117037834559191913266454084342712532869153,
    ),
}


def to_jacobian(point: Point) -> Jacobian:
    """Jacobian form of an affine point (Z = 1, or (1, 1, 0) for the identity)."""
    if point.is_identity():
        return JACOBIAN_IDENTITY
    x, y = point.affine()
    return (x, y, 1)
