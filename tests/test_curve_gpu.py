"""
zkgpu.curve_gpu on the GPU: exact Jacobian coordinates against the
reference's golden outputs (its tests/test_curve_gpu.py cases, every special
case included), conversions, broadcasting, and the fixed-base generator
against the C oracle and the reference's bases.
"""

from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from conftest import golden, h, hs
from oracle import c_oracle as co
from oracle import pyoracle as po
from zkgpu import curve_gpu
from zkgpu import workloads as wl
from zkgpu.curve import JACOBIAN_IDENTITY, G, P, Point, R

pytestmark = pytest.mark.gpu


def jacs(rows: list[list[str]]) -> list[tuple[int, int, int]]:
    return [tuple(hs(j)) for j in rows]


def test_add_matches_the_references_jacobian_coordinates():
    g = golden("curve.json")["add"]
    got = curve_gpu.add(curve_gpu.jacobian_to_device(jacs(g["a"])), curve_gpu.jacobian_to_device(jacs(g["b"])))
    assert curve_gpu.jacobian_ints(got) == jacs(g["out"])


def test_add_affine_matches_the_references_jacobian_coordinates():
    g = golden("curve.json")["add_affine"]
    q = [Point(*hs(p)) for p in g["b"]]
    got = curve_gpu.add_affine(curve_gpu.jacobian_to_device(jacs(g["a"])), curve_gpu.affine_to_device(q))
    assert curve_gpu.jacobian_ints(got) == jacs(g["out"])


def test_double_matches_the_references_jacobian_coordinates():
    g = golden("curve.json")["double"]
    got = curve_gpu.double(curve_gpu.jacobian_to_device(jacs(g["a"])))
    assert curve_gpu.jacobian_ints(got) == jacs(g["out"])


def test_to_affine_matches_the_references():
    g = golden("curve.json")["to_affine"]
    got = curve_gpu.from_device(curve_gpu.jacobian_to_device(jacs(g["a"])))
    assert got == [Point(*hs(p)) for p in g["out"]]


def test_chained_doublings_and_additions():
    """2^10 G + 3 G, all on the device, equals 1027 G."""
    acc = curve_gpu.to_device([G])
    for _ in range(10):
        acc = curve_gpu.double(acc)
    acc = curve_gpu.add_affine(acc, curve_gpu.affine_to_device([Point(*po.scalar_mul(po.G, 3))]))
    assert curve_gpu.from_device(acc) == [Point(*po.scalar_mul(po.G, 1027))]


def test_points_round_trip():
    five = Point(*po.scalar_mul(po.G, 5))
    pts = [G, five, -G, Point.identity()]
    rows = curve_gpu.to_device(pts)
    assert tuple(rows.shape) == (4, 3, 4)
    assert curve_gpu.from_device(rows) == pts
    assert curve_gpu.jacobian_ints(rows)[3] == JACOBIAN_IDENTITY


def test_from_device_revalidates_points():
    rows = curve_gpu.jacobian_to_device([(1, 3, 1)])
    with pytest.raises(ValueError, match="not on the BN254 curve"):
        curve_gpu.from_device(rows)


def test_single_point_broadcasts_on_either_side():
    g = golden("curve.json")["add"]
    js = jacs(g["a"])[:3]
    rows, one = curve_gpu.jacobian_to_device(js), curve_gpu.to_device([G])
    gj = (1, 2, 1)
    assert curve_gpu.jacobian_ints(curve_gpu.add(rows, one)) == [po.jacobian_add(j, gj) for j in js]
    assert curve_gpu.jacobian_ints(curve_gpu.add(one, rows)) == [po.jacobian_add(gj, j) for j in js]
    got = curve_gpu.add_affine(rows, curve_gpu.affine_to_device([G]))
    assert curve_gpu.jacobian_ints(got) == [po.jacobian_add_affine(j, 1, 2) for j in js]


def test_empty_batches():
    empty = curve_gpu.to_device([])
    assert tuple(empty.shape) == (0, 3, 4)
    assert curve_gpu.from_device(curve_gpu.add(empty, empty)) == []
    assert curve_gpu.from_device(curve_gpu.double(empty)) == []


def test_malformed_rows_raise():
    affine = curve_gpu.affine_to_device([G])
    with pytest.raises(TypeError, match=r"\(n, 3, 4\) uint64 array of Jacobian points"):
        curve_gpu.add(affine, affine)
    with pytest.raises(TypeError, match=r"\(n, 2, 4\) uint64 array of affine points"):
        curve_gpu.add_affine(curve_gpu.to_device([G]), curve_gpu.to_device([G]))


def test_point_operators_run_on_the_gpu():
    three = Point(*po.scalar_mul(po.G, 3))
    assert G + G == Point(*po.scalar_mul(po.G, 2)) == G.double()
    assert G + three == Point(*po.scalar_mul(po.G, 4))
    assert G + (-G) == Point.identity()
    assert G * 1027 == Point(*po.scalar_mul(po.G, 1027))
    assert 5 * G == Point(*po.scalar_mul(po.G, 5))
    assert G * R == Point.identity()


def test_self_test_passes():
    curve_gpu.compile_kernels()


def test_mul_generator_matches_c_oracle():
    k = wl.base_scalars(77, 3000)
    k[0] = [1, 0, 0, 0]
    k[1] = [2, 0, 0, 0]
    got = curve_gpu.mul_generator(k).cpu().numpy()
    want = co.mul_generator(k, threads=os.cpu_count() or 1)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", golden("msm.json")["seeded"], ids=lambda c: f"{c['kind']}-{c['n']}")
def test_mul_generator_reproduces_the_references_bases(case):
    bases = curve_gpu.mul_generator(wl.base_scalars(case["base_seed"], case["n"])).cpu().numpy()
    assert hashlib.sha256(np.ascontiguousarray(bases, dtype="<u8").tobytes()).hexdigest() == case["bases_sha256"]
    x = po.from_mont(wl.rows_to_ints(bases[0:1, 0])[0], P)
    assert x == h(case["bases_first"][0])
