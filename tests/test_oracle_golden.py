"""
The oracle, pinned: both restatements (oracle.pyoracle, oracle.c_oracle)
against golden vectors produced by running the reference itself
(tests/golden/make_golden.py) and against the known answers in the
reference's own tests. CPU only; these make the oracle trustworthy before it
checks the GPU's results.
"""

from __future__ import annotations

import hashlib
import os
import random

import numpy as np
import pytest

from conftest import golden, h, hs
from oracle import c_oracle as co
from oracle import pyoracle as po
from zkgpu import workloads as wl

R, P = po.R, po.P


def limbs(vals: list[int]) -> np.ndarray:
    return np.array([[(v >> (64 * j)) & (2**64 - 1) for j in range(4)] for v in vals], dtype=np.uint64).reshape(-1, 4)


def ints(rows: np.ndarray) -> list[int]:
    return wl.rows_to_ints(rows)


def digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u8").tobytes()).hexdigest()


# ------------------------------------------------------------------
# Known answers (reference tests/test_field256_gpu.py:60-85, test_domain.py,
# test_curve.py:26-29, test_msm.py:170-171)
# ------------------------------------------------------------------


def test_montgomery_constants_match_gnark():
    k = golden("known.json")
    assert h(k["fr_ninv"]) == 0xC2E1F593EFFFFFFF == po.montgomery_constants(R)["n_inv"]
    assert h(k["fq_ninv"]) == 0x87D20782E4866389 == po.montgomery_constants(P)["n_inv"]
    assert h(k["fr_r2"]) == po.montgomery_constants(R)["r2"]
    one = 0x0E0A77C19A07DF2F666EA36F7879462E36FC76959F60CD29AC96341C4FFFFFFB
    assert hs(k["fr_one_row"]) == [(one >> (64 * j)) & (2**64 - 1) for j in range(4)]


def test_roots_match_snarkjs_and_arkworks():
    k = golden("known.json")
    assert h(k["root_2_28"]) == 19103219067921713944291392827692070036145651957329286315305642004821462161904
    assert po.get_ntt_root(2**28, R) == h(k["root_2_28"])
    assert h(k["root_2_28_generator_7"]) == 1748695177688661943023146337482803886740723238769601073607632802312037301404
    assert po.quadratic_non_residue(R) == k["qnr"]["r"] == 5
    assert po.quadratic_non_residue(998244353) == 3
    assert po.coset_offset(8) == k["coset_offset_fr"] == 5


def test_two_g_matches_py_ecc_and_r_g_is_identity():
    k = golden("known.json")
    two_g = (1368015179489954701390400359078579693043519447331113978918064868415326638035,
             9918110051302171585080402603319702774565515993150576347155970296011118125764)
    assert (h(k["two_g"][0]), h(k["two_g"][1])) == two_g == po.scalar_mul(po.G, 2)
    assert po.scalar_mul(po.G, R) is None


def test_window_size_cost_model():
    k = golden("known.json")
    for n, w in k["pippenger_window_size"].items():
        assert po.pippenger_window_size(int(n)) == w
    assert [po.pippenger_window_size(n) for n in (0, 100, 1_000, 10_000, 100_000)] == [1, 5, 7, 10, 13]


# ------------------------------------------------------------------
# Field
# ------------------------------------------------------------------


@pytest.mark.parametrize("modulus", list(golden("field.json").keys()))
def test_field_rows_match_reference(modulus):
    g = golden("field.json")[modulus]
    p = h(modulus)
    a, b = hs(g["a"]), hs(g["b"])
    c = po.montgomery_constants(p)
    assert h(g["n_inv"]) == c["n_inv"] and h(g["r2"]) == c["r2"]
    A = [po.to_mont(v, p) for v in a]
    B = [po.to_mont(v, p) for v in b]
    assert A == hs(g["a_rows"])
    assert [po.mont_mul(x, y, p) for x, y in zip(A, B)] == hs(g["mul_rows"])
    assert [(x + y) % p for x, y in zip(A, B)] == hs(g["add_rows"])
    assert [(x - y) % p for x, y in zip(A, B)] == hs(g["sub_rows"])


@pytest.mark.parametrize("modulus,fid", [(R, co.FR), (P, co.FQ)], ids=["r", "p"])
def test_c_oracle_field_matches_reference(modulus, fid):
    g = golden("field.json")[f"{modulus:x}"]
    A = co.to_mont(fid, limbs(hs(g["a"])))
    B = co.to_mont(fid, limbs(hs(g["b"])))
    assert ints(A) == hs(g["a_rows"])
    assert ints(co.field_op("mul", fid, A, B)) == hs(g["mul_rows"])
    assert ints(co.field_op("add", fid, A, B)) == hs(g["add_rows"])
    assert ints(co.field_op("sub", fid, A, B)) == hs(g["sub_rows"])
    assert ints(co.from_mont(fid, A)) == hs(g["a"])


# ------------------------------------------------------------------
# NTT
# ------------------------------------------------------------------


def _small_ntt_cases():
    return sorted(golden("ntt.json")["small"].items(), key=lambda kv: int(kv[0]))


@pytest.mark.parametrize("n,entry", _small_ntt_cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_ntt_oracles_match_reference(n, entry):
    n = int(n)
    rng = random.Random(n)  # the reference test's inputs (tests/test_field256_gpu.py:182)
    a = [rng.randrange(R) for _ in range(n)]
    X = co.to_mont(co.FR, limbs(a))
    g = entry["coset_offset"]
    outs = {
        "fwd": co.ntt(X),
        "inv": co.ntt(X, invert=True),
        "coset_fwd": co.ntt(X, coset=g, threads=2),
        "coset_inv": co.ntt(X, invert=True, coset=g, threads=2),
    }
    for key, rows in outs.items():
        if key in entry:
            expected = hs(entry[key])
            assert ints(co.from_mont(co.FR, rows)) == expected, key
            if n <= 64:
                py = {"fwd": po.ntt(a), "inv": po.ntt(a, invert=True),
                      "coset_fwd": po.coset_fft(a, g), "coset_inv": po.coset_ifft(a, g)}[key]
                assert py == expected, key
        elif key + "_sha256" in entry:
            assert digest(rows) == entry[key + "_sha256"], key


@pytest.mark.parametrize("n", ["65536", "1048576"])
def test_c_oracle_large_ntt_matches_reference(n):
    entry = golden("ntt.json")["large"].get(n)
    if entry is None:
        pytest.skip("fixture generated with --quick")
    rows = wl.uniform_fr(entry["seed"], int(n))
    X = co.to_mont(co.FR, rows)
    assert digest(X) == entry["input_sha256"]
    threads = os.cpu_count() or 1
    assert digest(co.ntt(X, threads=threads)) == entry["fwd_sha256"]
    assert digest(co.ntt(X, invert=True, threads=threads)) == entry["inv_sha256"]
    if "coset_fwd_sha256" in entry:
        assert digest(co.ntt(X, coset=5, threads=threads)) == entry["coset_fwd_sha256"]
        assert digest(co.ntt(X, coset=5, invert=True, threads=threads)) == entry["coset_inv_sha256"]


def test_domain_elements():
    for n, els in golden("ntt.json")["elements"].items():
        assert po.domain_elements(int(n)) == hs(els)


# ------------------------------------------------------------------
# Curve
# ------------------------------------------------------------------


def _jac_rows(js: list[list[str]]) -> np.ndarray:
    vals = [po.to_mont(h(c), P) for j in js for c in j]
    return limbs(vals).reshape(-1, 3, 4)


def _jac_ints(rows: np.ndarray) -> list[list[int]]:
    flat = ints(co.from_mont(co.FQ, rows.reshape(-1, 4)))
    return [flat[k : k + 3] for k in range(0, len(flat), 3)]


def test_curve_oracles_match_reference():
    g = golden("curve.json")
    add, mixed, dbl = g["add"], g["add_affine"], g["double"]
    # Python restatement
    for a, b, out in zip(add["a"], add["b"], add["out"]):
        assert list(po.jacobian_add(tuple(hs(a)), tuple(hs(b)))) == hs(out)
    for a, b, out in zip(mixed["a"], mixed["b"], mixed["out"]):
        assert list(po.jacobian_add_affine(tuple(hs(a)), *hs(b))) == hs(out)
    for a, out in zip(dbl["a"], dbl["out"]):
        assert list(po.jacobian_double(tuple(hs(a)))) == hs(out)
    # C restatement
    got = _jac_ints(co.g1_op("add", _jac_rows(add["a"]), _jac_rows(add["b"])))
    assert got == [hs(o) for o in add["out"]]
    aff = limbs([po.to_mont(h(c), P) for q in mixed["b"] for c in q]).reshape(-1, 2, 4)
    got = _jac_ints(co.g1_op("add_affine", _jac_rows(mixed["a"]), aff))
    assert got == [hs(o) for o in mixed["out"]]
    got = _jac_ints(co.g1_op("double", _jac_rows(dbl["a"])))
    assert got == [hs(o) for o in dbl["out"]]
    ta = g["to_affine"]
    out = co.g1_to_affine(_jac_rows(ta["a"]))
    assert [[*ints(r[:4].reshape(1, 4)), *ints(r[4:8].reshape(1, 4))] for r in out] == [hs(o) for o in ta["out"]]


# ------------------------------------------------------------------
# MSM
# ------------------------------------------------------------------


def _case_inputs(case):
    pts = [tuple(hs(p)) for p in case["points"]]
    sc = [int(s) for s in case["raw_scalars"]] if "raw_scalars" in case else hs(case["scalars"])
    exp = None if case["expected"] is None else tuple(hs(case["expected"]))
    return pts, sc, exp


@pytest.mark.parametrize("case", golden("msm.json")["cases"], ids=lambda c: c["name"])
def test_msm_oracles_match_reference(case):
    pts, sc, exp = _case_inputs(case)
    if len(pts) <= 30:
        assert po.msm_pippenger(pts, sc, 5) == exp
        assert po.msm_double_and_add(pts, [s % R for s in sc]) == exp
    rows = limbs([po.to_mont(c, P) for q in pts for c in q]).reshape(-1, 2, 4)
    for w in (1, 4, 9, 16):
        out = co.msm(rows, limbs([s % R for s in sc]), w, threads=4)
        got = None if out[8] else (ints(out[:4].reshape(1, 4))[0], ints(out[4:8].reshape(1, 4))[0])
        assert got == exp, w


def _seeded_cases():
    return golden("msm.json")["seeded"]


@pytest.mark.parametrize("case", _seeded_cases(), ids=lambda c: f"{c['kind']}-{c['n']}")
def test_c_oracle_seeded_msm_matches_reference(case):
    n = case["n"]
    threads = os.cpu_count() or 1
    bases = co.mul_generator(wl.base_scalars(case["base_seed"], n), threads=threads)
    assert digest(bases) == case["bases_sha256"]
    first = ints(co.from_mont(co.FQ, bases[0]))
    assert first == hs(case["bases_first"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    out = co.msm(bases, sc, po.pippenger_window_size(n), threads=threads)
    got = None if out[8] else [ints(out[:4].reshape(1, 4))[0], ints(out[4:8].reshape(1, 4))[0]]
    assert got == (None if case["expected"] is None else hs(case["expected"]))


# ------------------------------------------------------------------
# Workload generators
# ------------------------------------------------------------------


def test_uniform_fr_is_canonical_and_deterministic():
    a = wl.uniform_fr(7, 5000)
    assert np.array_equal(a, wl.uniform_fr(7, 5000))
    assert all(v < R for v in ints(a))
    assert len(set(ints(a[:1000]))) == 1000


def test_skewed_scalars_distribution():
    s = ints(wl.skewed_scalars(11, 20000))
    small = sum(v < 2 for v in s) / len(s)
    mid = sum(2 <= v < 2**32 for v in s) / len(s)
    assert 0.57 < small < 0.63 and 0.17 < mid < 0.23
    assert all(v < R for v in s)
